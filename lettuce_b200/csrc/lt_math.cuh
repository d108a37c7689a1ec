// SU(3)/SU(2) arithmetic for the B200 kernels: 3x3 complex matrices in registers,
// Cabibbo-Marinari SU(2) subgroups, Gram-Schmidt reunitarisation, the Cayley-Hamilton
// exponential and its Morningstar-Peardon derivative coefficients, and the Philox4x32-10
// counter-based generator.  Everything is templated on the link arithmetic type T (float or
// double); the scalar coefficient chain of the exponential always runs in double.
//
// Reference semantics (timo-eichhorn/Lettuce, LettuceGauge/...):
//   Algebra / TracelessHermitian      math/su3.hpp:423-448
//   GramSchmidt / RestoreLastRow      math/su3.hpp:362-394
//   Extract0x / Embed0x / SU2_comp    math/su2.hpp:21-174
//   ExpConstants / SU3::exp           math/su3_exp.hpp:204-283, :419-432
//   ExpDerivativeConstants (r, b, B)  math/su3_exp.hpp:121-201, :389-415
#pragma once
#include <cstdint>
#include <cfloat>
#include <cuda_runtime.h>

#define LT_HD __host__ __device__ __forceinline__
#define LT_D __device__ __forceinline__

namespace lt {

template <typename T> struct __align__(2 * sizeof(T)) cx { T r, i; };

template <typename T> LT_HD cx<T> mkc(T r, T i) { cx<T> c; c.r = r; c.i = i; return c; }
template <typename T> LT_HD cx<T> operator+(cx<T> a, cx<T> b) { return mkc<T>(a.r + b.r, a.i + b.i); }
template <typename T> LT_HD cx<T> operator-(cx<T> a, cx<T> b) { return mkc<T>(a.r - b.r, a.i - b.i); }
template <typename T> LT_HD cx<T> operator-(cx<T> a) { return mkc<T>(-a.r, -a.i); }
template <typename T> LT_HD cx<T> operator*(cx<T> a, cx<T> b) { return mkc<T>(a.r * b.r - a.i * b.i, a.r * b.i + a.i * b.r); }
template <typename T> LT_HD cx<T> operator*(T s, cx<T> a) { return mkc<T>(s * a.r, s * a.i); }
template <typename T> LT_HD cx<T> conj(cx<T> a) { return mkc<T>(a.r, -a.i); }
// a * conj(b)
template <typename T> LT_HD cx<T> mulc(cx<T> a, cx<T> b) { return mkc<T>(a.r * b.r + a.i * b.i, a.i * b.r - a.r * b.i); }
// i * a
template <typename T> LT_HD cx<T> timesi(cx<T> a) { return mkc<T>(-a.i, a.r); }
template <typename T> LT_HD T norm2(cx<T> a) { return a.r * a.r + a.i * a.i; }
template <typename To, typename From> LT_HD cx<To> cvt(cx<From> a) { return mkc<To>((To)a.r, (To)a.i); }

template <typename T> struct M3 { cx<T> e[3][3]; };

template <typename T> LT_HD M3<T> zero3()
{
    M3<T> r;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) r.e[i][j] = mkc<T>(0, 0);
    return r;
}

template <typename T> LT_HD M3<T> unit3()
{
    M3<T> r = zero3<T>();
    r.e[0][0].r = r.e[1][1].r = r.e[2][2].r = 1;
    return r;
}

// Matrix products with optional adjoints, (A^[dag] B^[dag])_ij, written as explicit FMA
// chains: each complex term adds two fused multiply-adds to each running sum.  (A single
// expression like `re += a*b - c*d` would cost a multiply, an FMA and an add per term,
// since the compiler may not reassociate it.)  ROWS < 3 computes only the leading rows.
// RA / RB: the diagonal of a / b is known to be real (a Hermitian factor), so the products with
// its zero imaginary parts are left out (the compiler may not drop a multiplication by 0.0).
template <bool DA, bool DB, int ROWS = 3, bool RA = false, bool RB = false, typename T>
LT_HD M3<T> prod(const M3<T>& a, const M3<T>& b)
{
    M3<T> r;
#pragma unroll
    for (int i = 0; i < ROWS; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
        {
            T re = 0, im = 0;
#pragma unroll
            for (int k = 0; k < 3; ++k)
            {
                const bool xreal = RA && k == i, yreal = RB && k == j;
                const T xr = DA ? a.e[k][i].r : a.e[i][k].r;
                const T xi = DA ? -a.e[k][i].i : a.e[i][k].i;
                const T yr = DB ? b.e[j][k].r : b.e[k][j].r;
                const T yi = DB ? -b.e[j][k].i : b.e[k][j].i;
                re += xr * yr;
                if (!xreal && !yreal) re -= xi * yi;
                if (!yreal) im += xr * yi;
                if (!xreal) im += xi * yr;
            }
            r.e[i][j] = mkc<T>(re, im);
        }
    return r;
}

// A * B
template <typename T> LT_HD M3<T> mul(const M3<T>& a, const M3<T>& b) { return prod<false, false>(a, b); }
// Products with a Hermitian factor H (real diagonal): H X, X H, U^dagger H, H U^dagger
template <typename T> LT_HD M3<T> mul_hx(const M3<T>& h, const M3<T>& b) { return prod<false, false, 3, true, false>(h, b); }
template <typename T> LT_HD M3<T> mul_xh(const M3<T>& a, const M3<T>& h) { return prod<false, false, 3, false, true>(a, h); }
template <typename T> LT_HD M3<T> mul_dh(const M3<T>& a, const M3<T>& h) { return prod<true, false, 3, false, true>(a, h); }
template <typename T> LT_HD M3<T> mul_hd(const M3<T>& h, const M3<T>& b) { return prod<false, true, 3, true, false>(h, b); }
// A * B^dagger
template <typename T> LT_HD M3<T> mul_nd(const M3<T>& a, const M3<T>& b) { return prod<false, true>(a, b); }
// A^dagger * B
template <typename T> LT_HD M3<T> mul_dn(const M3<T>& a, const M3<T>& b) { return prod<true, false>(a, b); }
// A^dagger * B^dagger
template <typename T> LT_HD M3<T> mul_dd(const M3<T>& a, const M3<T>& b) { return prod<true, true>(a, b); }

// Rows 0 and 1 only of A * B, A * B^dagger and A^dagger * B (row 2 of the result is left
// unset); used where the product is an SU(3) matrix whose third row is rebuilt afterwards.
template <typename T> LT_HD M3<T> mul_rows(const M3<T>& a, const M3<T>& b) { return prod<false, false, 2>(a, b); }
template <typename T> LT_HD M3<T> mul_nd_rows(const M3<T>& a, const M3<T>& b) { return prod<false, true, 2>(a, b); }
template <typename T> LT_HD M3<T> mul_dn_rows(const M3<T>& a, const M3<T>& b) { return prod<true, false, 2>(a, b); }

template <typename T> LT_HD M3<T> adj(const M3<T>& a)
{
    M3<T> r;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) r.e[i][j] = conj(a.e[j][i]);
    return r;
}

template <typename T> LT_HD void acc(M3<T>& a, const M3<T>& b)
{
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) a.e[i][j] = a.e[i][j] + b.e[i][j];
}

template <typename T> LT_HD M3<T> operator+(M3<T> a, const M3<T>& b) { acc(a, b); return a; }
template <typename T> LT_HD M3<T> operator-(M3<T> a, const M3<T>& b)
{
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) a.e[i][j] = a.e[i][j] - b.e[i][j];
    return a;
}
template <typename T> LT_HD M3<T> operator*(T s, M3<T> a)
{
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) a.e[i][j] = s * a.e[i][j];
    return a;
}
template <typename T> LT_HD M3<T> operator*(cx<T> s, M3<T> a)
{
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) a.e[i][j] = s * a.e[i][j];
    return a;
}

template <typename T> LT_HD cx<T> trace(const M3<T>& a) { return a.e[0][0] + a.e[1][1] + a.e[2][2]; }

// Re tr(A B) without forming the product
template <typename T> LT_HD T retr_mul(const M3<T>& a, const M3<T>& b)
{
    T s = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int k = 0; k < 3; ++k)
        {
            s += a.e[i][k].r * b.e[k][i].r;
            s -= a.e[i][k].i * b.e[k][i].i;
        }
    return s;
}

// Re tr(A B^dag) = sum_ij Re(A_ij conj(B_ij))
template <typename T> LT_HD T retr_nd(const M3<T>& a, const M3<T>& b)
{
    T s = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
        {
            s += a.e[i][j].r * b.e[i][j].r;
            s += a.e[i][j].i * b.e[i][j].i;
        }
    return s;
}

// tr(A B) without forming the product
template <typename T> LT_HD cx<T> tr_mul(const M3<T>& a, const M3<T>& b)
{
    T re = 0, im = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int k = 0; k < 3; ++k)
        {
            re += a.e[i][k].r * b.e[k][i].r;
            re -= a.e[i][k].i * b.e[k][i].i;
            im += a.e[i][k].r * b.e[k][i].i;
            im += a.e[i][k].i * b.e[k][i].r;
        }
    return mkc<T>(re, im);
}

template <typename To, typename From> LT_HD M3<To> cvt(const M3<From>& a)
{
    M3<To> r;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) r.e[i][j] = cvt<To>(a.e[i][j]);
    return r;
}

// ---------------------------------------------------------------- algebra fields
// A traceless anti-Hermitian matrix X kept as 8 reals:
//   X00 = i a0, X11 = i a1, X22 = -i (a0 + a1), X01 = a2 + i a3, X02 = a4 + i a5, X12 = a6 + i a7.
template <typename T> struct A8 { T a[8]; };

// Algebra(M) = (M - M^dag)/2 - tr(M - M^dag)/6 (math/su3.hpp:423-426), packed
template <typename T> LT_HD A8<T> algebra8(const M3<T>& m)
{
    A8<T> x;
    T d0 = m.e[0][0].i, d1 = m.e[1][1].i, d2 = m.e[2][2].i;
    T t = (d0 + d1 + d2) * (T)(1.0 / 3.0);
    x.a[0] = d0 - t;
    x.a[1] = d1 - t;
    x.a[2] = (T)0.5 * (m.e[0][1].r - m.e[1][0].r);
    x.a[3] = (T)0.5 * (m.e[0][1].i + m.e[1][0].i);
    x.a[4] = (T)0.5 * (m.e[0][2].r - m.e[2][0].r);
    x.a[5] = (T)0.5 * (m.e[0][2].i + m.e[2][0].i);
    x.a[6] = (T)0.5 * (m.e[1][2].r - m.e[2][1].r);
    x.a[7] = (T)0.5 * (m.e[1][2].i + m.e[2][1].i);
    return x;
}

template <typename T> LT_HD M3<T> unpack_ah(const A8<T>& x)
{
    M3<T> m;
    m.e[0][0] = mkc<T>(0, x.a[0]);
    m.e[1][1] = mkc<T>(0, x.a[1]);
    m.e[2][2] = mkc<T>(0, -(x.a[0] + x.a[1]));
    m.e[0][1] = mkc<T>(x.a[2], x.a[3]);
    m.e[0][2] = mkc<T>(x.a[4], x.a[5]);
    m.e[1][2] = mkc<T>(x.a[6], x.a[7]);
    m.e[1][0] = mkc<T>(-x.a[2], x.a[3]);
    m.e[2][0] = mkc<T>(-x.a[4], x.a[5]);
    m.e[2][1] = mkc<T>(-x.a[6], x.a[7]);
    return m;
}

// Hermitian traceless H kept as 8 reals: H00 = h0, H11 = h1, H22 = -(h0+h1), H01 = h2 + i h3, ...
// TracelessHermitian(M) = (M + M^dag)/2 - tr(M + M^dag)/6 (math/su3.hpp:445-448), packed
template <typename T> LT_HD A8<T> traceless_herm8(const M3<T>& m)
{
    A8<T> x;
    T d0 = m.e[0][0].r, d1 = m.e[1][1].r, d2 = m.e[2][2].r;
    T t = (d0 + d1 + d2) * (T)(1.0 / 3.0);
    x.a[0] = d0 - t;
    x.a[1] = d1 - t;
    x.a[2] = (T)0.5 * (m.e[0][1].r + m.e[1][0].r);
    x.a[3] = (T)0.5 * (m.e[0][1].i - m.e[1][0].i);
    x.a[4] = (T)0.5 * (m.e[0][2].r + m.e[2][0].r);
    x.a[5] = (T)0.5 * (m.e[0][2].i - m.e[2][0].i);
    x.a[6] = (T)0.5 * (m.e[1][2].r + m.e[2][1].r);
    x.a[7] = (T)0.5 * (m.e[1][2].i - m.e[2][1].i);
    return x;
}

template <typename T> LT_HD M3<T> unpack_h(const A8<T>& x)
{
    M3<T> m;
    m.e[0][0] = mkc<T>(x.a[0], 0);
    m.e[1][1] = mkc<T>(x.a[1], 0);
    m.e[2][2] = mkc<T>(-(x.a[0] + x.a[1]), 0);
    m.e[0][1] = mkc<T>(x.a[2], x.a[3]);
    m.e[0][2] = mkc<T>(x.a[4], x.a[5]);
    m.e[1][2] = mkc<T>(x.a[6], x.a[7]);
    m.e[1][0] = mkc<T>(x.a[2], -x.a[3]);
    m.e[2][0] = mkc<T>(x.a[4], -x.a[5]);
    m.e[2][1] = mkc<T>(x.a[6], -x.a[7]);
    return m;
}

// ---------------------------------------------------------------- reunitarisation
// RestoreLastRow (math/su3.hpp:362-367): row 2 = conj(row 0 x row 1)
// g1 a + g2 b as an FMA chain
template <typename T> LT_HD cx<T> lincomb2(cx<T> g1, cx<T> a, cx<T> g2, cx<T> b)
{
    T re = g1.r * a.r;
    re -= g1.i * a.i;
    re += g2.r * b.r;
    re -= g2.i * b.i;
    T im = g1.r * a.i;
    im += g1.i * a.r;
    im += g2.r * b.i;
    im += g2.i * b.r;
    return mkc<T>(re, im);
}

// conj(p q - r s) as an FMA chain
template <typename T> LT_HD cx<T> conj_cross(cx<T> p, cx<T> q, cx<T> r, cx<T> s)
{
    T re = p.r * q.r;
    re -= p.i * q.i;
    re -= r.r * s.r;
    re += r.i * s.i;
    T im = p.r * q.i;
    im += p.i * q.r;
    im -= r.r * s.i;
    im -= r.i * s.r;
    return mkc<T>(re, -im);
}

// a + conj(p q - r s) as an FMA chain
template <typename T> LT_HD cx<T> acc_conj_cross(cx<T> a, cx<T> p, cx<T> q, cx<T> r, cx<T> s)
{
    T re = a.r;
    re += p.r * q.r;
    re -= p.i * q.i;
    re -= r.r * s.r;
    re += r.i * s.i;
    T im = a.i;
    im -= p.r * q.i;
    im -= p.i * q.r;
    im += r.r * s.i;
    im += r.i * s.r;
    return mkc<T>(re, im);
}

// a += p for an SU(3) matrix p of which only rows 0 and 1 are set: its third row
// (RestoreLastRow) is formed inside the sum
template <typename T> LT_HD void acc_restored(M3<T>& a, const M3<T>& p)
{
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) a.e[i][j] = a.e[i][j] + p.e[i][j];
    a.e[2][0] = acc_conj_cross(a.e[2][0], p.e[0][1], p.e[1][2], p.e[0][2], p.e[1][1]);
    a.e[2][1] = acc_conj_cross(a.e[2][1], p.e[0][2], p.e[1][0], p.e[0][0], p.e[1][2]);
    a.e[2][2] = acc_conj_cross(a.e[2][2], p.e[0][0], p.e[1][1], p.e[0][1], p.e[1][0]);
}

template <typename T> LT_HD void restore_last_row(M3<T>& a)
{
    a.e[2][0] = conj_cross(a.e[0][1], a.e[1][2], a.e[0][2], a.e[1][1]);
    a.e[2][1] = conj_cross(a.e[0][2], a.e[1][0], a.e[0][0], a.e[1][2]);
    a.e[2][2] = conj_cross(a.e[0][0], a.e[1][1], a.e[0][1], a.e[1][0]);
}

template <typename T> LT_D T rsqrt_t(T x);
// FP64: CUDA's double-precision reciprocal square root (within 1 ulp), not a square root and a
// division; the normalised results agree with 1 / sqrt to rounding
template <> LT_D double rsqrt_t<double>(double x) { return rsqrt(x); }
// FP32: the hardware reciprocal square root (rsqrtf, 2 ulp) instead of an IEEE square root and
// an IEEE division; every use normalises a vector or an SU(2) matrix whose FP32 rounding is of
// the same order, and each update ends with a Gram-Schmidt projection
template <> LT_D float rsqrt_t<float>(float x) { return rsqrtf(x); }
// FP32 square root by the hardware approximation (PTX sqrt.approx.f32, relative error within
// 2^-23 per the PTX ISA), for the sampler's sqrt(1 - x^2) terms; sqrt_approx(0) = 0
LT_D float sqrt_approx(float x)
{
    float r;
    asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// GramSchmidt (math/su3.hpp:370-394); RESTORE = false skips the third row (two-row storage)
template <typename T, bool RESTORE = true> LT_D void gram_schmidt(M3<T>& a)
{
    T n0 = rsqrt_t<T>(norm2(a.e[0][0]) + norm2(a.e[0][1]) + norm2(a.e[0][2]));
#pragma unroll
    for (int n = 0; n < 3; ++n) a.e[0][n] = n0 * a.e[0][n];
    T pr = 0, pi = 0;   // psi = sum_n row1_n conj(row0_n)
#pragma unroll
    for (int n = 0; n < 3; ++n)
    {
        pr += a.e[1][n].r * a.e[0][n].r;
        pr += a.e[1][n].i * a.e[0][n].i;
        pi += a.e[1][n].i * a.e[0][n].r;
        pi -= a.e[1][n].r * a.e[0][n].i;
    }
#pragma unroll
    for (int n = 0; n < 3; ++n)
    {
        T r = a.e[1][n].r, i = a.e[1][n].i;
        r -= pr * a.e[0][n].r;
        r += pi * a.e[0][n].i;
        i -= pr * a.e[0][n].i;
        i -= pi * a.e[0][n].r;
        a.e[1][n] = mkc<T>(r, i);
    }
    T n1 = rsqrt_t<T>(norm2(a.e[1][0]) + norm2(a.e[1][1]) + norm2(a.e[1][2]));
#pragma unroll
    for (int n = 0; n < 3; ++n) a.e[1][n] = n1 * a.e[1][n];
    if (RESTORE) restore_last_row(a);
}

// ---------------------------------------------------------------- SU(2) subgroups
template <typename T> struct S2 { cx<T> e11, e12; };

template <typename T> LT_HD S2<T> s2_mul(const S2<T>& a, const S2<T>& b)
{
    S2<T> r;
    r.e11 = a.e11 * b.e11 - mulc(a.e12, b.e12);
    r.e12 = a.e11 * b.e12 + mulc(a.e12, b.e11);
    return r;
}
template <typename T> LT_HD S2<T> s2_adj(const S2<T>& a) { S2<T> r; r.e11 = conj(a.e11); r.e12 = -a.e12; return r; }
template <typename T> LT_HD T s2_det(const S2<T>& a) { return norm2(a.e11) + norm2(a.e12); }

// Subgroup g in {0: (0,1), 1: (0,2), 2: (1,2)} as (row a, row b)
LT_HD int sg_a(int g) { return g == 2 ? 1 : 0; }
LT_HD int sg_b(int g) { return g == 0 ? 1 : 2; }

// Extract0x (math/su2.hpp:151-174)
template <typename T> LT_HD S2<T> extract(const M3<T>& w, int g)
{
    const int a = sg_a(g), b = sg_b(g);
    S2<T> r;
    r.e11 = (T)0.5 * (w.e[a][a] + conj(w.e[b][b]));
    r.e12 = (T)0.5 * (w.e[a][b] - conj(w.e[b][a]));
    return r;
}

// Embed0x(m) * X (math/su2.hpp:118-146): mixes rows a and b of X
template <typename T> LT_HD void embed_lmul(const S2<T>& m, int g, M3<T>& x)
{
    const int a = sg_a(g), b = sg_b(g);
#pragma unroll
    for (int n = 0; n < 3; ++n)
    {
        const cx<T> xa = x.e[a][n], xb = x.e[b][n];
        // row a: e11 xa + e12 xb
        T ar = m.e11.r * xa.r, ai = m.e11.r * xa.i;
        ar -= m.e11.i * xa.i;
        ai += m.e11.i * xa.r;
        ar += m.e12.r * xb.r;
        ai += m.e12.r * xb.i;
        ar -= m.e12.i * xb.i;
        ai += m.e12.i * xb.r;
        // row b: conj(e11) xb - conj(e12) xa
        T br = m.e11.r * xb.r, bi = m.e11.r * xb.i;
        br += m.e11.i * xb.i;
        bi -= m.e11.i * xb.r;
        br -= m.e12.r * xa.r;
        bi -= m.e12.r * xa.i;
        br -= m.e12.i * xa.i;
        bi += m.e12.i * xa.r;
        x.e[a][n] = mkc<T>(ar, ai);
        x.e[b][n] = mkc<T>(br, bi);
    }
}

// ---------------------------------------------------------------- Cayley-Hamilton exp
// xi_0(w) = sin(w)/w and xi_1(w) = cos(w)/w^2 - sin(w)/w^3 with the double-precision Taylor
// switches of ExpTaylorBounds<double> (math/su3_exp.hpp:38-82)
LT_D double xi0(double w)
{
    if (fabs(w) <= 0.05)
    {
        double w2 = w * w;
        return 1.0 - 1.0 / 6.0 * w2 * (1.0 - 1.0 / 20.0 * w2 * (1.0 - 1.0 / 42.0 * w2));
    }
    return sin(w) / w;
}

LT_D double xi1(double w)
{
    if (fabs(w) <= 0.115)
    {
        double w2 = w * w;
        return -1.0 / 3.0 + 1.0 / 30.0 * w2 * (1.0 - 1.0 / 28.0 * w2 * (1.0 - 1.0 / 54.0 * w2));
    }
    double s, c;
    sincos(w, &s, &c);
    return c / (w * w) - s / (w * w * w);
}

// Scalar part of ExpConstants (math/su3_exp.hpp:204-283) for a traceless Hermitian Q.
struct ExpScalars
{
    double u, w, u2, w2, c0max, denom;
    int signflip;
    cx<double> emiu, e2iu, cosw, ixi0, h0, h1, h2;
};

template <typename T> LT_D ExpScalars exp_scalars(const M3<T>& Q, const M3<T>& Q2)
{
    ExpScalars e;
    // c0 = det Q = tr(Q^3)/3 and c1 = tr(Q^2)/2, accumulated in double
    double c0s = 0.0, c1 = 0.0;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int k = 0; k < 3; ++k)
        {
            c0s += (double)Q.e[i][k].r * (double)Q2.e[k][i].r - (double)Q.e[i][k].i * (double)Q2.e[k][i].i;
        }
    c0s *= 1.0 / 3.0;
    c1 = 0.5 * ((double)Q2.e[0][0].r + (double)Q2.e[1][1].r + (double)Q2.e[2][2].r);
    double c0 = fabs(c0s);
    double c13 = c1 / 3.0;
    e.c0max = 2.0 * c13 * sqrt(c13);
    e.signflip = c0s < 0.0;
    double theta = acos(fmin(c0 / e.c0max, 1.0));
    double st3, ct3;
    sincos(theta / 3.0, &st3, &ct3);
    e.u = sqrt(c13) * ct3;
    e.w = sqrt(c1) * st3;
    e.u2 = e.u * e.u;
    e.w2 = e.w * e.w;
    double su, cu;
    sincos(e.u, &su, &cu);
    e.emiu = mkc<double>(cu, -su);
    // exp(2iu) = conj(exp(-iu)^2)
    e.e2iu = conj(e.emiu * e.emiu);
    e.cosw = mkc<double>(cos(e.w), 0.0);
    e.ixi0 = mkc<double>(0.0, xi0(e.w));
    if (e.c0max < DBL_MIN)
    {
        e.denom = 1.0;
        e.h0 = mkc<double>(1.0, 0.0);
        e.h1 = mkc<double>(0.0, 0.0);
        e.h2 = mkc<double>(0.0, 0.0);
        return e;
    }
    const double u = e.u, u2 = e.u2, w2 = e.w2;
    e.denom = 1.0 / (9.0 * u2 - w2);
    cx<double> h0 = (u2 - w2) * e.e2iu + e.emiu * ((8.0 * u2) * e.cosw + (2.0 * u * (3.0 * u2 + w2)) * e.ixi0);
    cx<double> h1 = (2.0 * u) * e.e2iu - e.emiu * ((2.0 * u) * e.cosw - (3.0 * u2 - w2) * e.ixi0);
    cx<double> h2 = e.e2iu - e.emiu * (e.cosw + (3.0 * u) * e.ixi0);
    if (e.signflip)
    {
        h0 = conj(h0);
        h1 = -conj(h1);
        h2 = conj(h2);
    }
    e.h0 = h0;
    e.h1 = h1;
    e.h2 = h2;
    return e;
}

// exp(iQ) = denom (h0 + h1 Q + h2 Q^2) (math/su3_exp.hpp:419-432)
template <typename T> LT_D M3<T> exp_from(const ExpScalars& e, const M3<T>& Q, const M3<T>& Q2)
{
    cx<T> f0 = cvt<T>(e.denom * e.h0), f1 = cvt<T>(e.denom * e.h1), f2 = cvt<T>(e.denom * e.h2);
    M3<T> r;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) r.e[i][j] = lincomb2(f1, Q.e[i][j], f2, Q2.e[i][j]);
    r.e[0][0] = r.e[0][0] + f0;
    r.e[1][1] = r.e[1][1] + f0;
    r.e[2][2] = r.e[2][2] + f0;
    return r;
}

// exp(iQ) = f0 + f1 Q + f2 Q^2 from the power series of exp reduced with Cayley-Hamilton,
// Q^3 = c1 Q + c0 (c0 = det Q = tr Q^3 / 3, c1 = tr Q^2 / 2): with Q^n = a_n + b_n Q + c_n Q^2,
// (a, b, c)_{n+1} = (c_n c0, a_n + c_n c1, b_n).  Valid when the spectral radius bound
// sqrt(2 c1) is at most 1; N terms then leave a truncation error below 1/(N+1)!.
// Same exponential as the closed form of SU3::exp (math/su3_exp.hpp:419-432) to rounding,
// without its acos/sincos chain.
template <int N, typename S> LT_D void exp_series(S c0, S c1, cx<S>& f0, cx<S>& f1, cx<S>& f2)
{
    S a = 1, b = 0, c = 0;   // scaled: (a_n, b_n, c_n) / n!
    S f0r = 0, f0i = 0, f1r = 0, f1i = 0, f2r = 0, f2i = 0;
#pragma unroll
    for (int n = 0; n <= N; ++n)
    {
        // i^n = 1, i, -1, -i
        switch (n & 3)
        {
            case 0: f0r += a; f1r += b; f2r += c; break;
            case 1: f0i += a; f1i += b; f2i += c; break;
            case 2: f0r -= a; f1r -= b; f2r -= c; break;
            default: f0i -= a; f1i -= b; f2i -= c; break;
        }
        const S inv = (S)(1.0 / (double)(n + 1));
        const S na = c * c0 * inv, nb = (a + c * c1) * inv, nc = b * inv;
        a = na; b = nb; c = nc;
    }
    f0 = mkc(f0r, f0i);
    f1 = mkc(f1r, f1i);
    f2 = mkc(f2r, f2i);
}

// The same series with its derivatives: f_j = sum_n i^n (a, b, c)_n / n! and d0_j = df_j/dc0,
// d1_j = df_j/dc1 by differentiating the recursion term by term.  With dc0 = tr(Q^2 dQ) and
// dc1 = tr(Q dQ), B_1 = sum_j d1_j Q^j and B_2 = sum_j d0_j Q^j are the matrices of
// ExpDerivativeConstants (math/su3_exp.hpp:286-416; Morningstar-Peardon, hep-lat/0311018).
template <int N, typename S>
LT_D void exp_series_deriv(S c0, S c1, cx<S> f[3], cx<S> d0[3], cx<S> d1[3])
{
    S x[3] = { 1, 0, 0 }, y[3] = { 0, 0, 0 }, z[3] = { 0, 0, 0 };   // (a, b, c)_n / n! and d/dc0, d/dc1
    S fr[3] = { 0, 0, 0 }, fi[3] = { 0, 0, 0 }, yr[3] = { 0, 0, 0 }, yi[3] = { 0, 0, 0 };
    S zr[3] = { 0, 0, 0 }, zi[3] = { 0, 0, 0 };
#pragma unroll
    for (int n = 0; n <= N; ++n)
    {
        const S sg = (n & 2) ? (S)-1 : (S)1;   // i^n = sg (n even) or sg i (n odd)
#pragma unroll
        for (int j = 0; j < 3; ++j)
        {
            if (n & 1)
            {
                fi[j] += sg * x[j];
                yi[j] += sg * y[j];
                zi[j] += sg * z[j];
            }
            else
            {
                fr[j] += sg * x[j];
                yr[j] += sg * y[j];
                zr[j] += sg * z[j];
            }
        }
        const S inv = (S)(1.0 / (double)(n + 1));
        const S na = x[2] * c0 * inv, nb = (x[0] + x[2] * c1) * inv, nc = x[1] * inv;
        const S ya = (y[2] * c0 + x[2]) * inv, yb = (y[0] + y[2] * c1) * inv, yc = y[1] * inv;
        const S za = z[2] * c0 * inv, zb = (z[0] + z[2] * c1 + x[2]) * inv, zc = z[1] * inv;
        x[0] = na; x[1] = nb; x[2] = nc;
        y[0] = ya; y[1] = yb; y[2] = yc;
        z[0] = za; z[1] = zb; z[2] = zc;
    }
#pragma unroll
    for (int j = 0; j < 3; ++j)
    {
        f[j] = mkc(fr[j], fi[j]);
        d0[j] = mkc(yr[j], yi[j]);
        d1[j] = mkc(zr[j], zi[j]);
    }
}

// Q^2 of a Hermitian Q (upper triangle computed, lower mirrored)
template <typename T> LT_D M3<T> herm_sq(const M3<T>& q)
{
    M3<T> r;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = i; j < 3; ++j)
        {
            T re = 0, im = 0;
#pragma unroll
            for (int k = 0; k < 3; ++k)
            {
                re += q.e[i][k].r * q.e[k][j].r;
                re -= q.e[i][k].i * q.e[k][j].i;
                im += q.e[i][k].r * q.e[k][j].i;
                im += q.e[i][k].i * q.e[k][j].r;
            }
            r.e[i][j] = mkc<T>(re, i == j ? (T)0 : im);
            if (j != i) r.e[j][i] = mkc<T>(re, -im);
        }
    return r;
}

// exp(c X) for X traceless anti-Hermitian: SU3::exp(-i c X) (gradient_flow.hpp:276,
// hmc_gauge.hpp:516, stout_smearing.hpp:52).  Small arguments (every flow and HMC step)
// take the Cayley-Hamilton-reduced series in the link arithmetic type (up to 19 terms in
// FP64: 1/20! = 4e-19; up to 12 terms in FP32: 1/13! = 2e-10); larger ones the closed form
// of ExpConstants with its scalar chain in FP64.
template <typename T> LT_D M3<T> exp_ah(const M3<T>& X, T c)
{
    // Q = -i c X is Hermitian traceless
    M3<T> Q;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) Q.e[i][j] = mkc<T>(c * X.e[i][j].i, -c * X.e[i][j].r);
    M3<T> Q2 = herm_sq(Q);
    const T c1 = (T)0.5 * (Q2.e[0][0].r + Q2.e[1][1].r + Q2.e[2][2].r);
    if (c1 <= (T)0.5)
    {
        T c0 = retr_mul(Q, Q2) * (T)(1.0 / 3.0);
        cx<T> g0, g1, g2;
        // the truncation error after N terms is below r^(N+1)/(N+1)! e^r for spectral radius
        // r <= sqrt(2 c1): at r <= 1/16 (the flow's steps of eps = 0.01) 10 terms leave 3e-19 in
        // FP64 and 5 terms 9e-9 in FP32; at r <= 1/4 (HMC steps) 13 terms leave 3e-18 in FP64
        // and 7 terms 1.6e-8 in FP32
        if (c1 <= (T)(1.0 / 512.0))
        {
            if (sizeof(T) == 8) exp_series<9>(c0, c1, g0, g1, g2);
            else exp_series<4>(c0, c1, g0, g1, g2);
        }
        else if (c1 <= (T)(1.0 / 32.0))
        {
            if (sizeof(T) == 8) exp_series<12>(c0, c1, g0, g1, g2);
            else exp_series<6>(c0, c1, g0, g1, g2);
        }
        else
        {
            if (sizeof(T) == 8) exp_series<18>(c0, c1, g0, g1, g2);
            else exp_series<11>(c0, c1, g0, g1, g2);
        }
        M3<T> r;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) r.e[i][j] = lincomb2(g1, Q.e[i][j], g2, Q2.e[i][j]);
        r.e[0][0] = r.e[0][0] + g0;
        r.e[1][1] = r.e[1][1] + g0;
        r.e[2][2] = r.e[2][2] + g0;
        return r;
    }
    ExpScalars e = exp_scalars(Q, Q2);
    return exp_from(e, Q, Q2);
}

// f1, f2 and B_1, B_2 of ExpDerivativeConstants (math/su3_exp.hpp:121-201, :389-415)
struct ExpDerivScalars
{
    cx<double> f1, f2, b10, b11, b12, b20, b21, b22;
};

LT_D ExpDerivScalars exp_deriv_scalars(const ExpScalars& e)
{
    ExpDerivScalars d;
    const double u = e.u, u2 = e.u2, w2 = e.w2;
    const cx<double> x0 = mkc<double>(xi0(e.w), 0.0), x1 = mkc<double>(xi1(e.w), 0.0);
    const cx<double> I1 = mkc<double>(0.0, 1.0);
    const cx<double> one = mkc<double>(1.0, 0.0);
    cx<double> f0 = e.denom * e.h0, f1 = e.denom * e.h1, f2 = e.denom * e.h2;
    const cx<double> emiu = e.emiu, e2iu = e.e2iu, cosw = e.cosw, ix0 = e.ixi0;
    cx<double> r10 = 2.0 * (mkc<double>(u, u2 - w2) * e2iu)
                   + 2.0 * (emiu * ((4.0 * u) * (mkc<double>(2.0, -u) * cosw)
                                    + ix0 * mkc<double>(9.0 * u2 + w2, -u * (3.0 * u2 + w2))));
    cx<double> r11 = 2.0 * (mkc<double>(1.0, 2.0 * u) * e2iu)
                   + emiu * ((-2.0) * (mkc<double>(1.0, -u) * cosw) + ix0 * mkc<double>(6.0 * u, w2 - 3.0 * u2));
    cx<double> r12 = 2.0 * (I1 * e2iu) + I1 * (emiu * (cosw - 3.0 * (mkc<double>(1.0, -u) * x0)));
    cx<double> r20 = (-2.0) * e2iu
                   + ((2.0 * u) * I1) * (emiu * (cosw + mkc<double>(1.0, 4.0 * u) * x0 + (3.0 * u2) * x1));
    cx<double> r21 = -(I1 * (emiu * (cosw + mkc<double>(1.0, 2.0 * u) * x0 - (3.0 * u2) * x1)));
    cx<double> r22 = emiu * (x0 - ((3.0 * u) * I1) * x1);
    (void)one;
    d.f1 = f1;
    d.f2 = f2;
    if (e.c0max < DBL_MIN)
    {
        d.b10 = d.b11 = d.b12 = d.b20 = d.b21 = d.b22 = mkc<double>(0.0, 0.0);
        return d;
    }
    double bd = 9.0 * u2 - w2;
    bd *= 2.0 * bd;
    bd = 1.0 / bd;
    const double k1 = 3.0 * u2 - w2, k2 = 2.0 * (15.0 * u2 + w2);
    if (e.signflip)
    {
        d.b10 = bd * conj((2.0 * u) * r10 + k1 * r20 - k2 * conj(f0));
        d.b11 = (-bd) * conj((2.0 * u) * r11 + k1 * r21 + k2 * conj(f1));
        d.b12 = bd * conj((2.0 * u) * r12 + k1 * r22 - k2 * conj(f2));
        d.b20 = (-bd) * conj(r10 - (3.0 * u) * r20 - (24.0 * u) * conj(f0));
        d.b21 = bd * conj(r11 - (3.0 * u) * r21 + (24.0 * u) * conj(f1));
        d.b22 = (-bd) * conj(r12 - (3.0 * u) * r22 - (24.0 * u) * conj(f2));
    }
    else
    {
        d.b10 = bd * ((2.0 * u) * r10 + k1 * r20 - k2 * f0);
        d.b11 = bd * ((2.0 * u) * r11 + k1 * r21 - k2 * f1);
        d.b12 = bd * ((2.0 * u) * r12 + k1 * r22 - k2 * f2);
        d.b20 = bd * (r10 - (3.0 * u) * r20 - (24.0 * u) * f0);
        d.b21 = bd * (r11 - (3.0 * u) * r21 - (24.0 * u) * f1);
        d.b22 = bd * (r12 - (3.0 * u) * r22 - (24.0 * u) * f2);
    }
    return d;
}

// ---------------------------------------------------------------- Philox4x32-10
// Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3" (SC'11).
struct U4 { uint32_t x, y, z, w; };

LT_HD U4 philox4x32(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1)
{
#pragma unroll
    for (int r = 0; r < 10; ++r)
    {
#ifdef __CUDA_ARCH__
        uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
        uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
#else
        uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
#endif
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        c1 = lo1;
        c3 = lo0;
        c0 = n0;
        c2 = n2;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    U4 o;
    o.x = c0; o.y = c1; o.z = c2; o.w = c3;
    return o;
}

// Stream tags (word 3 of the counter, bits 24..31)
enum : uint32_t { TAG_HEATBATH = 1, TAG_MOMENTA = 2, TAG_ACCEPT = 3, TAG_HAAR = 4 };

LT_HD double u01_from(uint32_t hi, uint32_t lo)
{
    return (double)((((uint64_t)hi << 32) | lo) >> 11) * 0x1.0p-53;
}

LT_HD float f01_from(uint32_t w) { return (float)(w >> 8) * 0x1.0p-24f; }

} // namespace lt
