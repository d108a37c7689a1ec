// Device data layout of the lattice fields and the neighbour arithmetic.
//
// Geometry: runtime extents n = {Nt, Nx, Ny, Nz} (all even, as the reference's checkerboard
// iterator requires, LettuceGauge/iterators/iterators.hpp:68).  The reference's lexicographic
// site index i = ((t*Nx + x)*Ny + y)*Nz + z (lattice.hpp:366-382) is kept as the "full"
// index; a site's parity is (t+x+y+z)&1 and its checkerboard index is i>>1 (unique within a
// parity because Nz is even).
//
// Link fields are even/odd structure-of-arrays: one plane of vh = V/2 complex numbers per
// (direction mu, parity, matrix element), plane index (mu*2 + parity)*(3*NR) + element.
// NR = 3 stores all 18 reals; NR = 2 stores the first two rows (12 reals) and rebuilds the
// third with RestoreLastRow (math/su3.hpp:362-367).  A warp reading consecutive
// checkerboard sites touches consecutive 16-byte (FP64) or 8-byte (FP32) words of every
// plane, so each matrix element is one fully coalesced load.
//
// Algebra fields (flow Z, HMC momenta, stout forces) keep 8 reals per link, plane index
// (mu*2 + parity)*8 + k, packed as in lt_math.cuh (A8).
#pragma once
#include "lt_math.cuh"

namespace lt {

// Reduction grid: 148 SMs x 8 blocks, fixed so that every reduction sums in the same order.
constexpr int kRedBlocks = 1184;
constexpr int kRedThreads = 256;

// Bits of a lattice handle's device status word (LT_STATUS_* of the C ABI)
constexpr unsigned kStatusNonFinite = 1u;   // a link holds NaN or Inf
constexpr unsigned kStatusUnitarity = 2u;   // max |U U^dag - 1| above the storage's tolerance
constexpr unsigned kStatusHbCap = 4u;       // a heatbath subgroup update hit its iteration cap
constexpr unsigned kStatusBarrierTimeout = 8u;   // a grid barrier of a persistent kernel gave up waiting

struct Geom
{
    int n[4];            // Nt, Nx, Ny, Nz
    int stride[4];       // full-index stride of each direction
    int V;               // sites
    int vh;              // sites per parity
    unsigned div_m[4];   // x / n[d] = umulhi(x, div_m[d]) >> div_s[d] for 0 <= x < 2^31
    int div_s[4];
};

inline Geom make_geom(const int ext[4])
{
    Geom g;
    for (int d = 0; d < 4; ++d)
    {
        g.n[d] = ext[d];
        // division by a run-time constant (Granlund-Montgomery): extents are >= 2, so with
        // l = ceil(log2 n) >= 1, m = ceil(2^(31 + l) / n) < 2^32 and the error of
        // x m / 2^(31 + l) stays below 1/n for x < 2^31
        const unsigned n = (unsigned)(ext[d] > 2 ? ext[d] : 2);
        int l = 1;
        while ((1ull << l) < n) ++l;
        g.div_m[d] = (unsigned)(((1ull << (31 + l)) + n - 1) / n);
        g.div_s[d] = l - 1;
    }
    g.stride[3] = 1;
    g.stride[2] = ext[3];
    g.stride[1] = ext[2] * ext[3];
    g.stride[0] = ext[1] * ext[2] * ext[3];
    g.V = ext[0] * ext[1] * ext[2] * ext[3];
    g.vh = g.V / 2;
    return g;
}

// x / n[d] for 0 <= x < 2^31 without a hardware division
LT_D int div_by(const Geom& g, int x, int d) { return (int)(__umulhi((unsigned)x, g.div_m[d]) >> g.div_s[d]); }

// Coordinates and full index of checkerboard site s of parity par
LT_D int site_coords(const Geom& g, int par, int s, int c[4])
{
    int i0 = 2 * s;
    int r = div_by(g, i0, 3);
    int z0 = i0 - r * g.n[3];
    int r2 = div_by(g, r, 2);
    c[2] = r - r2 * g.n[2];
    int r3 = div_by(g, r2, 1);
    c[1] = r2 - r3 * g.n[1];
    c[0] = r3;
    c[3] = z0 + ((c[0] + c[1] + c[2] + par) & 1);
    return i0 - z0 + c[3];
}

// a[k] for a run-time k without indexing the array (keeps small arrays in registers)
LT_D int pick4(const int a[4], int k) { return k == 0 ? a[0] : k == 1 ? a[1] : k == 2 ? a[2] : a[3]; }

// Full-index offset of a +1 / -1 step along a run-time direction d from a site with
// coordinates c
LT_D int step_up_rt(const Geom& g, int d, const int c[4])
{
    const int n = pick4(g.n, d), st = pick4(g.stride, d);
    return pick4(c, d) + 1 < n ? st : -(n - 1) * st;
}
LT_D int step_dn_rt(const Geom& g, int d, const int c[4])
{
    const int n = pick4(g.n, d), st = pick4(g.stride, d);
    return pick4(c, d) > 0 ? -st : (n - 1) * st;
}

// Full-index offset of a +1 / -1 step along d from a site with coordinate cd along d
LT_D int step_up(const Geom& g, int d, int cd) { return cd + 1 < g.n[d] ? g.stride[d] : -(g.n[d] - 1) * g.stride[d]; }
LT_D int step_dn(const Geom& g, int d, int cd) { return cd > 0 ? -g.stride[d] : (g.n[d] - 1) * g.stride[d]; }

template <typename T, int NR> struct Gauge
{
    cx<T>* __restrict__ p;
    int vh;

    LT_D size_t plane(int mu, int par, int c) const { return (size_t)((mu * 2 + par) * (3 * NR) + c) * (size_t)vh; }

    LT_D M3<T> ld(int mu, int par, int s) const
    {
        M3<T> m;
        const cx<T>* q = p + plane(mu, par, 0) + s;
#pragma unroll
        for (int r = 0; r < NR; ++r)
#pragma unroll
            for (int j = 0; j < 3; ++j) m.e[r][j] = q[(size_t)(3 * r + j) * vh];
        if (NR == 2) restore_last_row(m);
        return m;
    }

    // Rows 0 and 1 only (row 2 is not rebuilt for two-row storage)
    LT_D M3<T> ld_rows(int mu, int par, int s) const
    {
        if (NR == 3) return ld(mu, par, s);
        M3<T> m;
        const cx<T>* q = p + plane(mu, par, 0) + s;
#pragma unroll
        for (int r = 0; r < 2; ++r)
#pragma unroll
            for (int j = 0; j < 3; ++j) m.e[r][j] = q[(size_t)(3 * r + j) * vh];
        return m;
    }

    LT_D void st(int mu, int par, int s, const M3<T>& m) const
    {
        cx<T>* q = p + plane(mu, par, 0) + s;
#pragma unroll
        for (int r = 0; r < NR; ++r)
#pragma unroll
            for (int j = 0; j < 3; ++j) q[(size_t)(3 * r + j) * vh] = m.e[r][j];
    }
};

#ifndef LT_F32C_SCALAR
// Two-row FP32 storage: the 12 floats of a link as three float4 chunks, chunk c of plane
// (mu, par) at ((mu * 2 + par) * 3 + c) * vh, holding two consecutive complex entries of rows
// 0-1 (e00 e01 | e02 e10 | e11 e12).  A link is three 16-byte loads; a warp reads 512
// contiguous bytes per chunk.
template <> struct Gauge<float, 2>
{
    cx<float>* __restrict__ p;
    int vh;

    LT_D const float4* chunk(int mu, int par, int c) const
    {
        return reinterpret_cast<const float4*>(p) + (size_t)((mu * 2 + par) * 3 + c) * (size_t)vh;
    }

    // rows 0-1 of a link from its three chunks
    static LT_D M3<float> rows_of(const float4& a, const float4& b, const float4& c)
    {
        M3<float> m;
        m.e[0][0] = mkc<float>(a.x, a.y);
        m.e[0][1] = mkc<float>(a.z, a.w);
        m.e[0][2] = mkc<float>(b.x, b.y);
        m.e[1][0] = mkc<float>(b.z, b.w);
        m.e[1][1] = mkc<float>(c.x, c.y);
        m.e[1][2] = mkc<float>(c.z, c.w);
        return m;
    }

    LT_D M3<float> ld_rows(int mu, int par, int s) const
    {
        const float4* q = chunk(mu, par, 0) + s;
        return rows_of(q[0], q[vh], q[2 * (size_t)vh]);
    }

    LT_D M3<float> ld(int mu, int par, int s) const
    {
        M3<float> m = ld_rows(mu, par, s);
        restore_last_row(m);
        return m;
    }

    LT_D void st(int mu, int par, int s, const M3<float>& m) const
    {
        float4* q = const_cast<float4*>(chunk(mu, par, 0)) + s;
        q[0] = make_float4(m.e[0][0].r, m.e[0][0].i, m.e[0][1].r, m.e[0][1].i);
        q[vh] = make_float4(m.e[0][2].r, m.e[0][2].i, m.e[1][0].r, m.e[1][0].i);
        q[2 * (size_t)vh] = make_float4(m.e[1][1].r, m.e[1][1].i, m.e[1][2].r, m.e[1][2].i);
    }
};
#endif

template <typename T> struct Alg
{
    T* __restrict__ p;
    int vh;

    LT_D size_t plane(int mu, int par, int k) const { return (size_t)((mu * 2 + par) * 8 + k) * (size_t)vh; }

    LT_D A8<T> ld(int mu, int par, int s) const
    {
        A8<T> x;
        const T* q = p + plane(mu, par, 0) + s;
#pragma unroll
        for (int k = 0; k < 8; ++k) x.a[k] = q[(size_t)k * vh];
        return x;
    }

    LT_D void st(int mu, int par, int s, const A8<T>& x) const
    {
        T* q = p + plane(mu, par, 0) + s;
#pragma unroll
        for (int k = 0; k < 8; ++k) q[(size_t)k * vh] = x.a[k];
    }
};

// Full 3x3 complex per link (used for the local term of the stout-force recursion)
template <typename T> struct Full
{
    cx<T>* __restrict__ p;
    int vh;

    LT_D size_t plane(int mu, int par, int c) const { return (size_t)((mu * 2 + par) * 9 + c) * (size_t)vh; }

    LT_D M3<T> ld(int mu, int par, int s) const
    {
        M3<T> m;
        const cx<T>* q = p + plane(mu, par, 0) + s;
#pragma unroll
        for (int c = 0; c < 9; ++c) m.e[c / 3][c % 3] = q[(size_t)c * vh];
        return m;
    }

    LT_D void st(int mu, int par, int s, const M3<T>& m) const
    {
        cx<T>* q = p + plane(mu, par, 0) + s;
#pragma unroll
        for (int c = 0; c < 9; ++c) q[(size_t)c * vh] = m.e[c / 3][c % 3];
    }
};

// Six clover planes per site of an anti-Hermitian R_{mu nu} = C_{mu nu} - C_{mu nu}^dag
// (9 reals: 3 imaginary diagonal entries and the 3 complex upper entries), plane index
// (plane*2 + parity)*9 + k with plane = 0..5 for (01, 02, 03, 12, 13, 23).
template <typename T> struct Clov
{
    T* __restrict__ p;
    int vh;

    LT_D size_t plane(int pl, int par, int k) const { return (size_t)((pl * 2 + par) * 9 + k) * (size_t)vh; }

    LT_D void st(int pl, int par, int s, const M3<T>& r) const
    {
        T* q = p + plane(pl, par, 0) + s;
        q[0] = r.e[0][0].i;
        q[(size_t)1 * vh] = r.e[1][1].i;
        q[(size_t)2 * vh] = r.e[2][2].i;
        q[(size_t)3 * vh] = r.e[0][1].r;
        q[(size_t)4 * vh] = r.e[0][1].i;
        q[(size_t)5 * vh] = r.e[0][2].r;
        q[(size_t)6 * vh] = r.e[0][2].i;
        q[(size_t)7 * vh] = r.e[1][2].r;
        q[(size_t)8 * vh] = r.e[1][2].i;
    }

    // R_{rho sigma} for any ordered pair (R_{sigma rho} = -R_{rho sigma})
    LT_D M3<T> ld(int rho, int sigma, int par, int s) const
    {
        int a = rho < sigma ? rho : sigma, b = rho < sigma ? sigma : rho;
        int pl = a == 0 ? b - 1 : (a == 1 ? b + 1 : 5);
        T sg = rho < sigma ? (T)1 : (T)-1;
        const T* q = p + plane(pl, par, 0) + s;
        T v[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) v[k] = sg * q[(size_t)k * vh];
        M3<T> m;
        m.e[0][0] = mkc<T>(0, v[0]);
        m.e[1][1] = mkc<T>(0, v[1]);
        m.e[2][2] = mkc<T>(0, v[2]);
        m.e[0][1] = mkc<T>(v[3], v[4]);
        m.e[0][2] = mkc<T>(v[5], v[6]);
        m.e[1][2] = mkc<T>(v[7], v[8]);
        m.e[1][0] = mkc<T>(-v[3], v[4]);
        m.e[2][0] = mkc<T>(-v[5], v[6]);
        m.e[2][1] = mkc<T>(-v[7], v[8]);
        return m;
    }

    // -i R_{rho sigma}: the Hermitian matrix (real diagonal) whose i-multiple is the plane
    LT_D M3<T> ld_h(int rho, int sigma, int par, int s) const
    {
        int a = rho < sigma ? rho : sigma, b = rho < sigma ? sigma : rho;
        int pl = a == 0 ? b - 1 : (a == 1 ? b + 1 : 5);
        T sg = rho < sigma ? (T)1 : (T)-1;
        const T* q = p + plane(pl, par, 0) + s;
        T v[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) v[k] = sg * q[(size_t)k * vh];
        M3<T> m;
        m.e[0][0] = mkc<T>(v[0], 0);
        m.e[1][1] = mkc<T>(v[1], 0);
        m.e[2][2] = mkc<T>(v[2], 0);
        m.e[0][1] = mkc<T>(v[4], -v[3]);
        m.e[0][2] = mkc<T>(v[6], -v[5]);
        m.e[1][2] = mkc<T>(v[8], -v[7]);
        m.e[1][0] = mkc<T>(v[4], v[3]);
        m.e[2][0] = mkc<T>(v[6], v[5]);
        m.e[2][1] = mkc<T>(v[8], v[7]);
        return m;
    }
};

} // namespace lt
