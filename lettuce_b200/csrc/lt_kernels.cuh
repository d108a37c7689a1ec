// CUDA kernels of the pure-gauge SU(3) hot path (sm_100a, CUDA cores; 3x3 complex products
// are too small for a dense tensor-core contraction).  One thread owns one link (or one
// site for site-local observables); neighbour links are gathered from the even/odd SoA
// planes described in lt_field.cuh.
#pragma once
#include "lt_field.cuh"
#include <type_traits>

namespace lt {

constexpr int kThreads = 128;

// Minimum resident blocks per SM requested from ptxas for the hot kernels (caps registers
// per thread); tuned per arithmetic type on B200, overridable at build time.
#ifndef LT_MINB_SWEEP_F32
#define LT_MINB_SWEEP_F32 5
#endif
#ifndef LT_MINB_OR_F32C
#define LT_MINB_OR_F32C 7
#endif
#ifndef LT_MINB_HB_F32C
#define LT_MINB_HB_F32C 6
#endif
#ifndef LT_MINB_SWEEP_F64
#define LT_MINB_SWEEP_F64 3
#endif
#ifndef LT_MINB_LINK_F32
#define LT_MINB_LINK_F32 1
#endif
#ifndef LT_MINB_LINK_F64
#define LT_MINB_LINK_F64 1
#endif
#ifndef LT_MINB_LINK_F32C
#define LT_MINB_LINK_F32C 4
#endif
template <typename T> struct MinBlocks;
template <> struct MinBlocks<float> { static constexpr int sweep = LT_MINB_SWEEP_F32, link = LT_MINB_LINK_F32; };
template <> struct MinBlocks<double> { static constexpr int sweep = LT_MINB_SWEEP_F64, link = LT_MINB_LINK_F64; };
// the sweeps on two-row FP32 storage fit tighter register budgets (no spills at 7 and 6
// blocks of 128 per SM; measured fastest on B200)
template <typename T, int NR> struct OrMinBlocks
{
    static constexpr int value = (sizeof(T) == 4 && NR == 2) ? LT_MINB_OR_F32C : MinBlocks<T>::sweep;
};
template <typename T, int NR> struct HbMinBlocks
{
    static constexpr int value = (sizeof(T) == 4 && NR == 2) ? LT_MINB_HB_F32C : MinBlocks<T>::sweep;
};
// Checkerboard4 sub-sweeps (Wilson action) carry the sublattice enumeration on top
template <typename T, int NR> struct Cb4MinBlocks
{
    static constexpr int value = (sizeof(T) == 4 && NR == 2) ? 5 : MinBlocks<T>::sweep;
};
// Checkerboard4 sub-sweeps with rectangles: 4 blocks of 128 per SM on two-row FP32 storage
// (128 registers, 28 bytes spilled; 7 % faster than 3 blocks at 157 registers), no cap for
// the others (FP64 spills above 1 KB per thread at 4 blocks)
#ifndef LT_MINB_RECT_F32C
#define LT_MINB_RECT_F32C 4
#endif
template <typename T, int NR> struct RectMinBlocks
{
    static constexpr int value = (sizeof(T) == 4 && NR == 2) ? LT_MINB_RECT_F32C : 1;
};
// link-parallel kernels: two-row FP32 storage has its own setting
template <typename T, int NR> struct LinkMinBlocks
{
    static constexpr int value = (sizeof(T) == 4 && NR == 2) ? LT_MINB_LINK_F32C : MinBlocks<T>::link;
};
constexpr double kPi = 3.14159265358979323846;
constexpr float kTwoPiF = 6.28318530717958648f;

// Programmatic dependent launch (sm_90 and later): a kernel launched with the programmatic
// stream-serialisation attribute may be scheduled while its predecessor on the stream still
// drains, once every block of the predecessor has passed pdl_release(); it must pass
// pdl_wait(), which returns when the predecessor has completed and its writes are visible,
// before reading the predecessor's output.  Launched without the attribute, both are no-ops.
LT_D void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
LT_D void pdl_release() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// ---------------------------------------------------------------- reductions
// Kahan-compensated FP64 accumulation per thread, then a warp/block tree into one partial
// per block; k_reduce_final sums the partials of a slot in a fixed order.
struct Kahan
{
    double s = 0.0, c = 0.0;
    LT_D void add(double v)
    {
        double y = v - c;
        double t = s + y;
        c = (t - s) - y;
        s = t;
    }
};

LT_D double block_sum(double v, double* sh)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r += sh[w];
    __syncthreads();
    return r;
}

// out[j] = sum of partials[j * nblk .. + nblk) (Kahan, fixed order), one block per slot j
template <int Unused = 0>
__global__ void k_reduce_final(const double* __restrict__ partials, int nblk, double* __restrict__ out)
{
    __shared__ double sh[32];
    const double* p = partials + (size_t)blockIdx.x * nblk;
    Kahan k;
    for (int b = threadIdx.x; b < nblk; b += blockDim.x) k.add(p[b]);
    double r = block_sum(k.s - k.c, sh);
    if (threadIdx.x == 0) out[blockIdx.x] = r;
}

// Link-parallel stencil kernels: a block of 128 threads covers the four directions of 32
// consecutive sites (warp w = direction w), so every plane load of a warp is coalesced and
// the neighbour links of a site block are shared through L1/L2 by all four directions.
constexpr int kSitesPerBlock = 32;

LT_D bool link_of_thread(const Geom& g, int& mu, int& x)
{
    mu = threadIdx.x >> 5;
    x = blockIdx.x * kSitesPerBlock + (threadIdx.x & 31);
    return x < g.V;
}

// The same with the site order reversed when rev != 0.  Consecutive launches over the same
// fields alternate the order, so each launch starts on the sites the previous one touched
// last, which are still in L2.
LT_D bool link_of_thread(const Geom& g, int& mu, int& x, int rev)
{
    const bool ok = link_of_thread(g, mu, x);
    if (rev) x = g.V - 1 - x;
    return ok;
}

// Thread -> checkerboard index of a half-lattice kernel, reversed when rev != 0 (as above)
LT_D bool half_site_of_thread(const Geom& g, int& s, int rev)
{
    s = blockIdx.x * blockDim.x + threadIdx.x;
    const bool ok = s < g.vh;
    if (rev) s = g.vh - 1 - s;
    return ok;
}

// ---------------------------------------------------------------- staple
// Rectangular<1>::StaplePlaq (actions/gauge/rectangular_action.hpp:104-184):
//   sum_{nu != mu} U_nu(x) U_mu(x+nu) U_nu(x+mu)^dag + U_nu(x-nu)^dag U_mu(x-nu) U_nu(x-nu+mu)
// summed in ascending nu, each direction as (up + down).
template <typename T, int NR>
LT_D M3<T> staple(const Gauge<T, NR>& U, const Geom& g, int par, int i, const int c[4], int mu)
{
    const int op = par ^ 1;
    const int dmu = step_up_rt(g, mu, c);
    const int imu = i + dmu;
    M3<T> acc = zero3<T>();
#pragma unroll
    for (int nu = 0; nu < 4; ++nu)
    {
        if (nu == mu) continue;
        const int inu = i + step_up_rt(g, nu, c);
        const int ind = i + step_dn_rt(g, nu, c);
        M3<T> up, dn;
#ifdef LT_STAPLE_FULL_PRODUCTS
        if (false)
#else
        if (NR == 2)
#endif
        {
            // Two-row storage: each three-link path is an SU(3) matrix, so only its first two
            // rows are multiplied out and the third is rebuilt (RestoreLastRow), which also
            // spares the reconstruction of the leading factor of the upper path.
            up = mul_nd_rows(mul_rows(U.ld_rows(nu, par, i >> 1), U.ld(mu, op, inu >> 1)), U.ld(nu, op, imu >> 1));
            dn = mul_rows(mul_dn_rows(U.ld(nu, op, ind >> 1), U.ld(mu, op, ind >> 1)), U.ld(nu, par, (ind + dmu) >> 1));
            // path by path with the third rows formed inside the sum, as in the staged staple
            // (identical rounding)
            acc_restored(acc, up);
            acc_restored(acc, dn);
            continue;
        }
        else
        {
            up = mul_nd(mul(U.ld(nu, par, i >> 1), U.ld(mu, op, inu >> 1)), U.ld(nu, op, imu >> 1));
            dn = mul(mul_dn(U.ld(nu, op, ind >> 1), U.ld(mu, op, ind >> 1)), U.ld(nu, par, (ind + dmu) >> 1));
        }
        acc = acc + (up + dn);
    }
    return acc;
}

// ---------------------------------------------------------------- staged staple
// For two-row FP32 storage the sweep, flow, stout and momentum kernels stage the 18 staple
// links and the updated link through shared memory: each thread copies the three links of a
// staple path with cp.async (16-byte chunks, L2 only) into its own slot of a two-path ring,
// one path ahead of its use, so the loads of the next path are in flight while the current
// one is multiplied and hold no registers meanwhile.  A slot is refilled only after the
// products that read it, in program order (the copies are asm volatile with a memory
// clobber); the thread that reads a slot is the one that filled it, so wait_group alone
// orders the copies before the reads.  Same paths and products as staple(), summed path by
// path.
#ifndef LT_STAGED_STAPLE
#define LT_STAGED_STAPLE 1
#endif
#ifndef LT_MINB_STAGED
#define LT_MINB_STAGED 6
#endif
#ifndef LT_STAGED_THREADS
#define LT_STAGED_THREADS 128
#endif
constexpr int kStagedThreads = LT_STAGED_THREADS;

LT_D void cp_async16(void* dst, const void* src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}
LT_D void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> LT_D void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Two slots of three links (nine float4 chunks) per thread of a block of NT threads: 36,864
// bytes for 128 threads
template <int NT> struct StapleRingT
{
    float4 c[2][9][NT];
};
using StapleRing = StapleRingT<kStagedThreads>;

template <int NT> LT_D void stage_link(StapleRingT<NT>& r, int slot, int j, const float4* q, int vh)
{
    const int t = threadIdx.x;
    cp_async16(&r.c[slot][3 * j][t], q);
    cp_async16(&r.c[slot][3 * j + 1][t], q + vh);
    cp_async16(&r.c[slot][3 * j + 2][t], q + 2 * (size_t)vh);
}

template <int NT> LT_D M3<float> staged_rows(const StapleRingT<NT>& r, int slot, int j)
{
    const int t = threadIdx.x;
    return Gauge<float, 2>::rows_of(r.c[slot][3 * j][t], r.c[slot][3 * j + 1][t], r.c[slot][3 * j + 2][t]);
}

template <int NT> LT_D M3<float> staged_link(const StapleRingT<NT>& r, int slot, int j)
{
    M3<float> m = staged_rows(r, slot, j);
    restore_last_row(m);
    return m;
}

// Copies the three links of a staple path of (mu, x) along nu into `slot`: the upper path
// U_nu(x) U_mu(x+nu) U_nu(x+mu)^dag, or the lower path U_nu(x-nu)^dag U_mu(x-nu) U_nu(x-nu+mu).
template <bool UP, int NT>
LT_D void stage_path(StapleRingT<NT>& r, int slot, const Gauge<float, 2>& U, const Geom& g, int par, int i,
                     const int c[4], int mu, int nu, int dmu)
{
    const int op = par ^ 1;
    if (UP)
    {
        const int inu = i + step_up_rt(g, nu, c);
        stage_link(r, slot, 0, U.chunk(nu, par, 0) + (i >> 1), U.vh);
        stage_link(r, slot, 1, U.chunk(mu, op, 0) + (inu >> 1), U.vh);
        stage_link(r, slot, 2, U.chunk(nu, op, 0) + ((i + dmu) >> 1), U.vh);
    }
    else
    {
        const int ind = i + step_dn_rt(g, nu, c);
        stage_link(r, slot, 0, U.chunk(nu, op, 0) + (ind >> 1), U.vh);
        stage_link(r, slot, 1, U.chunk(mu, op, 0) + (ind >> 1), U.vh);
        stage_link(r, slot, 2, U.chunk(nu, par, 0) + ((ind + dmu) >> 1), U.vh);
    }
}

// Staple of the link (mu, x) (site i, checkerboard index s) and, in `u`, the link itself.
// Slot 0 carries the upper paths, slot 1 the lower ones; the next direction's path is copied
// into a slot as soon as its current path is multiplied out, and the link itself follows the
// last upper path.  Each half-iteration commits one copy group (possibly empty), so waiting
// for all but the latest group always completes the path about to be used.  The direction
// loop is unrolled or not (ROLLED): the rolled loop keeps the larger heatbath and flow kernels
// within the instruction caches (measured faster there, the unrolled one for overrelaxation).
template <bool ROLLED, int NT>
LT_D M3<float> staple_staged(StapleRingT<NT>& r, const Gauge<float, 2>& U, const Geom& g, int par, int i, int s,
                             const int c[4], int mu, M3<float>& u)
{
    const int dmu = step_up_rt(g, mu, c);
    const int nu0 = mu == 0 ? 1 : 0;
    stage_path<true>(r, 0, U, g, par, i, c, mu, nu0, dmu);
    cp_async_commit();
    stage_path<false>(r, 1, U, g, par, i, c, mu, nu0, dmu);
    cp_async_commit();
    M3<float> acc = zero3<float>();
#pragma unroll(ROLLED ? 1 : 3)
    for (int n = 0; n < 3; ++n)
    {
        const int nn = (n + 1) + (n + 1 >= mu ? 1 : 0);   // the direction after this one
        cp_async_wait<1>();
        M3<float> p = mul_nd_rows(mul_rows(staged_rows(r, 0, 0), staged_link(r, 0, 1)), staged_link(r, 0, 2));
        acc_restored(acc, p);
        if (n < 2)
            stage_path<true>(r, 0, U, g, par, i, c, mu, nn, dmu);
        else
            stage_link(r, 0, 0, U.chunk(mu, par, 0) + s, U.vh);
        cp_async_commit();
        cp_async_wait<1>();
        p = mul_rows(mul_dn_rows(staged_link(r, 1, 0), staged_link(r, 1, 1)), staged_link(r, 1, 2));
        acc_restored(acc, p);
        if (n < 2) stage_path<false>(r, 1, U, g, par, i, c, mu, nn, dmu);
        cp_async_commit();
    }
    cp_async_wait<0>();
    u = staged_link(r, 0, 0);
    return acc;
}

// exp(c X) U followed by GramSchmidt (gradient_flow.hpp:265-282, hmc_gauge.hpp:505-523,
// stout_smearing.hpp:52-53).  With two-row storage only rows 0 and 1 are formed: the store
// keeps only those and every load rebuilds the third.
template <typename T, int NR> LT_D M3<T> exp_update(const M3<T>& X, T c, const M3<T>& u)
{
    const M3<T> e = exp_ah(X, c);
    if (NR == 2)
    {
        M3<T> r = mul_rows(e, u);
        gram_schmidt<T, false>(r);
        return r;
    }
    M3<T> r = mul(e, u);
    gram_schmidt(r);
    return r;
}

// ---------------------------------------------------------------- layout conversion
// reference links [l0, l1) (link index site*4+mu) of the AoS field at aos into U
template <typename T, int NR>
__global__ void k_from_aos(Gauge<T, NR> U, Geom g, const double* __restrict__ aos, int l0, int l1)
{
    int l = l0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= l1) return;
    int i = l >> 2, mu = l & 3;
    int c[4];
    int r = i;
    c[3] = r % g.n[3]; r /= g.n[3];
    c[2] = r % g.n[2]; r /= g.n[2];
    c[1] = r % g.n[1]; c[0] = r / g.n[1];
    int par = (c[0] + c[1] + c[2] + c[3]) & 1;
    const double* a = aos + (size_t)18 * l;
    M3<T> m;
#pragma unroll
    for (int k = 0; k < 9; ++k) m.e[k / 3][k % 3] = mkc<T>((T)a[2 * k], (T)a[2 * k + 1]);
    U.st(mu, par, i >> 1, m);
}

template <typename T, int NR>
__global__ void k_to_aos(Gauge<T, NR> U, Geom g, double* __restrict__ aos)
{
    int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= 4 * g.V) return;
    int i = l >> 2, mu = l & 3;
    int c[4];
    int r = i;
    c[3] = r % g.n[3]; r /= g.n[3];
    c[2] = r % g.n[2]; r /= g.n[2];
    c[1] = r % g.n[1]; c[0] = r / g.n[1];
    int par = (c[0] + c[1] + c[2] + c[3]) & 1;
    M3<T> m = U.ld(mu, par, i >> 1);
    double* a = aos + (size_t)18 * l;
#pragma unroll
    for (int k = 0; k < 9; ++k)
    {
        a[2 * k] = (double)m.e[k / 3][k % 3].r;
        a[2 * k + 1] = (double)m.e[k / 3][k % 3].i;
    }
}

// Algebra field <-> reference AoS (full 3x3 anti-Hermitian per link)
template <typename T>
__global__ void k_alg_from_aos(Alg<T> P, Geom g, const double* __restrict__ aos)
{
    int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= 4 * g.V) return;
    int i = l >> 2, mu = l & 3;
    int c[4];
    int r = i;
    c[3] = r % g.n[3]; r /= g.n[3];
    c[2] = r % g.n[2]; r /= g.n[2];
    c[1] = r % g.n[1]; c[0] = r / g.n[1];
    int par = (c[0] + c[1] + c[2] + c[3]) & 1;
    const double* a = aos + (size_t)18 * l;
    M3<T> m;
#pragma unroll
    for (int k = 0; k < 9; ++k) m.e[k / 3][k % 3] = mkc<T>((T)a[2 * k], (T)a[2 * k + 1]);
    P.st(mu, par, i >> 1, algebra8(m));
}

template <typename T>
__global__ void k_alg_to_aos(Alg<T> P, Geom g, double* __restrict__ aos)
{
    int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= 4 * g.V) return;
    int i = l >> 2, mu = l & 3;
    int c[4];
    int r = i;
    c[3] = r % g.n[3]; r /= g.n[3];
    c[2] = r % g.n[2]; r /= g.n[2];
    c[1] = r % g.n[1]; c[0] = r / g.n[1];
    int par = (c[0] + c[1] + c[2] + c[3]) & 1;
    M3<T> m = unpack_ah(P.ld(mu, par, i >> 1));
    double* a = aos + (size_t)18 * l;
#pragma unroll
    for (int k = 0; k < 9; ++k)
    {
        a[2 * k] = (double)m.e[k / 3][k % 3].r;
        a[2 * k + 1] = (double)m.e[k / 3][k % 3].i;
    }
}

template <typename T, int NR>
__global__ void k_set_unit(Gauge<T, NR> U, int nlink)
{
    int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nlink) return;
    int vh = U.vh;
    int plane = l / vh, s = l - plane * vh;
    U.st(plane >> 1, plane & 1, s, unit3<T>());
}

// One link <-> 18 doubles (element access of GaugeField4D, lattice.hpp:113-136)
template <typename T, int NR>
__global__ void k_link_io(Gauge<T, NR> U, Geom g, int site, int mu, double* __restrict__ m, int write)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int c[4];
    int r = site;
    c[3] = r % g.n[3]; r /= g.n[3];
    c[2] = r % g.n[2]; r /= g.n[2];
    c[1] = r % g.n[1]; c[0] = r / g.n[1];
    int par = (c[0] + c[1] + c[2] + c[3]) & 1;
    if (write)
    {
        M3<T> a;
#pragma unroll
        for (int k = 0; k < 9; ++k) a.e[k / 3][k % 3] = mkc<T>((T)m[2 * k], (T)m[2 * k + 1]);
        U.st(mu, par, site >> 1, a);
    }
    else
    {
        M3<T> a = U.ld(mu, par, site >> 1);
#pragma unroll
        for (int k = 0; k < 9; ++k)
        {
            m[2 * k] = (double)a.e[k / 3][k % 3].r;
            m[2 * k + 1] = (double)a.e[k / 3][k % 3].i;
        }
    }
}

// ---------------------------------------------------------------- plaquette
// PlaquetteSum (observables/plaquette.hpp:26-43): sum over sites and mu<nu of ReTr P_{mu nu}
template <typename T, int NR>
__global__ void __launch_bounds__(kRedThreads) k_plaquette(Gauge<T, NR> U, Geom g, double* __restrict__ partials)
{
    __shared__ double sh[32];
    Kahan k;
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < g.V; x += gridDim.x * blockDim.x)
    {
        int par = x >= g.vh, s = x - par * g.vh;
        int c[4];
        int i = site_coords(g, par, s, c);
        const int op = par ^ 1;
        double acc = 0.0;
#pragma unroll
        for (int mu = 0; mu < 4; ++mu)
        {
            const int imu = i + step_up_rt(g, mu, c);
            // products in FP64 whatever the storage: the action enters HMC's dH and the
            // plaquette the FP32-vs-FP64 error budget, so only storage rounding remains
            const M3<double> umu = cvt<double>(U.ld(mu, par, s));
#pragma unroll
            for (int nu = mu + 1; nu < 4; ++nu)
            {
                const int inu = i + step_up_rt(g, nu, c);
                // ReTr(U_mu(x) U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag) = ReTr[(U_mu(x) U_nu(x+mu)) (U_nu(x) U_mu(x+nu))^dag]
                M3<double> a = mul(umu, cvt<double>(U.ld(nu, op, imu >> 1)));
                M3<double> b = mul(cvt<double>(U.ld(nu, par, s)), cvt<double>(U.ld(mu, op, inu >> 1)));
                acc += retr_nd(a, b);
            }
        }
        k.add(acc);
    }
    double r = block_sum(k.s - k.c, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = r;
}

// ---------------------------------------------------------------- BMW configuration files
// Payload of the BMW format (IO/config_io/bmw_format.hpp:27-47): records in t, z, y, x order
// (x fastest), per record the links of directions x, y, z, t (mu = 1, 2, 3, 0), per link NW =
// 12 (first two rows) or 18 (#18BMW) doubles, row-major re/im, big-endian.  Checksum_Adler64
// (bmw_format.hpp:63-97) over record b of 4 NW native 64-bit words w_k, d0/d1 = high/low halves:
//   A_b = sum_k (d0 + d1),  B_b = sum_k (2 + r_k d0 + (r_k - 1) d1) mod p,
//   r_k = (V - b) * 2 * 4 NW - 2 k  (wrapping 64-bit arithmetic), p = 4294967291;
// A and B are sums over records mod p, so every record is summed independently and the
// partial sums are reduced per block (A in partials[block], B in partials[nblk + block]).
constexpr unsigned long long kAdler64Prime = 4294967291ULL;

LT_D unsigned long long bswap64(unsigned long long v)
{
    const unsigned lo = (unsigned)v, hi = (unsigned)(v >> 32);
    return ((unsigned long long)__byte_perm(lo, 0, 0x0123) << 32) | __byte_perm(hi, 0, 0x0123);
}

// Record b -> (coordinates, full index) in the reference site order
LT_D int bmw_site(const Geom& g, int b, int c[4])
{
    int r = b;
    c[1] = r % g.n[1];
    r /= g.n[1];
    c[2] = r % g.n[2];
    r /= g.n[2];
    c[3] = r % g.n[3];
    c[0] = r / g.n[3];
    return ((c[0] * g.n[1] + c[1]) * g.n[2] + c[2]) * g.n[3] + c[3];
}

LT_D void adler_word(unsigned long long w, unsigned long long& revi, unsigned long long& sa, unsigned long long& sb)
{
    const unsigned long long d0 = w >> 32, d1 = w & 0xFFFFFFFFULL;
    sa += d0 + d1;
    sb += (2ULL + revi * d0 + (revi - 1ULL) * d1) % kAdler64Prime;
    revi -= 2ULL;
}

LT_D void adler_block_store(unsigned long long sa, unsigned long long sb, unsigned long long* __restrict__ partials)
{
    __shared__ unsigned long long sh[2][32];
    sa %= kAdler64Prime;
    sb %= kAdler64Prime;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
    {
        sa += __shfl_xor_sync(0xffffffffu, sa, o);
        sb += __shfl_xor_sync(0xffffffffu, sb, o);
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0)
    {
        sh[0][wid] = sa;
        sh[1][wid] = sb;
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        unsigned long long a = 0, b = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w)
        {
            a += sh[0][w];
            b += sh[1][w];
        }
        partials[blockIdx.x] = a % kAdler64Prime;
        partials[gridDim.x + blockIdx.x] = b % kAdler64Prime;
    }
}

// Links -> big-endian payload (out may be null: checksum only)
template <typename T, int NR, int NW>
__global__ void __launch_bounds__(kRedThreads) k_bmw_pack(Gauge<T, NR> U, Geom g, unsigned long long* __restrict__ out,
                                                           unsigned long long* __restrict__ partials)
{
    unsigned long long sa = 0, sb = 0;
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < g.V; b += gridDim.x * blockDim.x)
    {
        int c[4];
        const int i = bmw_site(g, b, c);
        const int par = (c[0] + c[1] + c[2] + c[3]) & 1;
        unsigned long long revi = (unsigned long long)(g.V - b) * (unsigned long long)(8 * NW);
        unsigned long long* o = out ? out + (size_t)b * 4 * NW : nullptr;
#pragma unroll
        for (int dp = 0; dp < 4; ++dp)
        {
            const M3<double> m = cvt<double>(U.ld((dp + 1) & 3, par, i >> 1));
#pragma unroll
            for (int k = 0; k < NW; ++k)
            {
                const cx<double> e = m.e[k / 6][(k % 6) / 2];
                const unsigned long long w = (unsigned long long)__double_as_longlong((k & 1) ? e.i : e.r);
                adler_word(w, revi, sa, sb);
                if (o) o[dp * NW + k] = bswap64(w);
            }
        }
    }
    adler_block_store(sa, sb, partials);
}

// Reference complex arithmetic without contraction: RestoreLastRow (math/su3.hpp:362-367) as
// the reference's loader evaluates it, row 2 = conj(row0 x row1), each product rounded
LT_D cx<double> cmul_rn(cx<double> a, cx<double> b)
{
    return mkc<double>(__dsub_rn(__dmul_rn(a.r, b.r), __dmul_rn(a.i, b.i)),
                       __dadd_rn(__dmul_rn(a.r, b.i), __dmul_rn(a.i, b.r)));
}
LT_D cx<double> conj_cross_rn(cx<double> p, cx<double> q, cx<double> r, cx<double> s)
{
    const cx<double> x = cmul_rn(p, q), y = cmul_rn(r, s);
    return mkc<double>(__dsub_rn(x.r, y.r), -__dsub_rn(x.i, y.i));
}

// Big-endian payload -> links (third row rebuilt for NW = 12, in the reference's rounding);
// a link failing SU3::Tests::IsGroupElement (su3.hpp:568-578: |1 - U^dag U|_F or |det U - 1|
// above 1e-6) sets bit 0 of *flags.
template <typename T, int NR, int NW>
__global__ void __launch_bounds__(kRedThreads) k_bmw_unpack(Gauge<T, NR> U, Geom g, const unsigned long long* __restrict__ in,
                                                             unsigned long long* __restrict__ partials, unsigned* flags)
{
    unsigned long long sa = 0, sb = 0;
    bool bad = false;
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < g.V; b += gridDim.x * blockDim.x)
    {
        int c[4];
        const int i = bmw_site(g, b, c);
        const int par = (c[0] + c[1] + c[2] + c[3]) & 1;
        unsigned long long revi = (unsigned long long)(g.V - b) * (unsigned long long)(8 * NW);
        const unsigned long long* p = in + (size_t)b * 4 * NW;
#pragma unroll
        for (int dp = 0; dp < 4; ++dp)
        {
            M3<double> m = zero3<double>();
#pragma unroll
            for (int k = 0; k < NW; ++k)
            {
                const unsigned long long w = bswap64(p[dp * NW + k]);
                adler_word(w, revi, sa, sb);
                const double v = __longlong_as_double((long long)w);
                cx<double>& e = m.e[k / 6][(k % 6) / 2];
                if (k & 1) e.i = v;
                else e.r = v;
            }
            if (NW == 12)
            {
                m.e[2][0] = conj_cross_rn(m.e[0][1], m.e[1][2], m.e[0][2], m.e[1][1]);
                m.e[2][1] = conj_cross_rn(m.e[0][2], m.e[1][0], m.e[0][0], m.e[1][2]);
                m.e[2][2] = conj_cross_rn(m.e[0][0], m.e[1][1], m.e[0][1], m.e[1][0]);
            }
            // IsGroupElement: Frobenius norm of 1 - U^dag U and |det U - 1|
            double f2 = 0.0;
#pragma unroll
            for (int a = 0; a < 3; ++a)
#pragma unroll
                for (int bb = 0; bb < 3; ++bb)
                {
                    double re = a == bb ? 1.0 : 0.0, im = 0.0;
#pragma unroll
                    for (int k = 0; k < 3; ++k)
                    {
                        re -= m.e[k][a].r * m.e[k][bb].r + m.e[k][a].i * m.e[k][bb].i;
                        im -= m.e[k][a].r * m.e[k][bb].i - m.e[k][a].i * m.e[k][bb].r;
                    }
                    f2 += re * re + im * im;
                }
            const cx<double> det = m.e[0][0] * (m.e[1][1] * m.e[2][2] - m.e[1][2] * m.e[2][1])
                                 - m.e[0][1] * (m.e[1][0] * m.e[2][2] - m.e[1][2] * m.e[2][0])
                                 + m.e[0][2] * (m.e[1][0] * m.e[2][1] - m.e[1][1] * m.e[2][0]);
            const double dr = det.r - 1.0;
            bad |= !(f2 <= 1e-12) || !(dr * dr + det.i * det.i <= 1e-12);
            U.st((dp + 1) & 3, par, i >> 1, cvt<T>(m));
        }
    }
    if (bad) atomicOr(flags, 1u);
    adler_block_store(sa, sb, partials);
}

// ---------------------------------------------------------------- link health
// Scans every link: non-finite entries set kStatusNonFinite; the largest entry of
// |U U^dag - 1| (products in FP64, third row rebuilt for two-row storage) goes to *maxbits as
// the bits of a non-negative float (whose unsigned order is its numeric order), and a link
// above tol sets kStatusUnitarity.
template <typename T, int NR>
__global__ void __launch_bounds__(kRedThreads) k_check_links(Gauge<T, NR> U, Geom g, double tol, unsigned* status,
                                                              unsigned* maxbits)
{
    float dmax = 0.0f;
    bool bad = false;
    for (int l = blockIdx.x * blockDim.x + threadIdx.x; l < 4 * g.V; l += gridDim.x * blockDim.x)
    {
        const int pl = l / g.vh, s = l - pl * g.vh;
        const M3<double> u = cvt<double>(U.ld(pl >> 1, pl & 1, s));
        double d = 0.0;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j)
            {
                bad |= !isfinite(u.e[i][j].r) || !isfinite(u.e[i][j].i);
                double re = i == j ? -1.0 : 0.0, im = 0.0;
#pragma unroll
                for (int k = 0; k < 3; ++k)
                {
                    re += u.e[i][k].r * u.e[j][k].r + u.e[i][k].i * u.e[j][k].i;
                    im += u.e[i][k].i * u.e[j][k].r - u.e[i][k].r * u.e[j][k].i;
                }
                d = fmax(d, fmax(fabs(re), fabs(im)));
            }
        if (d > tol) atomicOr(status, kStatusUnitarity);
        dmax = fmaxf(dmax, (float)d);
    }
    if (bad) atomicOr(status, kStatusNonFinite);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dmax = fmaxf(dmax, __shfl_xor_sync(0xffffffffu, dmax, o));
    if ((threadIdx.x & 31) == 0) atomicMax(maxbits, __float_as_uint(dmax));
}

// ---------------------------------------------------------------- rectangular actions
// Full-index offset of a shift by d (|d| <= 2) along direction a of the site with coordinates c
LT_D int shift_offset(const Geom& g, const int c[4], int a, int d)
{
    const int n = pick4(g.n, a), x = pick4(c, a) + d;
    const int w = x < 0 ? n : x >= n ? -n : 0;
    return (d + w) * pick4(g.stride, a);
}

// Full index of x + dm mu + dn nu (periodic) for the site x = i with coordinates c
LT_D int site_at(const Geom& g, int i, const int c[4], int mu, int dm, int nu, int dn)
{
    return i + shift_offset(g, c, mu, dm) + shift_offset(g, c, nu, dn);
}

// Rectangular<2>::StapleRect (actions/gauge/rectangular_action.hpp:187-233): for each
// nu = mu+1, mu+2, mu+3 (mod 4), the 1x2 loops orthogonal to the link (up and down) and the
// 2x1 loops along it that start at x and at x - mu, each with U_mu(x) removed.
template <typename T, int NR>
LT_D M3<T> staple_rect(const Gauge<T, NR>& U, const Geom& g, int par, int i, const int c[4], int mu)
{
    // link U_d at x + dm mu + dn nu
    auto L = [&](int d, int nu, int dm, int dn) -> M3<T> {
        const int j = site_at(g, i, c, mu, dm, nu, dn);
        return U.ld(d, par ^ ((dm + dn) & 1), j >> 1);
    };
    M3<T> st = zero3<T>();
#pragma unroll 1
    for (int off = 1; off < 4; ++off)
    {
        const int nu = (mu + off) & 3;
        // orthogonal: U_nu(x) U_nu(x+nu) U_mu(x+2nu) U_nu(x+mu+nu)^dag U_nu(x+mu)^dag
        //           + U_nu(x-nu)^dag U_nu(x-2nu)^dag U_mu(x-2nu) U_nu(x+mu-2nu) U_nu(x+mu-nu)
        const M3<T> o_up = mul_nd(mul_nd(mul(mul(L(nu, nu, 0, 0), L(nu, nu, 0, 1)), L(mu, nu, 0, 2)), L(nu, nu, 1, 1)),
                                  L(nu, nu, 1, 0));
        const M3<T> o_dn = mul(mul(mul(mul_dd(L(nu, nu, 0, -1), L(nu, nu, 0, -2)), L(mu, nu, 0, -2)), L(nu, nu, 1, -2)),
                               L(nu, nu, 1, -1));
        acc(st, o_up + o_dn);
        // along the link from x: [U_nu(x) U_mu(x+nu) U_mu(x+mu+nu) U_nu(x+2mu)^dag
        //                        + U_nu(x-nu)^dag U_mu(x-nu) U_mu(x+mu-nu) U_nu(x+2mu-nu)] U_mu(x+mu)^dag
        const M3<T> f_up = mul_nd(mul(mul(L(nu, nu, 0, 0), L(mu, nu, 0, 1)), L(mu, nu, 1, 1)), L(nu, nu, 2, 0));
        const M3<T> f_dn = mul(mul(mul_dn(L(nu, nu, 0, -1), L(mu, nu, 0, -1)), L(mu, nu, 1, -1)), L(nu, nu, 2, -1));
        acc(st, mul_nd(f_up + f_dn, L(mu, nu, 1, 0)));
        // along the link from x - mu: U_mu(x-mu)^dag [U_nu(x-mu) U_mu(x-mu+nu) U_mu(x+nu) U_nu(x+mu)^dag
        //                        + U_nu(x-mu-nu)^dag U_mu(x-mu-nu) U_mu(x-nu) U_nu(x+mu-nu)]
        const M3<T> b_up = mul_nd(mul(mul(L(nu, nu, -1, 0), L(mu, nu, -1, 1)), L(mu, nu, 0, 1)), L(nu, nu, 1, 0));
        const M3<T> b_dn = mul(mul(mul_dn(L(nu, nu, -1, -1), L(mu, nu, -1, -1)), L(mu, nu, 0, -1)), L(nu, nu, 1, -1));
        acc(st, mul_dn(L(mu, nu, -1, 0), b_up + b_dn));
    }
    return st;
}

// The handle's gauge action on the device: Rectangular<1> (the plaquette staple alone, whatever
// c_plaq) or Rectangular<2> (c_plaq StaplePlaq + c_rect StapleRect; rectangular_action.hpp:236-246)
template <bool RECT, typename T, int NR>
LT_D M3<T> action_staple(const Gauge<T, NR>& U, const Geom& g, int par, int i, const int c[4], int mu, T cp, T cr)
{
    if constexpr (RECT)
    {
        M3<T> st = cp * staple(U, g, par, i, c, mu);
        acc(st, cr * staple_rect(U, g, par, i, c, mu));
        return st;
    }
    else
        return staple(U, g, par, i, c, mu);
}

// Iterator::Checkerboard4 (iterators/iterators.hpp:141-166): for direction mu the links whose
// sites satisfy (t + x + y + z + x_mu) mod 4 = sub (every extent a multiple of 4).  Thread k
// of the V/4 in a sub-sweep gets the k-th such site, z fastest: for mu != z a stride-4 run of
// z per (t, x, y) row, for mu = z a stride-2 run on the rows with t + x + y = sub (mod 2).
LT_D int cb4_site(const Geom& g, int mu, int sub, int k, int c[4])
{
    // divisions by n/4 and n/2 as floor(4x / n) and floor(2x / n) (4 V < 2^31)
    if (mu != 3)
    {
        const int nz = g.n[3] >> 2, row = div_by(g, 4 * k, 3), j = k - row * nz;
        const int r2 = div_by(g, row, 2);
        c[2] = row - r2 * g.n[2];
        c[0] = div_by(g, r2, 1);
        c[1] = r2 - c[0] * g.n[1];
        const int z0 = (sub - c[0] - c[1] - c[2] - pick4(c, mu)) & 3;
        c[3] = z0 + 4 * j;
    }
    else
    {
        const int nz = g.n[3] >> 1, row = div_by(g, 2 * k, 3), j = k - row * nz;
        const int ny = g.n[2] >> 1, q = div_by(g, 2 * row, 2), m = row - q * ny;
        c[0] = div_by(g, q, 1);
        c[1] = q - c[0] * g.n[1];
        c[2] = 2 * m + ((sub - c[0] - c[1]) & 1);
        const int z0 = ((sub - c[0] - c[1] - c[2]) & 3) >> 1;
        c[3] = z0 + 2 * j;
    }
    return ((c[0] * g.n[1] + c[1]) * g.n[2] + c[2]) * g.n[3] + c[3];
}

// ---------------------------------------------------------------- staple output (tests)
template <typename T, int NR, bool RECT>
__global__ void k_staple_aos(Gauge<T, NR> U, Geom g, double* __restrict__ aos, T cp, T cr)
{
    int mu, x;
    if (!link_of_thread(g, mu, x)) return;
    int par = x >= g.vh, s = x - par * g.vh;
    int c[4];
    int i = site_coords(g, par, s, c);
    M3<T> st = action_staple<RECT>(U, g, par, i, c, mu, cp, cr);
    double* a = aos + (size_t)18 * (4 * i + mu);
#pragma unroll
    for (int k = 0; k < 9; ++k)
    {
        a[2 * k] = (double)st.e[k / 3][k % 3].r;
        a[2 * k + 1] = (double)st.e[k / 3][k % 3].i;
    }
}

// ---------------------------------------------------------------- overrelaxation
// OverrelaxationSubgroupKernel (updates/overrelaxation.hpp:68-117) on the links of one
// (mu, parity) sub-sweep of Iterator::Checkerboard (iterators/iterators.hpp:65-87).
template <typename T> LT_D S2<T> or_su2(const S2<T>& A)
{
    T an = rsqrt_t<T>(s2_det(A));
    S2<T> V;
    V.e11 = an * A.e11;
    V.e12 = an * A.e12;
    return s2_adj(s2_mul(V, V));
}

// The three subgroup reflections of u against its staple, then Gram-Schmidt (the third row
// is not rebuilt for two-row storage, which does not keep it)
template <typename T, int NR> LT_D void or_apply(M3<T>& u, const M3<T>& st)
{
    M3<T> w = mul_nd(u, st);   // U st^dag
#pragma unroll
    for (int sg = 0; sg < 3; ++sg)
    {
        S2<T> h = or_su2(extract(w, sg));
        embed_lmul(h, sg, u);
        if (sg < 2) embed_lmul(h, sg, w);
    }
    gram_schmidt<T, NR == 3>(u);
}

template <typename T, int NR>
LT_D void or_update(const Gauge<T, NR>& U, const Geom& g, int mu, int par, int s)
{
    int c[4];
    int i = site_coords(g, par, s, c);
    M3<T> st = staple(U, g, par, i, c, mu);
    M3<T> u = U.ld(mu, par, s);
    or_apply<T, NR>(u, st);
    U.st(mu, par, s, u);
}

template <typename T, int NR>
__global__ void __launch_bounds__(kThreads, (OrMinBlocks<T, NR>::value)) k_overrelax(Gauge<T, NR> U, Geom g, int mu, int par, int rev)
{
    int s;
    const bool ok = half_site_of_thread(g, s, rev);
    pdl_release();
    pdl_wait();
    if (!ok) return;
    or_update(U, g, mu, par, s);
}

// The same on two-row FP32 storage with the staged staple (6 blocks of 128 per SM: the
// shared-memory ring of 36,864 bytes per block bounds residency)
template <int Unused = 0>
__global__ void __launch_bounds__(kStagedThreads, LT_MINB_STAGED) k_overrelax_staged(Gauge<float, 2> U, Geom g, int mu, int par, int rev)
{
    __shared__ StapleRing ring;
    int s;
    const bool ok = half_site_of_thread(g, s, rev);
    pdl_release();
    pdl_wait();
    if (!ok) return;
    int c[4];
    const int i = site_coords(g, par, s, c);
    M3<float> u;
    const M3<float> st = staple_staged<false>(ring, U, g, par, i, s, c, mu, u);
    or_apply<float, 2>(u, st);
    U.st(mu, par, s, u);
}

// One (mu, sublattice) sub-sweep of Iterator::Checkerboard4 with the handle's action
template <typename T, int NR, bool RECT>
__global__ void __launch_bounds__(kThreads, (RECT ? RectMinBlocks<T, NR>::value : Cb4MinBlocks<T, NR>::value)) k_overrelax4(Gauge<T, NR> U, Geom g, int mu, int sub, T cp, T cr, int rev)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    pdl_release();
    pdl_wait();
    if (k >= (g.V >> 2)) return;
    if (rev) k = (g.V >> 2) - 1 - k;   // descending on alternate launches, as half_site_of_thread
    int c[4];
    const int i = cb4_site(g, mu, sub, k, c);
    const int par = (c[0] + c[1] + c[2] + c[3]) & 1, s = i >> 1;
    const M3<T> st = action_staple<RECT>(U, g, par, i, c, mu, cp, cr);
    M3<T> u = U.ld(mu, par, s);
    or_apply<T, NR>(u, st);
    U.st(mu, par, s, u);
}

// ---------------------------------------------------------------- heatbath
// HeatbathKernel::HeatbathSU2 (updates/heatbath.hpp:47-104): Kennedy-Pendleton /
// Fabricius-Haan sampling of x0 with lambda^2 = -(prefactor/4)/sqrt(det A) (ln r1 + cos^2(2 pi r2) ln r3),
// accept while r0^2 + lambda^2 < 1, at most max_iter+1 proposals, else the unit matrix
// (reported through `capped`; the kernel then sets kStatusHbCap in the handle's status word).
// Random numbers: Philox4x32-10, counter {link, counter lo, counter hi, tag|subgroup|call}.
template <typename T> struct HB;

// Random numbers carried between the three subgroup draws of one FP32 update: the direction
// numbers of subgroup 1 (drawn with those of subgroup 0) and the low 8 bits of the four words
// of subgroup 0's and subgroup 1's last proposals (the FP32 uniforms use the high 24 bits only)
struct HbCarry
{
    float spare[2];
    uint32_t low[2];
};

template <> struct HB<double>
{
    LT_D static S2<double> su2(const S2<double>& A, double prefactor, uint32_t link, uint64_t counter,
                                uint32_t sg, uint32_t k0, uint32_t k1, int max_iter, bool& capped, HbCarry&)
    {
        double an = rsqrt(s2_det(A));
        const uint32_t c1 = (uint32_t)counter, c2 = (uint32_t)(counter >> 32);
        const uint32_t tw = (TAG_HEATBATH << 24) | (sg << 16);
        double lsq = 0.0;
        for (int k = 0;; ++k)
        {
            U4 a = philox4x32(link, c1, c2, tw | (uint32_t)(2 * k), k0, k1);
            U4 b = philox4x32(link, c1, c2, tw | (uint32_t)(2 * k + 1), k0, k1);
            double r1 = 1.0 - u01_from(a.x, a.y), r2 = 1.0 - u01_from(a.z, a.w);
            double r3 = 1.0 - u01_from(b.x, b.y), r0 = u01_from(b.z, b.w);
            double x2 = cospi(2.0 * r2);
            lsq = -0.25 * prefactor * an * (log(r1) + x2 * x2 * log(r3));
            if (k > max_iter)
            {
                capped = true;
                S2<double> one;
                one.e11 = mkc(1.0, 0.0);
                one.e12 = mkc(0.0, 0.0);
                return one;
            }
            if (r0 * r0 + lsq < 1.0) break;
        }
        double x0 = 1.0 - 2.0 * lsq;
        double ax = sqrt(1.0 - x0 * x0);
        U4 d = philox4x32(link, c1, c2, tw | 0xFFFFu, k0, k1);
        double phi = u01_from(d.x, d.y);
        double ct = 1.0 - 2.0 * u01_from(d.z, d.w);
        double vn = ax * sqrt(1.0 - ct * ct);
        double sp, cp;
        sincospi(2.0 * phi, &sp, &cp);
        S2<double> x, V;
        x.e11 = mkc(x0, vn * cp);
        x.e12 = mkc(vn * sp, ax * ct);
        V.e11 = an * A.e11;
        V.e12 = an * A.e12;
        return s2_mul(x, s2_adj(V));
    }
};

// FP32: the special functions use the SFU approximations (__logf, __cosf, __sincosf, absolute
// error about 1e-6 on these arguments), below the FP32 rounding of the rest of the update;
// FP32 chains are validated statistically against the reference's chains.
// Philox calls per update: one per proposal and one more for all three directions.  The
// direction numbers of subgroups 0 and 1 come from one call (words x, y for subgroup 0; z, w,
// kept in carry.spare, for subgroup 1); those of subgroup 2 from the unused low bytes of the
// last proposals of subgroups 0 and 1 (each proposal word feeds a 24-bit uniform from its high
// bits; the low 8 bits of four words make one further 32-bit word, uniform and independent of
// the accept/reject test, which saw only the high bits).
LT_D uint32_t low_bytes(const U4& a)
{
    return (a.x & 0xffu) | ((a.y & 0xffu) << 8) | ((a.z & 0xffu) << 16) | ((a.w & 0xffu) << 24);
}

template <> struct HB<float>
{
    LT_D static S2<float> su2(const S2<float>& A, float prefactor, uint32_t link, uint64_t counter,
                               uint32_t sg, uint32_t k0, uint32_t k1, int max_iter, bool& capped, HbCarry& carry)
    {
        float an = rsqrtf(s2_det(A));
        const uint32_t c1 = (uint32_t)counter, c2 = (uint32_t)(counter >> 32);
        const uint32_t tw = (TAG_HEATBATH << 24) | (sg << 16);
        float lsq = 0.0f;
        for (int k = 0;; ++k)
        {
            U4 a = philox4x32(link, c1, c2, tw | (uint32_t)k, k0, k1);
            float r1 = 1.0f - f01_from(a.x), r2 = 1.0f - f01_from(a.y);
            float r3 = 1.0f - f01_from(a.z), r0 = f01_from(a.w);
            float x2 = __cosf(kTwoPiF * r2);
            lsq = -0.25f * prefactor * an * (__logf(r1) + x2 * x2 * __logf(r3));
            if (sg < 2) carry.low[sg] = low_bytes(a);
            if (k > max_iter)
            {
                capped = true;
                if (sg == 0)   // subgroup 1 still takes its direction numbers from this draw
                {
                    const U4 d = philox4x32(link, c1, c2, tw | 0xFFFFu, k0, k1);
                    carry.spare[0] = f01_from(d.z);
                    carry.spare[1] = 1.0f - 2.0f * f01_from(d.w);
                }
                S2<float> one;
                one.e11 = mkc(1.0f, 0.0f);
                one.e12 = mkc(0.0f, 0.0f);
                return one;
            }
            if (r0 * r0 + lsq < 1.0f) break;
        }
        float x0 = 1.0f - 2.0f * lsq;
        float ax = sqrt_approx(fmaxf(1.0f - x0 * x0, 0.0f));
        float phi, ct;
        if (sg == 1)
        {
            phi = carry.spare[0];
            ct = carry.spare[1];
        }
        else if (sg == 2)
        {
            phi = f01_from(carry.low[0]);
            ct = 1.0f - 2.0f * f01_from(carry.low[1]);
        }
        else
        {
            const U4 d = philox4x32(link, c1, c2, tw | 0xFFFFu, k0, k1);
            phi = f01_from(d.x);
            ct = 1.0f - 2.0f * f01_from(d.y);
            carry.spare[0] = f01_from(d.z);
            carry.spare[1] = 1.0f - 2.0f * f01_from(d.w);
        }
        float vn = ax * sqrt_approx(fmaxf(1.0f - ct * ct, 0.0f));
        float sp, cp;
        __sincosf(kTwoPiF * phi, &sp, &cp);
        S2<float> x, V;
        x.e11 = mkc(x0, vn * cp);
        x.e12 = mkc(vn * sp, ax * ct);
        V.e11 = an * A.e11;
        V.e12 = an * A.e12;
        return s2_mul(x, s2_adj(V));
    }
};

// HeatbathKernel::operator() (updates/heatbath.hpp:110-129) for one (mu, parity) sub-sweep
template <typename T, int NR>
__global__ void __launch_bounds__(kThreads, (HbMinBlocks<T, NR>::value)) k_heatbath(Gauge<T, NR> U, Geom g, int mu, int par, T prefactor,
                                                       uint64_t counter, uint32_t k0, uint32_t k1, int max_iter,
                                                       unsigned* status, int rev)
{
    int s;
    const bool ok = half_site_of_thread(g, s, rev);
    pdl_release();
    pdl_wait();
    if (!ok) return;
    hb_update(U, g, mu, par, s, prefactor, counter, k0, k1, max_iter, status);
}

template <typename T, int NR>
LT_D void hb_core(const Gauge<T, NR>& U, int mu, int par, int s, int i, const M3<T>& st, T prefactor,
                  uint64_t counter, uint32_t k0, uint32_t k1, int max_iter, unsigned* status);

template <typename T, int NR>
LT_D void hb_update(const Gauge<T, NR>& U, const Geom& g, int mu, int par, int s, T prefactor, uint64_t counter,
                    uint32_t k0, uint32_t k1, int max_iter, unsigned* status)
{
    int c[4];
    int i = site_coords(g, par, s, c);
    hb_core(U, mu, par, s, i, staple(U, g, par, i, c, mu), prefactor, counter, k0, k1, max_iter, status);
}

template <typename T, int NR>
LT_D void hb_core_u(const Gauge<T, NR>& U, int mu, int par, int s, int i, M3<T> u, const M3<T>& st, T prefactor,
                    uint64_t counter, uint32_t k0, uint32_t k1, int max_iter, unsigned* status);

// k_heatbath on two-row FP32 storage with the staged staple
template <int Unused = 0>
__global__ void __launch_bounds__(kStagedThreads, LT_MINB_STAGED) k_heatbath_staged(Gauge<float, 2> U, Geom g, int mu, int par,
                                                                 float prefactor, uint64_t counter, uint32_t k0,
                                                                 uint32_t k1, int max_iter, unsigned* status, int rev)
{
    __shared__ StapleRing ring;
    int s;
    const bool ok = half_site_of_thread(g, s, rev);
    pdl_release();
    pdl_wait();
    if (!ok) return;
    int c[4];
    const int i = site_coords(g, par, s, c);
    M3<float> u;
    const M3<float> st = staple_staged<true>(ring, U, g, par, i, s, c, mu, u);
    hb_core_u(U, mu, par, s, i, u, st, prefactor, counter, k0, k1, max_iter, status);
}

// One (mu, sublattice) sub-sweep of Iterator::Checkerboard4 with the handle's action
template <typename T, int NR, bool RECT>
__global__ void __launch_bounds__(kThreads, (RECT ? RectMinBlocks<T, NR>::value : Cb4MinBlocks<T, NR>::value)) k_heatbath4(Gauge<T, NR> U, Geom g, int mu, int sub, T prefactor,
                                                        uint64_t counter, uint32_t k0, uint32_t k1, int max_iter,
                                                        unsigned* status, T cp, T cr, int rev)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    pdl_release();
    pdl_wait();
    if (k >= (g.V >> 2)) return;
    if (rev) k = (g.V >> 2) - 1 - k;
    int c[4];
    const int i = cb4_site(g, mu, sub, k, c);
    const int par = (c[0] + c[1] + c[2] + c[3]) & 1;
    hb_core(U, mu, par, i >> 1, i, action_staple<RECT>(U, g, par, i, c, mu, cp, cr), prefactor, counter, k0, k1,
            max_iter, status);
}

// Cabibbo-Marinari update of U_mu at site i (checkerboard index s) against the staple st
template <typename T, int NR>
LT_D void hb_core(const Gauge<T, NR>& U, int mu, int par, int s, int i, const M3<T>& st, T prefactor,
                  uint64_t counter, uint32_t k0, uint32_t k1, int max_iter, unsigned* status)
{
    hb_core_u(U, mu, par, s, i, U.ld(mu, par, s), st, prefactor, counter, k0, k1, max_iter, status);
}

// The same with the link u already loaded
template <typename T, int NR>
LT_D void hb_core_u(const Gauge<T, NR>& U, int mu, int par, int s, int i, M3<T> u, const M3<T>& st, T prefactor,
                    uint64_t counter, uint32_t k0, uint32_t k1, int max_iter, unsigned* status)
{
    M3<T> w = mul_nd(u, st);
    const uint32_t link = (uint32_t)(4 * i + mu);
    bool capped = false;
    HbCarry carry = { { 0.0f, 0.0f }, { 0u, 0u } };
    // unrolled so that the subgroup rows are compile-time indices (keeps u and w in registers)
#pragma unroll
    for (int sg = 0; sg < 3; ++sg)
    {
        S2<T> h = HB<T>::su2(extract(w, sg), prefactor, link, counter, (uint32_t)sg, k0, k1, max_iter, capped, carry);
        embed_lmul(h, sg, u);
        if (sg < 2) embed_lmul(h, sg, w);
    }
    gram_schmidt<T, NR == 3>(u);
    U.st(mu, par, s, u);
    if (capped && status) atomicOr(status, kStatusHbCap);
}

// ---------------------------------------------------------------- batched sweeps
// Many lattices of any even extents (one storage format) advanced by one launch per
// (mu, parity) sub-sweep: each lattice owns a contiguous range of blocks, found by binary
// search over the block offsets.  Small lattices (12^4 has 10,368 sites per parity) cannot
// fill 148 SMs alone; packed together they do.
struct LatDesc
{
    Geom g;
    void* U;
    double prefactor;   // 3 / beta of this lattice (heatbath.hpp:40)
    uint32_t k0, k1;    // Philox key of this lattice
    int blk_begin[3];   // first block of this lattice for blocks of 64, 128 and 256 threads
    unsigned* status;   // the lattice handle's status word
};

constexpr int kBatchBlocks[3] = { 64, 128, 256 };

template <int SEL> LT_D int find_lattice(const LatDesc* __restrict__ d, int n, int b)
{
    int lo = 0, hi = n - 1;
    while (lo < hi)
    {
        const int mid = (lo + hi + 1) >> 1;
        if (d[mid].blk_begin[SEL] <= b) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Registers capped at the level tuned for the single-lattice sweeps: 640 resident threads per
// SM in FP32, 384 in FP64, and 768 for the staged two-row FP32 kernels of 64 and 128 threads,
// whose ring allows 6 blocks of 128 per SM (+2 % over 640; the unstaged FP32 kernels spill at
// 768)
#ifndef LT_BATCH_THREADS_F32C
#define LT_BATCH_THREADS_F32C 768
#endif
template <typename T, int NR, int BLOCK> struct BatchMinBlocks
{
    static constexpr int per_sm = (sizeof(T) == 4 && NR == 2 && LT_STAGED_STAPLE && BLOCK <= 128)
                                      ? LT_BATCH_THREADS_F32C
                                      : (sizeof(T) == 4 ? 640 : 384);
    static constexpr int value = per_sm / BLOCK > 0 ? per_sm / BLOCK : 1;
};

template <typename T, int NR, int SEL, int OP>   // OP: 0 heatbath, 1 overrelaxation
__global__ void __launch_bounds__(kBatchBlocks[SEL], (BatchMinBlocks<T, NR, kBatchBlocks[SEL]>::value))
    k_batch_sweep(const LatDesc* __restrict__ d, int n, int mu, int par, const uint64_t* __restrict__ counter,
                  int max_iter, int flip)
{
    constexpr int BLOCK = kBatchBlocks[SEL];
    // flip: the work units in descending order, so that a launch starts on the lattices the
    // previous one (ascending) ended on, which are still in L2
    const int b = flip ? (int)(gridDim.x - 1 - blockIdx.x) : (int)blockIdx.x;
    const int k = find_lattice<SEL>(d, n, b);
    const Geom g = d[k].g;
    const int s = (b - d[k].blk_begin[SEL]) * BLOCK + threadIdx.x;
    if (s >= g.vh) return;
    Gauge<T, NR> U;
    U.p = (cx<T>*)d[k].U;
    U.vh = g.vh;
    if constexpr (LT_STAGED_STAPLE && std::is_same<T, float>::value && NR == 2 && BLOCK <= 128)
    {
        // two-row FP32 links: the staged staple of the single-lattice sweeps
        __shared__ StapleRingT<BLOCK> ring;
        int c[4];
        const int i = site_coords(g, par, s, c);
        M3<float> u;
        const M3<float> st = staple_staged<OP == 0>(ring, U, g, par, i, s, c, mu, u);
        if (OP == 0)
            hb_core_u(U, mu, par, s, i, u, st, (T)d[k].prefactor, *counter, d[k].k0, d[k].k1, max_iter, d[k].status);
        else
        {
            or_apply<float, 2>(u, st);
            U.st(mu, par, s, u);
        }
    }
    else if (OP == 0)
        hb_update(U, g, mu, par, s, (T)d[k].prefactor, *counter, d[k].k0, d[k].k1, max_iter, d[k].status);
    else
        or_update(U, g, mu, par, s);
}

// ---------------------------------------------------------------- persistent batched round
// One launch for a whole round (n_hb heatbath + n_or overrelaxation sweeps, 8 (mu, parity)
// sub-sweeps each) over all lattices of an ensemble: the grid is cooperative (every block
// resident at once), each block walks the batch's work units (the blocks of k_batch_sweep)
// of a sub-sweep with a grid stride, and a grid barrier separates consecutive sub-sweeps.
//
// The barrier waits a bounded time: a block that waits more than `limit` polls, or that sees
// another block's timeout flag, sets kStatusBarrierTimeout in *status and the whole kernel
// returns early (the links are then inconsistent and the host reports an error).  Nothing
// here can hang: every wait either sees the last arrival or gives up.
struct GridBarrier
{
    unsigned* count;     // arrivals at the current barrier (zeroed by the host before the launch)
    unsigned* gen;       // generation, bumped by the last arrival
    unsigned* status;    // kStatusBarrierTimeout on give-up
    long long limit;     // polls before giving up (each poll sleeps about 100 ns)
};

LT_D bool grid_barrier(const GridBarrier& b)
{
    __shared__ int ok_s;
    __syncthreads();
    if (threadIdx.x == 0)
    {
        int ok = 1;
        volatile unsigned* vgen = b.gen;
        volatile unsigned* vstatus = b.status;
        const unsigned g = *vgen;
        __threadfence();   // this block's link updates before its arrival
        const unsigned arrived = atomicAdd(b.count, 1u);
        if (arrived == gridDim.x - 1)
        {
            atomicExch(b.count, 0u);
            __threadfence();
            atomicAdd(b.gen, 1u);
        }
        else
        {
            long long polls = 0;
            while (*vgen == g)
            {
                if (++polls > b.limit || (*vstatus & kStatusBarrierTimeout))
                {
                    ok = 0;
                    break;
                }
                __nanosleep(100);
            }
        }
        if (!ok) atomicOr(b.status, kStatusBarrierTimeout);
        __threadfence();   // the other blocks' updates before this block reads them
        ok_s = ok;
    }
    __syncthreads();
    return ok_s != 0;
}

// One work unit u of a batched sub-sweep (the body of k_batch_sweep for block u)
template <typename T, int NR, int BLOCK, int RB>
LT_D void batch_unit(StapleRingT<RB>& ring, const LatDesc* __restrict__ d, int n, int u, int op, int mu, int par,
                     uint64_t counter, int max_iter)
{
    const int k = find_lattice<BLOCK == 64 ? 0 : BLOCK == 128 ? 1 : 2>(d, n, u);
    const int sel = BLOCK == 64 ? 0 : BLOCK == 128 ? 1 : 2;
    const Geom g = d[k].g;
    const int s = (u - d[k].blk_begin[sel]) * BLOCK + threadIdx.x;
    if (s >= g.vh) return;
    Gauge<T, NR> U;
    U.p = (cx<T>*)d[k].U;
    U.vh = g.vh;
    if constexpr (LT_STAGED_STAPLE && std::is_same<T, float>::value && NR == 2 && BLOCK <= 128 && RB == BLOCK)
    {
        int c[4];
        const int i = site_coords(g, par, s, c);
        M3<float> uu;
        if (op == 0)
        {
            const M3<float> st = staple_staged<true>(ring, U, g, par, i, s, c, mu, uu);
            hb_core_u(U, mu, par, s, i, uu, st, (T)d[k].prefactor, counter, d[k].k0, d[k].k1, max_iter, d[k].status);
        }
        else
        {
            const M3<float> st = staple_staged<false>(ring, U, g, par, i, s, c, mu, uu);
            or_apply<float, 2>(uu, st);
            U.st(mu, par, s, uu);
        }
    }
    else if (op == 0)
        hb_update(U, g, mu, par, s, (T)d[k].prefactor, counter, d[k].k0, d[k].k1, max_iter, d[k].status);
    else
        or_update(U, g, mu, par, s);
}

#ifndef LT_PERSIST_POLLS
#define LT_PERSIST_POLLS 10000000   // about one second of polling at ~100 ns per poll
#endif

// Blocks of 128 threads (the staged kernels' tuned size); register cap as k_batch_sweep's
// Work units are handed out dynamically: each block takes the next unit of the current
// sub-sweep from the sub-sweep's own counter in next[] (zeroed by the host before the launch),
// as the hardware scheduler hands out the blocks of a batched launch.
template <typename T, int NR>
__global__ void __launch_bounds__(128, (BatchMinBlocks<T, NR, 128>::value))
    k_batch_round(const LatDesc* __restrict__ d, int n, int n_units, int n_hb, int n_or, int reverse,
                  uint64_t* __restrict__ counter, int max_iter, GridBarrier bar, unsigned* __restrict__ next)
{
    // the staged staple's ring for two-row FP32 links; a token one otherwise
    constexpr bool kStagedRound = LT_STAGED_STAPLE && std::is_same<T, float>::value && NR == 2;
    __shared__ StapleRingT<kStagedRound ? 128 : 1> ring;
    __shared__ int unit_s;
    const uint64_t c0 = *counter;
    const int n_sub = 8 * (n_hb + n_or);
    for (int q = 0; q < n_sub; ++q)
    {
        // the reference's order (iterators.hpp:65-87): n_hb heatbath sweeps then n_or
        // overrelaxation sweeps, (mu, parity) lexicographic within each; reversed in full.
        // Heatbath sweeps take consecutive counter values in the order they run.
        const int qq = reverse ? n_sub - 1 - q : q;
        const int sweep = qq >> 3, idx = qq & 7;
        const int op = sweep < n_hb ? 0 : 1;
        const int hb_rank = reverse ? n_hb - 1 - sweep : sweep;
        const uint64_t cnt = c0 + (uint64_t)(op == 0 ? hb_rank : 0);
        const int mu = idx >> 1, par = idx & 1;
        for (;;)
        {
            if (threadIdx.x == 0) unit_s = (int)atomicAdd(&next[q], 1u);
            __syncthreads();
            const int u = unit_s;
            __syncthreads();   // every thread has read unit_s before thread 0 overwrites it
            if (u >= n_units) break;
            batch_unit<T, NR, 128>(ring, d, n, u, op, mu, par, cnt, max_iter);
        }
        if (q + 1 < n_sub && !grid_barrier(bar)) return;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *counter = c0 + (uint64_t)n_hb;
}

// Advances the device-side sweep counter (read by the heatbath inside captured graphs)
template <int Unused = 0> __global__ void k_counter_add(uint64_t* c, uint64_t n)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) *c += n;
}

// ---------------------------------------------------------------- gradient flow
// One fused RK3 stage (smearing/gradient_flow.hpp:120-168, :265-332): for every link
//   Z   <- c_old Z + c_new Algebra(st U^dag)   (CalculateZ / UpdateZ)
//   U'  <- exp(c_exp Z) U, Gram-Schmidt          (UpdateFields)
// reading U from Uin and writing Uout (ping-pong), so all staples see the pre-stage field
// exactly as the reference's separate Z and field sweeps do.
template <typename T, int NR, bool RECT>
__global__ void __launch_bounds__(kThreads, (LinkMinBlocks<T, NR>::value)) k_flow_stage(Gauge<T, NR> Uin, Gauge<T, NR> Uout, Alg<T> Z, Geom g,
                                                         T c_old, T c_new, T c_exp, int read_z, int write_z, T cp, T cr,
                                                         int rev)
{
    pdl_release();
    pdl_wait();
    int mu, x;
    if (!link_of_thread(g, mu, x, rev)) return;
    int par = x >= g.vh, s = x - par * g.vh;
    int c[4];
    int i = site_coords(g, par, s, c);
    M3<T> u = Uin.ld(mu, par, s);
    M3<T> st = action_staple<RECT>(Uin, g, par, i, c, mu, cp, cr);
    A8<T> a = algebra8(mul_nd(st, u));
    A8<T> z;
    if (read_z)
    {
        A8<T> zo = Z.ld(mu, par, s);
#pragma unroll
        for (int k = 0; k < 8; ++k) z.a[k] = c_old * zo.a[k] + c_new * a.a[k];
    }
    else
    {
#pragma unroll
        for (int k = 0; k < 8; ++k) z.a[k] = c_new * a.a[k];
    }
    if (write_z) Z.st(mu, par, s, z);
    Uout.st(mu, par, s, exp_update<T, NR>(unpack_ah(z), c_exp, u));
}

// k_flow_stage (Wilson action) on two-row FP32 storage with the staged staple; Z of the link
// is read before the staple so that its loads are in flight meanwhile
#ifndef LT_MINB_FLOW_STAGED
#define LT_MINB_FLOW_STAGED 5
#endif
template <int Unused = 0>
__global__ void __launch_bounds__(4 * kSitesPerBlock, LT_MINB_FLOW_STAGED)
    k_flow_stage_staged(Gauge<float, 2> Uin, Gauge<float, 2> Uout, Alg<float> Z, Geom g, float c_old, float c_new,
                        float c_exp, int read_z, int write_z, int rev)
{
    static_assert(4 * kSitesPerBlock == kStagedThreads, "one ring slot per thread");
    __shared__ StapleRing ring;
    pdl_release();
    pdl_wait();
    int mu, x;
    if (!link_of_thread(g, mu, x, rev)) return;
    const int par = x >= g.vh, s = x - par * g.vh;
    int c[4];
    const int i = site_coords(g, par, s, c);
    A8<float> z;
    if (read_z)
        z = Z.ld(mu, par, s);
    M3<float> u;
    const M3<float> st = staple_staged<true>(ring, Uin, g, par, i, s, c, mu, u);
    const A8<float> a = algebra8(mul_nd(st, u));
#pragma unroll
    for (int k = 0; k < 8; ++k) z.a[k] = read_z ? c_old * z.a[k] + c_new * a.a[k] : c_new * a.a[k];
    if (write_z) Z.st(mu, par, s, z);
    Uout.st(mu, par, s, exp_update<float, 2>(unpack_ah(z), c_exp, u));
}

// ---------------------------------------------------------------- Zeuthen flow
// The Zeuthen flow (Ramos and Sint, Eur. Phys. J. C 76 (2016) 15, arXiv:1508.05552; not in the
// reference, which flows with the simulated action's force only, gradient_flow.hpp:298-332):
// the force of the Luescher-Weisz action, X_mu(x) = Algebra(st_LW U_mu(x)^dag), acted on by
// (1 + 1/12 nabla*_mu nabla_mu), the adjoint covariant second difference along the link:
//   F_mu(x) = X_mu(x) + 1/12 [U_mu(x) X_mu(x+mu) U_mu(x)^dag
//                             + U_mu(x-mu)^dag X_mu(x-mu) U_mu(x-mu) - 2 X_mu(x)],
// integrated with the stages of the flow integrators exactly as the plain force.
// Pass 1 of a stage: X for every link.
// (Also the first half of the split FP64 flow stage, below, with the handle's action.)
// The rectangle force pass (the Zeuthen flow's Luescher-Weisz force) on two-row FP32 links:
// 6 blocks of 128 per SM (80 registers; the spills, 412 bytes, stay in L1) for 14.8 Zeuthen
// RK3 steps/s at 48^4, against 14.6 at 5 blocks, 14.2 at 4 (128 registers) and 12.5 uncapped
// (149 registers, 3 blocks)
#ifndef LT_MINB_FLOW_FORCE_RECT_F32C
#define LT_MINB_FLOW_FORCE_RECT_F32C 6
#endif
template <typename T, int NR, bool RECT> struct FlowForceMinBlocks
{
    static constexpr int value = (sizeof(T) == 4 && NR == 2 && RECT) ? LT_MINB_FLOW_FORCE_RECT_F32C : 1;
};
template <typename T, int NR, bool RECT>
__global__ void __launch_bounds__(kThreads, (FlowForceMinBlocks<T, NR, RECT>::value)) k_flow_force(Gauge<T, NR> U, Alg<T> X, Geom g, T cp, T cr, int rev)
{
    pdl_release();
    pdl_wait();
    int mu, x;
    if (!link_of_thread(g, mu, x, rev)) return;
    const int par = x >= g.vh, s = x - par * g.vh;
    int c[4];
    const int i = site_coords(g, par, s, c);
    const M3<T> u = U.ld(mu, par, s);
    X.st(mu, par, s, algebra8(mul_nd(action_staple<RECT>(U, g, par, i, c, mu, cp, cr), u)));
}

// The second half of a split flow stage: Z <- c_old Z + c_new X, U' = exp(c_exp Z) U, with
// X = Algebra(st U^dag) from k_flow_force.  FP64 links run the stage as these two kernels:
// the fused stage needs 254 registers (two blocks of 128 per SM), the halves far fewer each.
template <typename T, int NR>
__global__ void __launch_bounds__(kThreads) k_flow_update(Gauge<T, NR> Uin, Gauge<T, NR> Uout, Alg<T> Z, Alg<T> X,
                                                          Geom g, T c_old, T c_new, T c_exp, int read_z, int write_z,
                                                          int rev)
{
    pdl_release();
    pdl_wait();
    int mu, x;
    if (!link_of_thread(g, mu, x, rev)) return;
    const int par = x >= g.vh, s = x - par * g.vh;
    const A8<T> a = X.ld(mu, par, s);
    A8<T> z;
    if (read_z)
    {
        const A8<T> zo = Z.ld(mu, par, s);
#pragma unroll
        for (int k = 0; k < 8; ++k) z.a[k] = c_old * zo.a[k] + c_new * a.a[k];
    }
    else
    {
#pragma unroll
        for (int k = 0; k < 8; ++k) z.a[k] = c_new * a.a[k];
    }
    if (write_z) Z.st(mu, par, s, z);
    Uout.st(mu, par, s, exp_update<T, NR>(unpack_ah(z), c_exp, Uin.ld(mu, par, s)));
}

// Pass 2: the Zeuthen force from X at x and x +- mu, then the stage's Z update and exponential
// update (as k_flow_stage), Uin -> Uout
template <typename T, int NR>
__global__ void __launch_bounds__(kThreads) k_flow_zeuthen_stage(Gauge<T, NR> Uin, Gauge<T, NR> Uout, Alg<T> Z,
                                                                 Alg<T> X, Geom g, T c_old, T c_new, T c_exp,
                                                                 int read_z, int write_z, int rev)
{
    pdl_release();
    pdl_wait();
    int mu, x;
    if (!link_of_thread(g, mu, x, rev)) return;
    const int par = x >= g.vh, s = x - par * g.vh, op = par ^ 1;
    int c[4];
    const int i = site_coords(g, par, s, c);
    const int ip = (i + step_up_rt(g, mu, c)) >> 1, im = (i + step_dn_rt(g, mu, c)) >> 1;
    const M3<T> u = Uin.ld(mu, par, s);
    const M3<T> um = Uin.ld(mu, op, im);
    const M3<T> xc = unpack_ah(X.ld(mu, par, s));
    const M3<T> fwd = mul_nd(mul(u, unpack_ah(X.ld(mu, op, ip))), u);
    const M3<T> bwd = mul(mul_dn(um, unpack_ah(X.ld(mu, op, im))), um);
    M3<T> f = xc;
    const T k12 = (T)(1.0 / 12.0);
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b)
        {
            f.e[a][b].r += k12 * (fwd.e[a][b].r + bwd.e[a][b].r - (T)2 * xc.e[a][b].r);
            f.e[a][b].i += k12 * (fwd.e[a][b].i + bwd.e[a][b].i - (T)2 * xc.e[a][b].i);
        }
    const A8<T> a = algebra8(f);
    A8<T> z;
    if (read_z)
    {
        const A8<T> zo = Z.ld(mu, par, s);
#pragma unroll
        for (int k = 0; k < 8; ++k) z.a[k] = c_old * zo.a[k] + c_new * a.a[k];
    }
    else
    {
#pragma unroll
        for (int k = 0; k < 8; ++k) z.a[k] = c_new * a.a[k];
    }
    if (write_z) Z.st(mu, par, s, z);
    Uout.st(mu, par, s, exp_update<T, NR>(unpack_ah(z), c_exp, u));
}

// ---------------------------------------------------------------- stout smearing
// StoutSmearing4D (smearing/stout_smearing.hpp:29-57): U' = exp(rho Algebra(st U^dag)) U, Gram-Schmidt
// With St.p set, the staple of every link is also stored (the metadynamics force's Lambda
// kernel reads it back instead of recomputing it).
template <typename T, int NR>
__global__ void __launch_bounds__(kThreads, (LinkMinBlocks<T, NR>::value)) k_stout(Gauge<T, NR> Uin, Gauge<T, NR> Uout, Geom g, T rho,
                                                    Full<T> St)
{
    pdl_release();
    pdl_wait();
    int mu, x;
    if (!link_of_thread(g, mu, x)) return;
    int par = x >= g.vh, s = x - par * g.vh;
    int c[4];
    int i = site_coords(g, par, s, c);
    M3<T> u = Uin.ld(mu, par, s);
    M3<T> st = staple(Uin, g, par, i, c, mu);
    if (St.p) St.st(mu, par, s, st);
    Uout.st(mu, par, s, exp_update<T, NR>(unpack_ah(algebra8(mul_nd(st, u))), rho, u));
}

// k_stout on two-row FP32 storage with the staged staple
template <int Unused = 0>
__global__ void __launch_bounds__(4 * kSitesPerBlock, LT_MINB_FLOW_STAGED)
    k_stout_staged(Gauge<float, 2> Uin, Gauge<float, 2> Uout, Geom g, float rho, Full<float> St)
{
    __shared__ StapleRing ring;
    pdl_release();
    pdl_wait();
    int mu, x;
    if (!link_of_thread(g, mu, x)) return;
    const int par = x >= g.vh, s = x - par * g.vh;
    int c[4];
    const int i = site_coords(g, par, s, c);
    M3<float> u;
    const M3<float> st = staple_staged<true>(ring, Uin, g, par, i, s, c, mu, u);
    if (St.p) St.st(mu, par, s, st);
    Uout.st(mu, par, s, exp_update<float, 2>(unpack_ah(algebra8(mul_nd(st, u))), rho, u));
}

// ---------------------------------------------------------------- clover observables
// Read-only view of a link field that widens every loaded link to FP64, so that measurements
// (Q, E) run their products in FP64 whatever the storage.
template <typename T, int NR> struct Widened
{
    Gauge<T, NR> U;
    LT_D M3<double> ld(int mu, int par, int s) const { return cvt<double>(U.ld(mu, par, s)); }
};

// Four-leaf clover C_{mu nu}(x) (observables/clover.hpp:94-152, plaquette.hpp:82-114), in the
// arithmetic type of the field view F (Gauge<T, NR> or Widened<T, NR>).
template <typename F>
LT_D auto clover_leaves(const F& U, const Geom& g, int par, int i, const int c[4], int mu, int nu)
{
    using M = decltype(U.ld(0, 0, 0));
    const int op = par ^ 1;
    const int dmu_p = step_up_rt(g, mu, c), dmu_m = step_dn_rt(g, mu, c);
    const int dnu_p = step_up_rt(g, nu, c), dnu_m = step_dn_rt(g, nu, c);
    const int s = i >> 1;
    const M umu = U.ld(mu, par, s), unu = U.ld(nu, par, s);
    const int imd = i + dmu_m, ind = i + dnu_m;
    // I:   U_mu(x) U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag
    M leaf = mul_nd(mul(umu, U.ld(nu, op, (i + dmu_p) >> 1)), mul(unu, U.ld(mu, op, (i + dnu_p) >> 1)));
    // II:  U_nu(x) U_mu(x-mu+nu)^dag U_nu(x-mu)^dag U_mu(x-mu)
    M umu_md = U.ld(mu, op, imd >> 1);
    acc(leaf, mul(mul_nd(unu, U.ld(mu, par, (imd + dnu_p) >> 1)), mul_dn(U.ld(nu, op, imd >> 1), umu_md)));
    // III: U_mu(x-mu)^dag U_nu(x-mu-nu)^dag U_mu(x-mu-nu) U_nu(x-nu)
    const int imdnd = imd + dnu_m;
    acc(leaf, mul(mul_dd(umu_md, U.ld(nu, par, imdnd >> 1)), mul(U.ld(mu, par, imdnd >> 1), U.ld(nu, op, ind >> 1))));
    // IV:  U_nu(x-nu)^dag U_mu(x-nu) U_nu(x-nu+mu) U_mu(x)^dag
    acc(leaf, mul_nd(mul(mul_dn(U.ld(nu, op, ind >> 1), U.ld(mu, op, ind >> 1)), U.ld(nu, par, (ind + dmu_p) >> 1)), umu));
    return leaf;
}

// Per-site clover charge density q(x) = ReTr(F01 F23 - F02 F13 + F03 F12), F = C - C^dag
// (observables/topological_charge.hpp:97-200) and energy density
// e(x) = sum_{mu<nu} ReTr(F~^2), F~ = Traceless(-i/8 (C - C^dag))
// (observables/field_strength_tensor.hpp:28-66, :107-134, :154-175).
// Products run in FP64 for every storage: the cancellations in F = C - C^dag of a smooth
// (flowed) field would otherwise lift FP32 rounding of the leaves into Q and E.
// Unnormalised clover densities of one site: q = ReTr(F01 F23 - F02 F13 + F03 F12) and
// e = sum_{mu<nu} ReTr(F~^2) with F = C - C^dag, F~ = Traceless(-i/8 F)
template <typename T, int NR>
LT_D void clover_densities(const Widened<T, NR>& U, const Geom& g, int par, int i, const int c[4], double& q, double& e)
{
    q = 0.0;
    e = 0.0;
    const int pairs[3][4] = { { 0, 1, 2, 3 }, { 0, 2, 1, 3 }, { 0, 3, 1, 2 } };
#pragma unroll 1
    for (int p = 0; p < 3; ++p)
    {
        M3<double> ca = clover_leaves(U, g, par, i, c, pairs[p][0], pairs[p][1]);
        M3<double> cb = clover_leaves(U, g, par, i, c, pairs[p][2], pairs[p][3]);
        M3<double> fa = ca - adj(ca), fb = cb - adj(cb);
        double t = retr_mul(fa, fb);
        q += p == 1 ? -t : t;
        // energy: F~ = -i/8 F made traceless; ReTr(F~^2) = sum |F~_ij|^2 (Hermitian)
#pragma unroll
        for (int h = 0; h < 2; ++h)
        {
            const M3<double>& f = h == 0 ? fa : fb;
            double tr3 = (f.e[0][0].i + f.e[1][1].i + f.e[2][2].i) / 3.0;
            double acc2 = 0.0;
#pragma unroll
            for (int a = 0; a < 3; ++a)
            {
                double d = f.e[a][a].i - tr3;
                acc2 += d * d;
#pragma unroll
                for (int b = 0; b < 3; ++b)
                    if (a != b) acc2 += norm2(f.e[a][b]);
            }
            e += acc2 * (1.0 / 64.0);
        }
    }
}

template <typename T, int NR>
__global__ void __launch_bounds__(kRedThreads) k_clover_obs(Gauge<T, NR> Ust, Geom g, double* __restrict__ partials)
{
    __shared__ double sh[32];
    const Widened<T, NR> U{ Ust };
    Kahan kq, ke;
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < g.V; x += gridDim.x * blockDim.x)
    {
        int par = x >= g.vh, s = x - par * g.vh;
        int c[4];
        int i = site_coords(g, par, s, c);
        double q, e;
        clover_densities(U, g, par, i, c, q, e);
        kq.add(q);
        ke.add(e);
    }
    double rq = block_sum(kq.s - kq.c, sh);
    double re = block_sum(ke.s - ke.c, sh);
    if (threadIdx.x == 0)
    {
        partials[blockIdx.x] = rq;
        partials[gridDim.x + blockIdx.x] = re;
    }
}

// CalculateClover<1, 1> (observables/clover.hpp:94-152) into a FullTensor4D in the reference
// layout double[V][4][4][3][3][2] (lattice.hpp:447-590, index ((site 4 + mu) 4 + nu)):
// C_{mu nu} for mu < nu from FP64 products, C_{nu mu} = C_{mu nu}^dag; the diagonal is left to
// the caller's zeroed buffer.  One thread per (site, plane mu < nu).
template <typename T, int NR>
__global__ void k_clover_tensor(Gauge<T, NR> Ust, Geom g, double* __restrict__ out)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 6LL * g.V) return;
    const int plane = (int)(t % 6), x = (int)(t / 6);
    const int mu = plane < 3 ? 0 : plane < 5 ? 1 : 2;
    const int nu = plane < 3 ? plane + 1 : plane < 5 ? plane - 1 : 3;
    const Widened<T, NR> U{ Ust };
    const int par = x >= g.vh, s = x - par * g.vh;
    int c[4];
    const int i = site_coords(g, par, s, c);
    const M3<double> C = clover_leaves(U, g, par, i, c, mu, nu);
    double* a = out + (size_t)18 * (16 * (size_t)i + 4 * mu + nu);
    double* b = out + (size_t)18 * (16 * (size_t)i + 4 * nu + mu);
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int q = 0; q < 3; ++q)
        {
            a[6 * r + 2 * q] = C.e[r][q].r;
            a[6 * r + 2 * q + 1] = C.e[r][q].i;
            b[6 * q + 2 * r] = C.e[r][q].r;
            b[6 * q + 2 * r + 1] = -C.e[r][q].i;
        }
}

// TopChargeClover(const FullTensor&) (observables/topological_charge.hpp:202-231): per site
// F_{mu nu} = C_{mu nu} - C_{nu mu} from the tensor as given, ReTr(F01 F23 - F02 F13 + F03 F12),
// Kahan-summed per thread, block partials to partials[blockIdx.x]
LT_D M3<double> tensor_entry(const double* __restrict__ C, int i, int mu, int nu)
{
    const double* p = C + (size_t)18 * (16 * (size_t)i + 4 * mu + nu);
    M3<double> m;
#pragma unroll
    for (int k = 0; k < 9; ++k) m.e[k / 3][k % 3] = mkc(p[2 * k], p[2 * k + 1]);
    return m;
}

template <int Unused = 0>
__global__ void __launch_bounds__(kRedThreads) k_topcharge_tensor(const double* __restrict__ C, int V,
                                                                  double* __restrict__ partials)
{
    __shared__ double sh[32];
    Kahan k;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < V; i += gridDim.x * blockDim.x)
    {
        const int pairs[3][4] = { { 0, 1, 2, 3 }, { 0, 2, 1, 3 }, { 0, 3, 1, 2 } };
        double q = 0.0;
#pragma unroll 1
        for (int p = 0; p < 3; ++p)
        {
            const M3<double> fa = tensor_entry(C, i, pairs[p][0], pairs[p][1]) - tensor_entry(C, i, pairs[p][1], pairs[p][0]);
            const M3<double> fb = tensor_entry(C, i, pairs[p][2], pairs[p][3]) - tensor_entry(C, i, pairs[p][3], pairs[p][2]);
            const double t = retr_mul(fa, fb);
            q += p == 1 ? -t : t;
        }
        k.add(q);
    }
    const double r = block_sum(k.s - k.c, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = r;
}

// ---------------------------------------------------------------- measurement bundle
// The observables of the reference driver's measurement step (SU3_main.cpp:89-235), all with
// products in FP64 whatever the storage.

// Coordinates and parity of the site with full index i
LT_D int coords_of(const Geom& g, int i, int c[4])
{
    const int r = div_by(g, i, 3);
    c[3] = i - r * g.n[3];
    const int r2 = div_by(g, r, 2);
    c[2] = r - r2 * g.n[2];
    c[0] = div_by(g, r2, 1);
    c[1] = r2 - c[0] * g.n[1];
    return (c[0] + c[1] + c[2] + c[3]) & 1;
}

// Full index of the site c moved by L steps along d (periodic)
LT_D int shifted(const Geom& g, const int c[4], int d, int L)
{
    const int i = ((c[0] * g.n[1] + c[1]) * g.n[2] + c[2]) * g.n[3] + c[3];
    const int n = pick4(g.n, d), x = pick4(c, d);
    return i + ((x + L) % n - x) * pick4(g.stride, d);
}

// TopChargeCloverTimeslice / EnergyDensity::CloverTimeslice (topological_charge.hpp:338-364,
// field_strength_tensor.hpp:178-195): block (bx, t) sums the clover densities of timeslice t;
// partials[t * nbx + bx] (q) and partials[(Nt + t) * nbx + bx] (e)
template <typename T, int NR>
__global__ void __launch_bounds__(kRedThreads) k_clover_timeslice(Gauge<T, NR> Ust, Geom g, double* __restrict__ partials)
{
    __shared__ double sh[32];
    const Widened<T, NR> U{ Ust };
    const int t = blockIdx.y, nbx = gridDim.x;
    const int vs = g.V / g.n[0];
    Kahan kq, ke;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < vs; k += nbx * blockDim.x)
    {
        const int i = t * vs + k;
        int c[4];
        const int par = coords_of(g, i, c);
        double q, e;
        clover_densities(U, g, par, i, c, q, e);
        kq.add(q);
        ke.add(e);
    }
    double rq = block_sum(kq.s - kq.c, sh);
    double re = block_sum(ke.s - ke.c, sh);
    if (threadIdx.x == 0)
    {
        partials[t * nbx + blockIdx.x] = rq;
        partials[(g.n[0] + t) * nbx + blockIdx.x] = re;
    }
}

// Per site over the six planes mu < nu: the plaquette traces (slot 0), the 1x2 and 2x1 loop
// traces of Rectangular<2>::Action (slot 1; rectangular_action.hpp:61-94, wilson_loop.hpp:155-175)
// and the plaquette charge density of TopChargePlaquette (slot 2; topological_charge.hpp:366-416)
template <typename T, int NR>
__global__ void __launch_bounds__(kRedThreads) k_loops(Gauge<T, NR> Ust, Geom g, double* __restrict__ partials)
{
    __shared__ double sh[32];
    const Widened<T, NR> U{ Ust };
    Kahan kp, kr, kq;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.V; i += gridDim.x * blockDim.x)
    {
        int c[4];
        const int par = coords_of(g, i, c), op = par ^ 1;
        M3<double> F[6];
        double sp = 0.0, sr = 0.0;
        int pl = 0;
#pragma unroll 1
        for (int mu = 0; mu < 4; ++mu)
#pragma unroll 1
            for (int nu = mu + 1; nu < 4; ++nu, ++pl)
            {
                const int imu = shifted(g, c, mu, 1), inu = shifted(g, c, nu, 1);
                int cmu[4], cnu[4];
                coords_of(g, imu, cmu);
                coords_of(g, inu, cnu);
                const int imunu = shifted(g, cmu, nu, 1), imu2 = shifted(g, cmu, mu, 1), inu2 = shifted(g, cnu, nu, 1);
                const M3<double> umu = U.ld(mu, par, i >> 1), unu = U.ld(nu, par, i >> 1);
                const M3<double> unu_mu = U.ld(nu, op, imu >> 1), umu_nu = U.ld(mu, op, inu >> 1);
                // P = U_mu(x) U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag
                const M3<double> a = mul(umu, unu_mu);
                const M3<double> p = mul_nd(a, mul(unu, umu_nu));
                sp += p.e[0][0].r + p.e[1][1].r + p.e[2][2].r;
                F[pl] = p - adj(p);   // times -i below
                // 1x2: U_mu(x) U_nu(x+mu) U_nu(x+mu+nu) U_mu(x+2nu)^dag U_nu(x+nu)^dag U_nu(x)^dag
                const M3<double> r12 = mul_nd(mul(a, U.ld(nu, par, imunu >> 1)),
                                              mul(mul(unu, U.ld(nu, op, inu >> 1)), U.ld(mu, par, inu2 >> 1)));
                // 2x1: U_mu(x) U_mu(x+mu) U_nu(x+2mu) U_mu(x+mu+nu)^dag U_mu(x+nu)^dag U_nu(x)^dag
                const M3<double> r21 = mul_nd(mul(mul(umu, U.ld(mu, op, imu >> 1)), U.ld(nu, par, imu2 >> 1)),
                                              mul(mul(unu, umu_nu), U.ld(mu, par, imunu >> 1)));
                sr += r12.e[0][0].r + r12.e[1][1].r + r12.e[2][2].r + r21.e[0][0].r + r21.e[1][1].r + r21.e[2][2].r;
            }
        // F_mu,nu = -i (P - P^dag); Re tr(F01 F23 + F02 F31 + F03 F12) with F31 = -F13 and
        // (-i)^2 = -1: -(G01 G23 - G02 G13 + G03 G12) for G = P - P^dag (planes 01 02 03 12 13 23)
        const double q = -(retr_mul(F[0], F[5]) - retr_mul(F[1], F[4]) + retr_mul(F[2], F[3]));
        kp.add(sp);
        kr.add(sr);
        kq.add(q);
    }
    double a = block_sum(kp.s - kp.c, sh);
    double b = block_sum(kr.s - kr.c, sh);
    double d = block_sum(kq.s - kq.c, sh);
    if (threadIdx.x == 0)
    {
        partials[blockIdx.x] = a;
        partials[gridDim.x + blockIdx.x] = b;
        partials[2 * gridDim.x + blockIdx.x] = d;
    }
}

// Straight line products for WilsonLoop (observables/wilson_loop.hpp:63-124), kept as full
// FP64 matrices C_mu(x) = U_mu(x) U_mu(x+mu) ... U_mu(x+(L-1)mu): init (L = 1), extension by one
// link (L -> L+1) and doubling (L -> 2L)
template <typename T, int NR>
__global__ void k_chain_init(Gauge<T, NR> Ust, Full<double> C, Geom g)
{
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= 4 * g.V) return;
    const int pl = l / g.vh, s = l - pl * g.vh;
    C.st(pl >> 1, pl & 1, s, cvt<double>(Ust.ld(pl >> 1, pl & 1, s)));
}

template <int Unused = 0>
__global__ void k_chain_unit(Full<double> C, Geom g)
{
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= 4 * g.V) return;
    const int pl = l / g.vh, s = l - pl * g.vh;
    C.st(pl >> 1, pl & 1, s, unit3<double>());
}

template <typename T, int NR>
__global__ void k_chain_extend(Full<double> Cin, Gauge<T, NR> Ust, Full<double> Cout, Geom g, int L)
{
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= 4 * g.V) return;
    const int pl = l / g.vh, s = l - pl * g.vh, mu = pl >> 1, par = pl & 1;
    int c[4];
    const int i = site_coords(g, par, s, c);
    (void)i;
    const int j = shifted(g, c, mu, L);
    int cj[4];
    const int pj = coords_of(g, j, cj);
    Cout.st(mu, par, s, mul(Cin.ld(mu, par, s), cvt<double>(Ust.ld(mu, pj, j >> 1))));
}

template <int Unused = 0>
__global__ void k_chain_double(Full<double> Cin, Full<double> Cout, Geom g, int L)
{
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= 4 * g.V) return;
    const int pl = l / g.vh, s = l - pl * g.vh, mu = pl >> 1, par = pl & 1;
    int c[4];
    site_coords(g, par, s, c);
    const int j = shifted(g, c, mu, L);
    int cj[4];
    const int pj = coords_of(g, j, cj);
    Cout.st(mu, par, s, mul(Cin.ld(mu, par, s), Cin.ld(mu, pj, j >> 1)));
}

// sum over sites and mu < nu of Re tr(C_mu(x) C_nu(x+L mu) C_mu(x+L nu)^dag C_nu(x)^dag)
template <int Unused = 0>
__global__ void __launch_bounds__(kRedThreads) k_wilson_square(Full<double> C, Geom g, int L, double* __restrict__ partials)
{
    __shared__ double sh[32];
    Kahan k;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.V; i += gridDim.x * blockDim.x)
    {
        int c[4];
        const int par = coords_of(g, i, c);
        double w = 0.0;
#pragma unroll 1
        for (int mu = 0; mu < 4; ++mu)
        {
            const M3<double> cmu = C.ld(mu, par, i >> 1);
            const int jm = shifted(g, c, mu, L);
            int cm[4];
            const int pm = coords_of(g, jm, cm);
#pragma unroll 1
            for (int nu = mu + 1; nu < 4; ++nu)
            {
                const int jn = shifted(g, c, nu, L);
                int cn[4];
                const int pn = coords_of(g, jn, cn);
                const M3<double> a = mul(cmu, C.ld(nu, pm, jm >> 1));
                const M3<double> b = mul(C.ld(nu, par, i >> 1), C.ld(mu, pn, jn >> 1));
                w += retr_nd(a, b);
            }
        }
        k.add(w);
    }
    double r = block_sum(k.s - k.c, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = r;
}

// PolyakovLoop (observables/polyakov_loop.hpp:32-49): tr of the product of the Nt links in
// direction t over every spatial site; re in slot 0, im in slot 1
template <typename T, int NR>
__global__ void __launch_bounds__(kRedThreads) k_polyakov(Gauge<T, NR> Ust, Geom g, double* __restrict__ partials)
{
    __shared__ double sh[32];
    const int vs = g.V / g.n[0];
    Kahan kr, ki;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < vs; k += gridDim.x * blockDim.x)
    {
        M3<double> m = unit3<double>();
        for (int t = 0; t < g.n[0]; ++t)
        {
            const int i = t * vs + k;
            int c[4];
            const int par = coords_of(g, i, c);
            m = mul(m, cvt<double>(Ust.ld(0, par, i >> 1)));
        }
        const cx<double> tr = trace(m);
        kr.add(tr.r);
        ki.add(tr.i);
    }
    double a = block_sum(kr.s - kr.c, sh);
    double b = block_sum(ki.s - ki.c, sh);
    if (threadIdx.x == 0)
    {
        partials[blockIdx.x] = a;
        partials[gridDim.x + blockIdx.x] = b;
    }
}

// ---------------------------------------------------------------- HMC
// HMC momentum kick P += eps * (beta/6 Algebra(st U^dag) + F)  (updates/hmc_gauge.hpp:450-464,
// updates/hmc_metadynamics.hpp:441-459).  With P = null the force itself is written to F_out.
template <typename T, int NR, bool RECT>
__global__ void __launch_bounds__(kThreads, (LinkMinBlocks<T, NR>::value)) k_momenta(Gauge<T, NR> U, Alg<T> P, Alg<T> F, Geom g, T coef, T eps, int use_f, T cp, T cr)
{
    int mu, x;
    if (!link_of_thread(g, mu, x)) return;
    int par = x >= g.vh, s = x - par * g.vh;
    int c[4];
    int i = site_coords(g, par, s, c);
    M3<T> st = action_staple<RECT>(U, g, par, i, c, mu, cp, cr);
    A8<T> a = algebra8(mul_nd(st, U.ld(mu, par, s)));
    A8<T> p = P.ld(mu, par, s);
    if (use_f)
    {
        A8<T> f = F.ld(mu, par, s);
#pragma unroll
        for (int k = 0; k < 8; ++k) p.a[k] += eps * (coef * a.a[k] + f.a[k]);
    }
    else
    {
#pragma unroll
        for (int k = 0; k < 8; ++k) p.a[k] += eps * coef * a.a[k];
    }
    P.st(mu, par, s, p);
}

// k_momenta (Wilson action) on two-row FP32 storage with the staged staple; P (and F) of the
// link are read before the staple so that their loads are in flight meanwhile
template <int Unused = 0>
__global__ void __launch_bounds__(4 * kSitesPerBlock, LT_MINB_FLOW_STAGED)
    k_momenta_staged(Gauge<float, 2> U, Alg<float> P, Alg<float> F, Geom g, float coef, float eps, int use_f)
{
    __shared__ StapleRing ring;
    int mu, x;
    if (!link_of_thread(g, mu, x)) return;
    const int par = x >= g.vh, s = x - par * g.vh;
    int c[4];
    const int i = site_coords(g, par, s, c);
    A8<float> p = P.ld(mu, par, s), f;
    if (use_f)
        f = F.ld(mu, par, s);
    M3<float> u;
    const M3<float> st = staple_staged<true>(ring, U, g, par, i, s, c, mu, u);
    const A8<float> a = algebra8(mul_nd(st, u));
#pragma unroll
    for (int k = 0; k < 8; ++k) p.a[k] += use_f ? eps * (coef * a.a[k] + f.a[k]) : eps * coef * a.a[k];
    P.st(mu, par, s, p);
}

// U <- exp(eps P) U, Gram-Schmidt (updates/hmc_gauge.hpp:505-523)
template <typename T, int NR>
__global__ void __launch_bounds__(kThreads) k_fields(Gauge<T, NR> U, Alg<T> P, int nlink, T eps)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nlink) return;
    int vh = U.vh;
    int plane = t / vh, s = t - plane * vh;
    int mu = plane >> 1, par = plane & 1;
    U.st(mu, par, s, exp_update<T, NR>(unpack_ah(P.ld(mu, par, s)), eps, U.ld(mu, par, s)));
}

// P <- a P + b F over the flat algebra field (n reals; F may be null): the Metadynamics
// momentum update with a stored force (updates/hmc_metadynamics.hpp:478-491), ReverseMomenta
// (updates/hmc_gauge.hpp:432-446) and the friction factor of UpdateMomentaFriction (:469-503)
template <typename T>
__global__ void k_alg_axpby(T* __restrict__ P, const T* __restrict__ F, size_t n, T a, T b)
{
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride)
        P[k] = F ? a * P[k] + b * F[k] : a * P[k];
}

// ParityUpdate (updates/parity_update.hpp:22-47): the spatial reflection x -> -x - 1 (per
// spatial extent), out of place.  Time links move with their sites; a spatial link U_i(x)
// becomes the adjoint of the reflected link that ends at the reflected site.
template <typename T, int NR>
__global__ void __launch_bounds__(kThreads) k_parity(Gauge<T, NR> Uin, Gauge<T, NR> Uout, Geom g)
{
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= 4 * g.V) return;
    const int pl = l / g.vh, s = l - pl * g.vh, mu = pl >> 1, par = pl & 1;
    int c[4];
    site_coords(g, par, s, c);
    int r1 = g.n[1] - c[1] - 1, r2 = g.n[2] - c[2] - 1, r3 = g.n[3] - c[3] - 1;
    if (mu == 1) r1 = r1 > 0 ? r1 - 1 : g.n[1] - 1;
    if (mu == 2) r2 = r2 > 0 ? r2 - 1 : g.n[2] - 1;
    if (mu == 3) r3 = r3 > 0 ? r3 - 1 : g.n[3] - 1;
    const int j = ((c[0] * g.n[1] + r1) * g.n[2] + r2) * g.n[3] + r3;
    const int pj = (c[0] + r1 + r2 + r3) & 1;
    const M3<T> m = Uin.ld(mu, pj, j >> 1);
    Uout.st(mu, par, s, mu == 0 ? m : adj(m));
}

// RandomMomentum (updates/hmc_gauge.hpp:400-428): P = 1/2 i phi_a lambda_a with eight
// Box-Muller Gaussians from Philox calls j = 0..3 of tag TAG_MOMENTA.
template <typename T>
__global__ void k_random_momenta(Alg<T> P, Geom g, uint64_t counter, uint32_t k0, uint32_t k1)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 4 * g.V) return;
    int plane = t / g.vh, s = t - plane * g.vh;
    int mu = plane >> 1, par = plane & 1;
    int c[4];
    int i = site_coords(g, par, s, c);
    const uint32_t link = (uint32_t)(4 * i + mu);
    double phi[8];
#pragma unroll
    for (int j = 0; j < 4; ++j)
    {
        U4 w = philox4x32(link, (uint32_t)counter, (uint32_t)(counter >> 32), (TAG_MOMENTA << 24) | (uint32_t)j, k0, k1);
        double u1 = u01_from(w.x, w.y), u2 = u01_from(w.z, w.w);
        double r = sqrt(-2.0 * log(1.0 - u1));
        double sp, cp;
        sincospi(2.0 * u2, &sp, &cp);
        phi[2 * j] = r * cp;
        phi[2 * j + 1] = r * sp;
    }
    const double is3 = 0.57735026918962576451;
    A8<T> a;
    a.a[0] = (T)(0.5 * (phi[2] + phi[7] * is3));
    a.a[1] = (T)(0.5 * (-phi[2] + phi[7] * is3));
    a.a[2] = (T)(0.5 * phi[1]);
    a.a[3] = (T)(0.5 * phi[0]);
    a.a[4] = (T)(0.5 * phi[4]);
    a.a[5] = (T)(0.5 * phi[3]);
    a.a[6] = (T)(0.5 * phi[6]);
    a.a[7] = (T)(0.5 * phi[5]);
    P.st(mu, par, s, a);
}

// Kinetic energy -sum ReTr(P^2) (updates/hmc_gauge.hpp:525-541) = sum_ij |P_ij|^2
template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_kinetic(Alg<T> P, int nlink, double* __restrict__ partials)
{
    __shared__ double sh[32];
    Kahan k;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nlink; t += gridDim.x * blockDim.x)
    {
        int vh = P.vh;
        int plane = t / vh, s = t - plane * vh;
        A8<T> a = P.ld(plane >> 1, plane & 1, s);
        double a0 = a.a[0], a1 = a.a[1], a2 = a0 + a1;
        double off = 0.0;
#pragma unroll
        for (int j = 2; j < 8; ++j) off += (double)a.a[j] * (double)a.a[j];
        k.add(a0 * a0 + a1 * a1 + a2 * a2 + 2.0 * off);
    }
    double r = block_sum(k.s - k.c, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = r;
}

// ---------------------------------------------------------------- MetaD force chain
// R_{mu nu}(x) = C_{mu nu}(x) - C_{mu nu}(x)^dag for the six planes (observables/clover.hpp:94-152,
// :256-262)
template <typename T, int NR>
__global__ void __launch_bounds__(kThreads) k_clover_R(Gauge<T, NR> U, Clov<T> R, Geom g)
{
    pdl_release();
    pdl_wait();
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 6 * g.V) return;
    int pl = t / g.V, x = t - pl * g.V;
    int par = x >= g.vh, s = x - par * g.vh;
    int c[4];
    int i = site_coords(g, par, s, c);
    // planes 01 02 03 12 13 23
    const int pm = pl < 3 ? 0 : pl < 5 ? 1 : 2, pn = pl < 3 ? pl + 1 : pl < 5 ? pl - 1 : 3;
    M3<T> cl = clover_leaves(U, g, par, i, c, pm, pn);
    R.st(pl, par, s, cl - adj(cl));
}

// TopChargeClover(const FullTensor&) (observables/topological_charge.hpp:202-231) from the
// stored clover planes R = C - C^dag: per site ReTr(R01 R23 - R02 R13 + R03 R12), products
// in FP64; the force of the metadynamics chain builds R anyway (CalculateClover,
// hmc_metadynamics.hpp:397-399), so its charge costs one pass over R
template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_topcharge_R(Clov<T> R, Geom g, double* __restrict__ partials)
{
    __shared__ double sh[32];
    Kahan k;
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < g.V; x += gridDim.x * blockDim.x)
    {
        const int par = x >= g.vh, s = x - par * g.vh;
        double q = retr_mul(cvt<double>(R.ld(0, 1, par, s)), cvt<double>(R.ld(2, 3, par, s)));
        q -= retr_mul(cvt<double>(R.ld(0, 2, par, s)), cvt<double>(R.ld(1, 3, par, s)));
        q += retr_mul(cvt<double>(R.ld(0, 3, par, s)), cvt<double>(R.ld(1, 2, par, s)));
        k.add(q);
    }
    double r = block_sum(k.s - k.c, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = r;
}

// CloverDerivativeComponent (observables/clover.hpp:238-276)
template <typename T, int NR>
LT_D M3<T> clover_deriv_component(const Gauge<T, NR>& U, const Clov<T>& R, const Geom& g, int par, int i,
                                  const int c[4], int mu, int nu, int rho, int sigma)
{
    const int op = par ^ 1;
    const int dmu = step_up_rt(g, mu, c);
    const int imu = i + dmu, inu = i + step_up_rt(g, nu, c), ind = i + step_dn_rt(g, nu, c);
    // x+mu+nu and x+mu-nu share the nu offsets of x (coordinate c[nu] unchanged by the mu step)
    const int imunu = inu + dmu, imund = ind + dmu;
    // Every term is linear in the planes R: with R = i H (H = -i R Hermitian, real diagonal) the
    // sum is computed with H through the Hermitian-aware products and multiplied by i at the end
    M3<T> r;
    {
        const M3<T> u_s_nu = U.ld(nu, par, i >> 1);
        const M3<T> u_mup_nu = U.ld(nu, op, imu >> 1);
        const M3<T> u_nup_mu = U.ld(mu, op, inu >> 1);
        const M3<T> H_s = R.ld_h(rho, sigma, par, i >> 1);
        M3<T> tmp1 = mul_nd(u_mup_nu, u_nup_mu);          // U(x+mu,nu) U(x+nu,mu)^dag
        r = mul(tmp1, mul_dh(u_s_nu, H_s) + mul_hd(R.ld_h(rho, sigma, op, inu >> 1), u_s_nu));
        asm volatile("" ::: "memory");
        M3<T> tmp2 = mul_dd(u_nup_mu, u_s_nu);            // U(x+nu,mu)^dag U(x,nu)^dag
        acc(r, mul(mul_xh(u_mup_nu, R.ld_h(rho, sigma, par, imunu >> 1)) + mul_hx(R.ld_h(rho, sigma, op, imu >> 1), u_mup_nu), tmp2));
    }
    asm volatile("" ::: "memory");
    {
        const M3<T> u_mupnud_nu = U.ld(nu, par, imund >> 1);
        const M3<T> u_nud_mu = U.ld(mu, op, ind >> 1);
        const M3<T> u_nud_nu = U.ld(nu, op, ind >> 1);
        M3<T> tmp3 = mul_dd(u_mupnud_nu, u_nud_mu);       // U(x+mu-nu,nu)^dag U(x-nu,mu)^dag
        r = r - mul(tmp3, mul_xh(u_nud_nu, R.ld_h(rho, sigma, par, i >> 1)) + mul_hx(R.ld_h(rho, sigma, op, ind >> 1), u_nud_nu));
        asm volatile("" ::: "memory");
        M3<T> tmp4 = mul_dn(u_nud_mu, u_nud_nu);          // U(x-nu,mu)^dag U(x-nu,nu)
        r = r - mul(mul_dh(u_mupnud_nu, R.ld_h(rho, sigma, par, imund >> 1)) + mul_hd(R.ld_h(rho, sigma, op, imu >> 1), u_mupnud_nu), tmp4);
    }
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) r.e[a][b] = timesi(r.e[a][b]);
    return r;
}

// CloverDerivative (observables/clover.hpp:279-321) times `scale` (dV/dQ):
// Sigma_n = scale * (-2/(512 pi^2)) Algebra(U_mu(x) sum_eps-terms)
// The component is computed in two halves separated by compiler memory fences, so that the
// loads of the second half are not hoisted into the first: FP32 links then fit 3 blocks of
// 128 per SM (168 registers, no spills; 201 registers unfenced without a cap, 253 before)
template <typename T> struct CloverDerivMinBlocks
{
    static constexpr int value = sizeof(T) == 4 ? 3 : 1;
};
template <typename T, int NR>
__global__ void __launch_bounds__(kThreads, CloverDerivMinBlocks<T>::value) k_clover_deriv(Gauge<T, NR> U, Clov<T> R, Alg<T> out, Geom g, T scale)
{
    pdl_release();
    pdl_wait();
    int mu, x;
    if (!link_of_thread(g, mu, x)) return;
    int par = x >= g.vh, s = x - par * g.vh;
    int c[4];
    int i = site_coords(g, par, s, c);
    // the three epsilon-tensor terms of direction mu: nu = the k-th other direction, (rho,
    // sigma) the remaining two in ascending order, sign = parity of (mu, nu, rho, sigma)
    const int o0 = mu == 0 ? 1 : 0, o1 = mu <= 1 ? 2 : 1, o2 = mu <= 2 ? 3 : 2;
    M3<T> d = zero3<T>();
#pragma unroll 1
    for (int k = 0; k < 3; ++k)
    {
        const int nu = k == 0 ? o0 : k == 1 ? o1 : o2, rho = k == 0 ? o1 : o0, sigma = k == 2 ? o1 : o2;
        const int inv = (mu > nu) + (mu > rho) + (mu > sigma) + (nu > rho) + (nu > sigma) + (rho > sigma);
        M3<T> comp = clover_deriv_component(U, R, g, par, i, c, mu, nu, rho, sigma);
        d = (inv & 1) ? d - comp : d + comp;
    }
    d = mul(U.ld(mu, par, s), d);
    A8<T> a = algebra8(d);
    const T pref = (T)(-2.0 / (512.0 * kPi * kPi)) * scale;
#pragma unroll
    for (int k = 0; k < 8; ++k) a.a[k] *= pref;
    out.st(mu, par, s, a);
}

// First half of StoutForceRecursion (smearing/stout_smearing.hpp:152-175) with CalculateLambda
// (:122-150): for level k-1 field U and level k field Up, Sigma' = Up^dag Sigma,
// Lambda = TracelessHermitian(tr(B1 U Sigma') Q + tr(B2 U Sigma') Q^2 + f1 U Sigma' + f2 (Q U Sigma' + U Sigma' Q)),
// with Q = -i rho Algebra(st U^dag); the exponential constants are recomputed from U here
// rather than stored during the forward smearing.  Also writes the link-local part of the
// recursion, Tloc = Sigma' exp(iQ) + i rho st^dag Lambda.
// Lambda kernel on FP32 links: 3 blocks of 128 per SM (168 registers, a few spilled) measured
// 1.5 % faster for the whole force than 2 blocks without spills; FP64 keeps no cap (a cap of
// 3 spills 2 KB per thread)
#ifndef LT_MINB_LAMBDA_F32
#define LT_MINB_LAMBDA_F32 3
#endif
template <typename T> struct LambdaMinBlocks
{
    static constexpr int value = sizeof(T) == 4 ? LT_MINB_LAMBDA_F32 : 1;
};
// First half of StoutForceRecursion for the link (mu, x) given its level-(k-1) link u and
// staple st: Lambda (written) and the link-local term Tloc (written)
template <typename T, int NR>
LT_D void stout_lambda_core(const Gauge<T, NR>& Up, const Alg<T>& Sigma, const Alg<T>& Lam, const Full<T>& Tloc,
                            T rho, int mu, int par, int s, const M3<T>& u, const M3<T>& st)
{
    M3<T> sp = mul_dn(Up.ld(mu, par, s), unpack_ah(Sigma.ld(mu, par, s)));
    // Q = -i rho C with C = Algebra(st U^dag), packed as a Hermitian matrix (real diagonal):
    // for C = unpack_ah(c), Q = unpack_h(rho (c0, c1, c3, -c2, c5, -c4, c7, -c6))
    const A8<T> c8 = algebra8(mul_nd(st, u));
    A8<T> q8;
    q8.a[0] = rho * c8.a[0];
    q8.a[1] = rho * c8.a[1];
    q8.a[2] = rho * c8.a[3];
    q8.a[3] = -rho * c8.a[2];
    q8.a[4] = rho * c8.a[5];
    q8.a[5] = -rho * c8.a[4];
    q8.a[6] = rho * c8.a[7];
    q8.a[7] = -rho * c8.a[6];
    const M3<T> Q = unpack_h(q8);
    M3<T> Q2 = herm_sq(Q);
    M3<T> tmp = mul(u, sp);
    M3<T> Qt = mul_hx(Q, tmp), tQ = mul_xh(tmp, Q);
    // tr(B_j tmp) = b_j0 tr(tmp) + b_j1 tr(Q tmp) + b_j2 tr(Q^2 tmp)
    const cx<T> r0 = trace(tmp), r1 = trace(Qt), r2 = tr_mul(Q2, tmp);
    cx<T> t1, t2, f1, f2;
    M3<T> ex;
    const T c1 = (T)0.5 * (Q2.e[0][0].r + Q2.e[1][1].r + Q2.e[2][2].r);
    if (sizeof(T) == 4 && c1 <= (T)0.5)
    {
        // FP32 links, small arguments (every stout step of the chain): the Cayley-Hamilton
        // series and its derivatives in FP32 (11 or 17 terms), no transcendental scalar chain.  FP64
        // keeps the closed form: its 23-term series costs more registers than it saves.
        const T c0 = retr_mul(Q, Q2) * (T)(1.0 / 3.0);
        cx<T> f[3], b2[3], b1[3];
        // spectral radius r <= sqrt(2 c1): at r <= 1/2 the tails after 11 terms are below
        // 1e-11 for f and 6e-9 for its derivatives
        if (c1 <= (T)0.125)
            exp_series_deriv<10>(c0, c1, f, b2, b1);
        else
            exp_series_deriv<16>(c0, c1, f, b2, b1);
        t1 = b1[0] * r0 + b1[1] * r1 + b1[2] * r2;
        t2 = b2[0] * r0 + b2[1] * r1 + b2[2] * r2;
        f1 = f[1];
        f2 = f[2];
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) ex.e[a][b] = lincomb2(f[1], Q.e[a][b], f[2], Q2.e[a][b]);
        ex.e[0][0] = ex.e[0][0] + f[0];
        ex.e[1][1] = ex.e[1][1] + f[0];
        ex.e[2][2] = ex.e[2][2] + f[0];
    }
    else
    {
        ExpScalars e = exp_scalars(Q, Q2);
        ExpDerivScalars d = exp_deriv_scalars(e);
        const cx<double> tr0 = cvt<double>(r0), tr1 = cvt<double>(r1), tr2 = cvt<double>(r2);
        t1 = cvt<T>(d.b10 * tr0 + d.b11 * tr1 + d.b12 * tr2);
        t2 = cvt<T>(d.b20 * tr0 + d.b21 * tr1 + d.b22 * tr2);
        f1 = cvt<T>(d.f1);
        f2 = cvt<T>(d.f2);
        ex = exp_from(e, Q, Q2);
    }
    M3<T> lam;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b)
            lam.e[a][b] = t1 * Q.e[a][b] + t2 * Q2.e[a][b] + f1 * tmp.e[a][b] + f2 * (Qt.e[a][b] + tQ.e[a][b]);
    A8<T> l8 = traceless_herm8(lam);
    Lam.st(mu, par, s, l8);
    M3<T> loc = mul(sp, ex);
    M3<T> sl = mul_dh(st, unpack_h(l8));   // st^dag Lambda
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) loc.e[a][b] = loc.e[a][b] + rho * timesi(sl.e[a][b]);
    Tloc.st(mu, par, s, loc);
}

template <typename T, int NR>
__global__ void __launch_bounds__(kThreads, LambdaMinBlocks<T>::value) k_stout_lambda(Gauge<T, NR> U, Gauge<T, NR> Up, Alg<T> Sigma, Alg<T> Lam,
                                                           Full<T> Tloc, Geom g, T rho)
{
    pdl_release();
    pdl_wait();
    int mu, x;
    if (!link_of_thread(g, mu, x)) return;
    int par = x >= g.vh, s = x - par * g.vh;
    int c[4];
    int i = site_coords(g, par, s, c);
    stout_lambda_core(Up, Sigma, Lam, Tloc, rho, mu, par, s, U.ld(mu, par, s), staple(U, g, par, i, c, mu));
}

// k_stout_lambda with the staple stored by the forward stout step of the level (St)
template <typename T, int NR>
__global__ void __launch_bounds__(kThreads, LambdaMinBlocks<T>::value) k_stout_lambda_st(Gauge<T, NR> U, Gauge<T, NR> Up, Alg<T> Sigma, Alg<T> Lam,
                                                              Full<T> Tloc, Full<T> St, Geom g, T rho)
{
    pdl_release();
    pdl_wait();
    int mu, x;
    if (!link_of_thread(g, mu, x)) return;
    const int par = x >= g.vh, s = x - par * g.vh;
    stout_lambda_core(Up, Sigma, Lam, Tloc, rho, mu, par, s, U.ld(mu, par, s), St.ld(mu, par, s));
}

// k_stout_lambda on two-row FP32 storage with the staged staple
template <int Unused = 0>
__global__ void __launch_bounds__(4 * kSitesPerBlock, LT_MINB_LAMBDA_F32)
    k_stout_lambda_staged(Gauge<float, 2> U, Gauge<float, 2> Up, Alg<float> Sigma, Alg<float> Lam, Full<float> Tloc,
                          Geom g, float rho)
{
    __shared__ StapleRing ring;
    pdl_release();
    pdl_wait();
    int mu, x;
    if (!link_of_thread(g, mu, x)) return;
    const int par = x >= g.vh, s = x - par * g.vh;
    int c[4];
    const int i = site_coords(g, par, s, c);
    M3<float> u;
    const M3<float> st = staple_staged<true>(ring, U, g, par, i, s, c, mu, u);
    stout_lambda_core(Up, Sigma, Lam, Tloc, rho, mu, par, s, u, st);
}

// Second half of StoutForceRecursion (smearing/stout_smearing.hpp:177-230):
// Sigma_{k-1} = Algebra(U (Tloc - i rho sum_{nu != mu} [six-term neighbour sum of U and Lambda]))
template <typename T, int NR>
__global__ void __launch_bounds__(kThreads) k_stout_recursion(Gauge<T, NR> U, Alg<T> Lam, Full<T> Tloc, Alg<T> Sigma,
                                                              Geom g, T rho)
{
    pdl_release();
    pdl_wait();
    int mu, x;
    if (!link_of_thread(g, mu, x)) return;
    int par = x >= g.vh, s = x - par * g.vh;
    int c[4];
    int i = site_coords(g, par, s, c);
    const int op = par ^ 1;
    const int dmu = step_up_rt(g, mu, c);
    const int imu = i + dmu;
    M3<T> fs = zero3<T>();
#pragma unroll 1
    for (int nu = 0; nu < 4; ++nu)
    {
        if (nu == mu) continue;
        const int inu = i + step_up_rt(g, nu, c), ind = i + step_dn_rt(g, nu, c);
        const int imund = ind + dmu;
        const M3<T> u_s_nu = U.ld(nu, par, i >> 1);
        const M3<T> u_nud_mu = U.ld(mu, op, ind >> 1);
        const M3<T> u_mupnud_nu = U.ld(nu, par, imund >> 1);
        M3<T> tmp1 = mul_nd(U.ld(nu, op, imu >> 1), U.ld(mu, op, inu >> 1));
        M3<T> tmp2 = mul_dh(u_nud_mu, unpack_h(Lam.ld(mu, op, ind >> 1)) - unpack_h(Lam.ld(nu, op, ind >> 1)));
        // rows 1 and 6 of eq. C6 in arXiv:2307.04742
        acc(fs, mul(tmp1, mul_dh(u_s_nu, unpack_h(Lam.ld(nu, par, i >> 1)))
                          + mul_hd(unpack_h(Lam.ld(mu, op, inu >> 1)), u_s_nu)));
        // rows 2, 3 and 4
        acc(fs, mul(mul_dn(u_mupnud_nu, tmp2 + mul_hd(unpack_h(Lam.ld(nu, par, imund >> 1)), u_nud_mu)),
                    U.ld(nu, op, ind >> 1)));
        // row 5
        fs = fs - mul_nd(mul_hx(unpack_h(Lam.ld(nu, op, imu >> 1)), tmp1), u_s_nu);
    }
    M3<T> loc = Tloc.ld(mu, par, s);
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) loc.e[a][b] = loc.e[a][b] - rho * timesi(fs.e[a][b]);
    Sigma.st(mu, par, s, algebra8(mul(U.ld(mu, par, s), loc)));
}

} // namespace lt
