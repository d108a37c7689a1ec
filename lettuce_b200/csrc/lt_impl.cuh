// Backend implementation for one storage format: launches the kernels of lt_kernels.cuh.
#pragma once
#include <algorithm>
#include <atomic>
#include <type_traits>

#include "lt_backend.h"
#include "lt_kernels.cuh"

namespace lt {

inline int nblocks(long long n, int threads) { return (int)((n + threads - 1) / threads); }

// Site order of the next launch on a handle: ascending and descending in turn (the handle
// counts its launches), so a launch starts where the previous one ended
inline int next_order(const Ctx& c)
{
#ifdef LT_NO_ORDER_FLIP
    return 0;
#else
    return c.order ? ((*c.order)++ & 1) : 0;
#endif
}

#ifndef LT_PDL
#define LT_PDL 1
#endif

// Launch of a kernel that follows a dependent kernel on the same stream (sweeps, flow and
// stout stages).  With LT_PDL the launch carries the programmatic stream-serialisation
// attribute, so that its blocks are scheduled while the predecessor drains and wait in
// pdl_wait() (lt_kernels.cuh) for its completion.
template <typename... KArgs, typename... Args>
inline void launch_chained(void (*k)(KArgs...), int grid, int block, cudaStream_t s, Args... args)
{
#if LT_PDL
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, k, static_cast<KArgs>(args)...);
#else
    k<<<grid, block, 0, s>>>(static_cast<KArgs>(args)...);
#endif
}

// Kernels with a shared-memory ring ask for the largest shared-memory carveout (set once per
// device and kernel), so that their residency is bounded by registers and the ring alone
template <auto K> inline void prefer_shared()
{
    static std::atomic<unsigned long long> done{0};
    int dev = 0;
    cudaGetDevice(&dev);
    const unsigned long long bit = 1ull << (dev & 63);
    if (done.load(std::memory_order_relaxed) & bit) return;
    cudaFuncSetAttribute(K, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared);
    done.fetch_or(bit);
}

template <typename T, int NR> class BackendImpl final : public Backend
{
    using G = Gauge<T, NR>;

    static G gauge(const void* p, const Geom& g) { G u; u.p = (cx<T>*)p; u.vh = g.vh; return u; }
    static Alg<T> alg(const void* p, const Geom& g) { Alg<T> a; a.p = (T*)p; a.vh = g.vh; return a; }
    static Full<T> full(const void* p, const Geom& g) { Full<T> a; a.p = (cx<T>*)p; a.vh = g.vh; return a; }
    static Clov<T> clov(const void* p, const Geom& g) { Clov<T> a; a.p = (T*)p; a.vh = g.vh; return a; }
    static Full<double> full64(const void* p, const Geom& g) { Full<double> a; a.p = (cx<double>*)p; a.vh = g.vh; return a; }

    static void finish(const Ctx& c, int slot, int nslot)
    {
        k_reduce_final<<<nslot, kRedThreads, 0, c.stream>>>(c.partials + (size_t)slot * kRedBlocks, kRedBlocks,
                                                              c.results + slot);
    }

public:
    int real_bytes() const override { return (int)sizeof(T); }
    size_t gauge_bytes(const Geom& g) const override { return (size_t)4 * g.V * 3 * NR * sizeof(cx<T>); }
    size_t alg_bytes(const Geom& g) const override { return (size_t)4 * g.V * 8 * sizeof(T); }
    size_t full_bytes(const Geom& g) const override { return (size_t)4 * g.V * 9 * sizeof(cx<T>); }
    size_t clov_bytes(const Geom& g) const override { return (size_t)6 * g.V * 9 * sizeof(T); }

    void from_aos(const Ctx& c, void* U, const double* aos) const override { from_aos_sites(c, U, aos, 0, c.g.V); }
    void from_aos_sites(const Ctx& c, void* U, const double* aos, long long i0, long long i1) const override
    {
        if (i1 <= i0) return;
        k_from_aos<T, NR><<<nblocks(4LL * (i1 - i0), 256), 256, 0, c.stream>>>(gauge(U, c.g), c.g, aos, (int)(4 * i0),
                                                                              (int)(4 * i1));
    }
    void to_aos(const Ctx& c, const void* U, double* aos) const override
    {
        k_to_aos<T, NR><<<nblocks(4LL * c.g.V, 256), 256, 0, c.stream>>>(gauge(U, c.g), c.g, aos);
    }
    void alg_from_aos(const Ctx& c, void* P, const double* aos) const override
    {
        k_alg_from_aos<T><<<nblocks(4LL * c.g.V, 256), 256, 0, c.stream>>>(alg(P, c.g), c.g, aos);
    }
    void alg_to_aos(const Ctx& c, const void* P, double* aos) const override
    {
        k_alg_to_aos<T><<<nblocks(4LL * c.g.V, 256), 256, 0, c.stream>>>(alg(P, c.g), c.g, aos);
    }
    void set_unit(const Ctx& c, void* U) const override
    {
        k_set_unit<T, NR><<<nblocks(4LL * c.g.V, 256), 256, 0, c.stream>>>(gauge(U, c.g), 4 * c.g.V);
    }
    void link_io(const Ctx& c, void* U, int site, int mu, double* m, int write) const override
    {
        k_link_io<T, NR><<<1, 32, 0, c.stream>>>(gauge(U, c.g), c.g, site, mu, m, write);
    }
    void staples_aos(const Ctx& c, const void* U, double* aos) const override
    {
        auto k = c.rect ? k_staple_aos<T, NR, true> : k_staple_aos<T, NR, false>;
        k<<<nblocks(c.g.V, kSitesPerBlock), 4 * kSitesPerBlock, 0, c.stream>>>(gauge(U, c.g), c.g, aos, (T)c.cp, (T)c.cr);
    }

    void plaquette(const Ctx& c, const void* U, int slot) const override
    {
        k_plaquette<T, NR><<<kRedBlocks, kRedThreads, 0, c.stream>>>(gauge(U, c.g), c.g,
                                                                      c.partials + (size_t)slot * kRedBlocks);
        finish(c, slot, 1);
    }
    void clover_obs(const Ctx& c, const void* U, int slot) const override
    {
        k_clover_obs<T, NR><<<kRedBlocks, kRedThreads, 0, c.stream>>>(gauge(U, c.g), c.g,
                                                                       c.partials + (size_t)slot * kRedBlocks);
        finish(c, slot, 2);
    }
    void kinetic(const Ctx& c, const void* P, int slot) const override
    {
        k_kinetic<T><<<kRedBlocks, kRedThreads, 0, c.stream>>>(alg(P, c.g), 4 * c.g.V,
                                                                c.partials + (size_t)slot * kRedBlocks);
        finish(c, slot, 1);
    }

    static constexpr bool kStaged = LT_STAGED_STAPLE && std::is_same<T, float>::value && NR == 2;

    void overrelax(const Ctx& c, void* U, int mu, int par) const override
    {
        if constexpr (kStaged)
        {
            prefer_shared<k_overrelax_staged<0>>();
            launch_chained(k_overrelax_staged<0>, nblocks(c.g.vh, kStagedThreads), kStagedThreads, c.stream, gauge(U, c.g), c.g, mu,
                           par, next_order(c));
        }
        else
            launch_chained(k_overrelax<T, NR>, nblocks(c.g.vh, kThreads), kThreads, c.stream, gauge(U, c.g), c.g, mu,
                           par, next_order(c));
    }
    void heatbath(const Ctx& c, void* U, int mu, int par, double prefactor, uint64_t counter, uint64_t seed,
                  int max_iter) const override
    {
        if constexpr (kStaged)
        {
            prefer_shared<k_heatbath_staged<0>>();
            launch_chained(k_heatbath_staged<0>, nblocks(c.g.vh, kStagedThreads), kStagedThreads, c.stream, gauge(U, c.g), c.g, mu,
                           par, (T)prefactor, counter, (uint32_t)seed, (uint32_t)(seed >> 32), max_iter, c.status,
                           next_order(c));
        }
        else
            launch_chained(k_heatbath<T, NR>, nblocks(c.g.vh, kThreads), kThreads, c.stream, gauge(U, c.g), c.g, mu,
                           par, (T)prefactor, counter, (uint32_t)seed, (uint32_t)(seed >> 32), max_iter, c.status,
                           next_order(c));
    }
    void check_links(const Ctx& c, const void* U, double tol, unsigned* maxbits) const override
    {
        k_check_links<T, NR><<<kRedBlocks, kRedThreads, 0, c.stream>>>(gauge(U, c.g), c.g, tol, c.status, maxbits);
    }
    void clover_timeslices(const Ctx& c, const void* U, double* partials, int nbx) const override
    {
        k_clover_timeslice<T, NR><<<dim3(nbx, c.g.n[0]), kRedThreads, 0, c.stream>>>(gauge(U, c.g), c.g, partials);
    }
    void loops(const Ctx& c, const void* U, int slot) const override
    {
        k_loops<T, NR><<<kRedBlocks, kRedThreads, 0, c.stream>>>(gauge(U, c.g), c.g, c.partials + (size_t)slot * kRedBlocks);
        finish(c, slot, 3);
    }
    void polyakov(const Ctx& c, const void* U, int slot) const override
    {
        k_polyakov<T, NR><<<kRedBlocks, kRedThreads, 0, c.stream>>>(gauge(U, c.g), c.g, c.partials + (size_t)slot * kRedBlocks);
        finish(c, slot, 2);
    }
    void chain_init(const Ctx& c, const void* U, void* C) const override
    {
        k_chain_init<T, NR><<<nblocks(4LL * c.g.V, 256), 256, 0, c.stream>>>(gauge(U, c.g), full64(C, c.g), c.g);
    }
    void chain_unit(const Ctx& c, void* C) const override
    {
        k_chain_unit<<<nblocks(4LL * c.g.V, 256), 256, 0, c.stream>>>(full64(C, c.g), c.g);
    }
    void chain_extend(const Ctx& c, const void* Cin, const void* U, void* Cout, int L) const override
    {
        k_chain_extend<T, NR><<<nblocks(4LL * c.g.V, 256), 256, 0, c.stream>>>(full64(Cin, c.g), gauge(U, c.g),
                                                                                full64(Cout, c.g), c.g, L);
    }
    void chain_double(const Ctx& c, const void* Cin, void* Cout, int L) const override
    {
        k_chain_double<<<nblocks(4LL * c.g.V, 256), 256, 0, c.stream>>>(full64(Cin, c.g), full64(Cout, c.g), c.g, L);
    }
    void wilson_square(const Ctx& c, const void* C, int L, int slot) const override
    {
        k_wilson_square<<<kRedBlocks, kRedThreads, 0, c.stream>>>(full64(C, c.g), c.g, L,
                                                                   c.partials + (size_t)slot * kRedBlocks);
        finish(c, slot, 1);
    }
    void bmw_pack(const Ctx& c, const void* U, int full, void* out, unsigned long long* partials) const override
    {
        auto* o = static_cast<unsigned long long*>(out);
        if (full) k_bmw_pack<T, NR, 18><<<kRedBlocks, kRedThreads, 0, c.stream>>>(gauge(U, c.g), c.g, o, partials);
        else k_bmw_pack<T, NR, 12><<<kRedBlocks, kRedThreads, 0, c.stream>>>(gauge(U, c.g), c.g, o, partials);
    }
    void bmw_unpack(const Ctx& c, void* U, int full, const void* in, unsigned long long* partials,
                    unsigned* flags) const override
    {
        auto* p = static_cast<const unsigned long long*>(in);
        if (full)
            k_bmw_unpack<T, NR, 18><<<kRedBlocks, kRedThreads, 0, c.stream>>>(gauge(U, c.g), c.g, p, partials, flags);
        else
            k_bmw_unpack<T, NR, 12><<<kRedBlocks, kRedThreads, 0, c.stream>>>(gauge(U, c.g), c.g, p, partials, flags);
    }
    bool flow_split() const override { return std::is_same<T, double>::value; }
    void flow_stage(const Ctx& c, const void* Uin, void* Uout, void* Z, double c_old, double c_new, double c_exp,
                    int read_z, int write_z, void* X) const override
    {
        if constexpr (std::is_same<T, double>::value)
        {
            if (X)
            {
                const int nb = nblocks(c.g.V, kSitesPerBlock);
                launch_chained(c.rect ? k_flow_force<T, NR, true> : k_flow_force<T, NR, false>, nb, 4 * kSitesPerBlock,
                               c.stream, gauge(Uin, c.g), alg(X, c.g), c.g, (T)c.cp, (T)c.cr, next_order(c));
                launch_chained(k_flow_update<T, NR>, nb, 4 * kSitesPerBlock, c.stream, gauge(Uin, c.g),
                               gauge(Uout, c.g), alg(Z, c.g), alg(X, c.g), c.g, (T)c_old, (T)c_new, (T)c_exp, read_z,
                               write_z, next_order(c));
                return;
            }
        }
        if constexpr (kStaged)
        {
            if (!c.rect)
            {
                prefer_shared<k_flow_stage_staged<0>>();
                launch_chained(k_flow_stage_staged<0>, nblocks(c.g.V, kSitesPerBlock), 4 * kSitesPerBlock, c.stream,
                               gauge(Uin, c.g), gauge(Uout, c.g), alg(Z, c.g), c.g, (T)c_old, (T)c_new, (T)c_exp,
                               read_z, write_z, next_order(c));
                return;
            }
        }
        launch_chained(c.rect ? k_flow_stage<T, NR, true> : k_flow_stage<T, NR, false>, nblocks(c.g.V, kSitesPerBlock),
                       4 * kSitesPerBlock, c.stream, gauge(Uin, c.g), gauge(Uout, c.g), alg(Z, c.g), c.g, (T)c_old,
                       (T)c_new, (T)c_exp, read_z, write_z, (T)c.cp, (T)c.cr, next_order(c));
    }
    void flow_zeuthen_stage(const Ctx& c, const void* Uin, void* Uout, void* Z, void* X, double c_old, double c_new,
                            double c_exp, int read_z, int write_z, double cp, double cr) const override
    {
        const int nb = nblocks(c.g.V, kSitesPerBlock);
        launch_chained(k_flow_force<T, NR, true>, nb, 4 * kSitesPerBlock, c.stream, gauge(Uin, c.g), alg(X, c.g),
                       c.g, (T)cp, (T)cr, next_order(c));
        launch_chained(k_flow_zeuthen_stage<T, NR>, nb, 4 * kSitesPerBlock, c.stream, gauge(Uin, c.g),
                       gauge(Uout, c.g), alg(Z, c.g), alg(X, c.g), c.g, (T)c_old, (T)c_new, (T)c_exp, read_z,
                       write_z, next_order(c));
    }
    void stout(const Ctx& c, const void* Uin, void* Uout, double rho, void* st_out) const override
    {
        if constexpr (kStaged)
        {
            prefer_shared<k_stout_staged<0>>();
            launch_chained(k_stout_staged<0>, nblocks(c.g.V, kSitesPerBlock), 4 * kSitesPerBlock, c.stream,
                           gauge(Uin, c.g), gauge(Uout, c.g), c.g, (T)rho, full(st_out, c.g));
            return;
        }
        launch_chained(k_stout<T, NR>, nblocks(c.g.V, kSitesPerBlock), 4 * kSitesPerBlock, c.stream, gauge(Uin, c.g),
                       gauge(Uout, c.g), c.g, (T)rho, full(st_out, c.g));
    }

    void momenta(const Ctx& c, const void* U, void* P, const void* F, double coef, double eps) const override
    {
        if constexpr (kStaged)
        {
            if (!c.rect)
            {
                prefer_shared<k_momenta_staged<0>>();
                k_momenta_staged<0><<<nblocks(c.g.V, kSitesPerBlock), 4 * kSitesPerBlock, 0, c.stream>>>(
                    gauge(U, c.g), alg(P, c.g), alg(F, c.g), c.g, (T)coef, (T)eps, F != nullptr);
                return;
            }
        }
        auto k = c.rect ? k_momenta<T, NR, true> : k_momenta<T, NR, false>;
        k<<<nblocks(c.g.V, kSitesPerBlock), 4 * kSitesPerBlock, 0, c.stream>>>(
            gauge(U, c.g), alg(P, c.g), alg(F, c.g), c.g, (T)coef, (T)eps, F != nullptr, (T)c.cp, (T)c.cr);
    }
    void fields(const Ctx& c, void* U, const void* P, double eps) const override
    {
        k_fields<T, NR><<<nblocks(4LL * c.g.V, kThreads), kThreads, 0, c.stream>>>(gauge(U, c.g), alg(P, c.g),
                                                                                   4 * c.g.V, (T)eps);
    }
    void sweep4(const Ctx& c, void* U, int op, int mu, int sub, double prefactor, uint64_t counter, uint64_t seed,
                int max_iter) const override
    {
        const int nb = nblocks(c.g.V / 4, kThreads);
        if (op == 0)
            launch_chained(c.rect ? k_heatbath4<T, NR, true> : k_heatbath4<T, NR, false>, nb, kThreads, c.stream,
                           gauge(U, c.g), c.g, mu, sub, (T)prefactor, counter, (uint32_t)seed, (uint32_t)(seed >> 32),
                           max_iter, c.status, (T)c.cp, (T)c.cr, next_order(c));
        else
            launch_chained(c.rect ? k_overrelax4<T, NR, true> : k_overrelax4<T, NR, false>, nb, kThreads, c.stream,
                           gauge(U, c.g), c.g, mu, sub, (T)c.cp, (T)c.cr, next_order(c));
    }
    void alg_axpby(const Ctx& c, void* P, const void* F, double a, double b) const override
    {
        const size_t n = (size_t)4 * c.g.V * 8;
        const int blocks = (int)std::min<size_t>((n + 255) / 256, (size_t)kRedBlocks * 4);
        k_alg_axpby<T><<<blocks, 256, 0, c.stream>>>(static_cast<T*>(P), static_cast<const T*>(F), n, (T)a, (T)b);
    }
    void parity(const Ctx& c, const void* Uin, void* Uout) const override
    {
        k_parity<T, NR><<<nblocks(4LL * c.g.V, kThreads), kThreads, 0, c.stream>>>(gauge(Uin, c.g), gauge(Uout, c.g), c.g);
    }
    void random_momenta(const Ctx& c, void* P, uint64_t counter, uint64_t seed) const override
    {
        k_random_momenta<T><<<nblocks(4LL * c.g.V, 256), 256, 0, c.stream>>>(alg(P, c.g), c.g, counter,
                                                                               (uint32_t)seed, (uint32_t)(seed >> 32));
    }

    template <int SEL>
    static void batch_launch(cudaStream_t s, const void* desc, int n_lat, int n_blocks, int op, int mu, int par,
                             const uint64_t* counter, int max_iter, int flip)
    {
        const LatDesc* d = static_cast<const LatDesc*>(desc);
        if (op == 0)
        {
            if constexpr (kStaged && kBatchBlocks[SEL] <= 128) prefer_shared<k_batch_sweep<T, NR, SEL, 0>>();
            k_batch_sweep<T, NR, SEL, 0><<<n_blocks, kBatchBlocks[SEL], 0, s>>>(d, n_lat, mu, par, counter, max_iter,
                                                                                 flip);
        }
        else
        {
            if constexpr (kStaged && kBatchBlocks[SEL] <= 128) prefer_shared<k_batch_sweep<T, NR, SEL, 1>>();
            k_batch_sweep<T, NR, SEL, 1><<<n_blocks, kBatchBlocks[SEL], 0, s>>>(d, n_lat, mu, par, counter, max_iter,
                                                                                 flip);
        }
    }

    void batch_sweep(cudaStream_t s, const void* desc, int n_lat, int n_blocks, int sel, int op, int mu, int par,
                     const uint64_t* counter, int max_iter, int flip) const override
    {
        if (sel == 0) batch_launch<0>(s, desc, n_lat, n_blocks, op, mu, par, counter, max_iter, flip);
        else if (sel == 1) batch_launch<1>(s, desc, n_lat, n_blocks, op, mu, par, counter, max_iter, flip);
        else batch_launch<2>(s, desc, n_lat, n_blocks, op, mu, par, counter, max_iter, flip);
    }

    cudaError_t batch_round(cudaStream_t s, const void* desc, int n_lat, int n_units, int blocks_per_sm, int n_hb,
                            int n_or, int reverse, uint64_t* counter, int max_iter, unsigned* bar,
                            long long polls) const override
    {
        if constexpr (kStaged) prefer_shared<k_batch_round<T, NR>>();
        int dev = 0, sms = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const LatDesc* d = static_cast<const LatDesc*>(desc);
        GridBarrier b{ bar, bar + 1, bar + 2, polls };
        unsigned* next = bar + 4;   // one unit counter per sub-sweep, zeroed before the launch
        cudaError_t e = cudaMemsetAsync(next, 0, sizeof(unsigned) * 8 * (size_t)(n_hb + n_or), s);
        if (e != cudaSuccess) return e;
        void* args[] = { (void*)&d, (void*)&n_lat, (void*)&n_units, (void*)&n_hb, (void*)&n_or, (void*)&reverse,
                         (void*)&counter, (void*)&max_iter, (void*)&b, (void*)&next };
        return cudaLaunchCooperativeKernel((const void*)k_batch_round<T, NR>, dim3(blocks_per_sm * sms), dim3(128),
                                           args, 0, s);
    }
    int batch_round_max_blocks_per_sm() const override
    {
        if constexpr (kStaged) prefer_shared<k_batch_round<T, NR>>();
        int n = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_batch_round<T, NR>, 128, 0);
        return n;
    }

    void clover_tensor(const Ctx& c, const void* U, double* tensor) const override
    {
        k_clover_tensor<T, NR><<<nblocks(6LL * c.g.V, kThreads), kThreads, 0, c.stream>>>(gauge(U, c.g), c.g, tensor);
    }
    void topcharge_tensor(const Ctx& c, const double* tensor, int slot) const override
    {
        k_topcharge_tensor<0><<<kRedBlocks, kRedThreads, 0, c.stream>>>(tensor, c.g.V,
                                                                        c.partials + (size_t)slot * kRedBlocks);
        finish(c, slot, 1);
    }
    void clover_R(const Ctx& c, const void* U, void* R) const override
    {
        launch_chained(k_clover_R<T, NR>, nblocks(6LL * c.g.V, kThreads), kThreads, c.stream, gauge(U, c.g),
                       clov(R, c.g), c.g);
    }
    void topcharge_R(const Ctx& c, const void* R, int slot) const override
    {
        k_topcharge_R<T><<<kRedBlocks, kRedThreads, 0, c.stream>>>(clov(R, c.g), c.g, c.partials + (size_t)slot * kRedBlocks);
        finish(c, slot, 1);
    }
    void clover_deriv(const Ctx& c, const void* U, const void* R, void* out, double scale) const override
    {
        launch_chained(k_clover_deriv<T, NR>, nblocks(c.g.V, kSitesPerBlock), 4 * kSitesPerBlock, c.stream,
                       gauge(U, c.g), clov(R, c.g), alg(out, c.g), c.g, (T)scale);
    }
    void stout_lambda(const Ctx& c, const void* U, const void* Up, const void* Sigma, void* Lam, void* Tloc,
                      double rho, const void* st_in) const override
    {
        if (st_in)
        {
            launch_chained(k_stout_lambda_st<T, NR>, nblocks(c.g.V, kSitesPerBlock), 4 * kSitesPerBlock, c.stream,
                           gauge(U, c.g), gauge(Up, c.g), alg(Sigma, c.g), alg(Lam, c.g), full(Tloc, c.g),
                           full(st_in, c.g), c.g, (T)rho);
            return;
        }
        if constexpr (kStaged)
        {
            prefer_shared<k_stout_lambda_staged<0>>();
            launch_chained(k_stout_lambda_staged<0>, nblocks(c.g.V, kSitesPerBlock), 4 * kSitesPerBlock, c.stream,
                           gauge(U, c.g), gauge(Up, c.g), alg(Sigma, c.g), alg(Lam, c.g), full(Tloc, c.g), c.g,
                           (T)rho);
            return;
        }
        launch_chained(k_stout_lambda<T, NR>, nblocks(c.g.V, kSitesPerBlock), 4 * kSitesPerBlock, c.stream,
                       gauge(U, c.g), gauge(Up, c.g), alg(Sigma, c.g), alg(Lam, c.g), full(Tloc, c.g), c.g, (T)rho);
    }
    void stout_recursion(const Ctx& c, const void* U, const void* Lam, const void* Tloc, void* Sigma,
                         double rho) const override
    {
        launch_chained(k_stout_recursion<T, NR>, nblocks(c.g.V, kSitesPerBlock), 4 * kSitesPerBlock, c.stream,
                       gauge(U, c.g), alg(Lam, c.g), full(Tloc, c.g), alg(Sigma, c.g), c.g, (T)rho);
    }
};

} // namespace lt
