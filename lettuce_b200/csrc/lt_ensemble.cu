// Ensembles of lattices advanced together: independent Markov chains and the streams of
// parallel tempering, each lattice with its own extents and coupling, one storage format.
// A round of heatbath + overrelaxation sweeps is one launch per (mu, parity) sub-sweep over
// all lattices (k_batch_sweep), captured once as a CUDA graph and replayed; the heatbath
// counter lives in device memory so replays draw fresh random numbers.  The block size of the
// two batched kernels is chosen by timing the candidates on a scratch copy of the links
// (lt_ensemble_autotune).  Also the tempering swap of the reference's two-stream
// MetadynamicsTemperingKernel, generalised to streams with scaled biases.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <map>
#include <new>
#include <string>
#include <tuple>
#include <vector>

#include "lt_handle.h"
#include "lt_kernels.cuh"

struct lt_ensemble
{
    std::vector<lt_lattice*> lats;
    std::vector<double> betas;
    uint64_t seed = 0;
    int prec = 0;
    int device = 0;
    const lt::Backend* be = nullptr;
    cudaStream_t stream = nullptr;
    lt::LatDesc* d_desc = nullptr;
    uint64_t* d_counter = nullptr;
    int n_blocks[3] = { 0, 0, 0 };
    int sel_hb = 1, sel_or = 1;   // 64 / 128 / 256 threads per block: index 0 / 1 / 2
    std::map<std::tuple<int, int, int, int, int>, cudaGraphExec_t> graphs;
    // LT_ENSEMBLE_GRAPH: a captured graph of one batched launch per sub-sweep;
    // LT_ENSEMBLE_PERSISTENT: one cooperative launch per round with grid barriers
    int mode = LT_ENSEMBLE_GRAPH;
    int blocks_per_sm = 0;        // persistent mode: resident blocks per SM (0: the occupancy limit)
    unsigned* d_bar = nullptr;    // persistent mode: barrier count, generation, status, (pad), unit counters
    long long polls = LT_PERSIST_POLLS;
};

namespace {

int launched(const char* what)
{
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return lt::cuda_error(e, what);
    return LT_OK;
}

// Descriptors from the handles' current link pointers (a lattice's storage can move: flow
// ping-pong, lt_swap), uploaded on the ensemble stream before every use.
int refresh(lt_ensemble* e)
{
    std::vector<lt::LatDesc> d(e->lats.size());
    int begin[3] = { 0, 0, 0 };
    for (size_t k = 0; k < e->lats.size(); ++k)
    {
        const lt_lattice* h = e->lats[k];
        d[k].g = h->g;
        d[k].U = h->U;
        d[k].prefactor = 3.0 / e->betas[k];
        d[k].status = h->status;
        const uint64_t key = e->seed + (uint64_t)k;   // lattice k draws from the stream keyed seed + k
        d[k].k0 = (uint32_t)key;
        d[k].k1 = (uint32_t)(key >> 32);
        for (int s = 0; s < 3; ++s)
        {
            d[k].blk_begin[s] = begin[s];
            begin[s] += (h->g.vh + lt::kBatchBlocks[s] - 1) / lt::kBatchBlocks[s];
        }
    }
    for (int s = 0; s < 3; ++s) e->n_blocks[s] = begin[s];
    LT_CK(cudaMemcpyAsync(e->d_desc, d.data(), sizeof(lt::LatDesc) * d.size(), cudaMemcpyHostToDevice, e->stream));
    // the staging vector dies here: wait for the copy
    LT_CK(cudaStreamSynchronize(e->stream));
    return LT_OK;
}

// The ensemble stream waits for every lattice's stream, and vice versa afterwards.
int join_in(lt_ensemble* e)
{
    for (lt_lattice* h : e->lats)
    {
        cudaEvent_t ev;
        LT_CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        LT_CK(cudaEventRecord(ev, h->stream));
        LT_CK(cudaStreamWaitEvent(e->stream, ev, 0));
        LT_CK(cudaEventDestroy(ev));
    }
    return LT_OK;
}

int join_out(lt_ensemble* e)
{
    cudaEvent_t ev;
    LT_CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    LT_CK(cudaEventRecord(ev, e->stream));
    for (lt_lattice* h : e->lats) LT_CK(cudaStreamWaitEvent(h->stream, ev, 0));
    LT_CK(cudaEventDestroy(ev));
    return LT_OK;
}

// The launches of one round: n_hb heatbath sweeps then n_or overrelaxation sweeps, each in
// the reference's (mu, parity) order (iterators/iterators.hpp:65-87); reverse = the whole
// sequence backwards (with the single-sub-sweep updates being reversible, the even mixture
// of a round and its reverse is a reversible Markov step).
#ifndef LT_BATCH_FLIP
#define LT_BATCH_FLIP 1
#endif
constexpr bool kBatchFlip = LT_BATCH_FLIP;

void enqueue_round(lt_ensemble* e, cudaStream_t s, int n_hb, int n_or, int reverse, int sel_hb, int sel_or,
                   const uint64_t* counter)
{
    const int n = (int)e->lats.size();
    // consecutive launches take the work units in ascending and descending order in turn
    int launch = 0;
    auto flip = [&] { return kBatchFlip ? (launch++ & 1) : 0; };
    auto hb_sweep = [&](bool rev) {
        for (int q = 0; q < 8; ++q)
        {
            const int idx = rev ? 7 - q : q;
            e->be->batch_sweep(s, e->d_desc, n, e->n_blocks[sel_hb], sel_hb, 0, idx >> 1, idx & 1, counter, 10,
                               flip());
        }
        lt::k_counter_add<<<1, 32, 0, s>>>(const_cast<uint64_t*>(counter), 1);
    };
    auto or_sweep = [&](bool rev) {
        for (int q = 0; q < 8; ++q)
        {
            const int idx = rev ? 7 - q : q;
            e->be->batch_sweep(s, e->d_desc, n, e->n_blocks[sel_or], sel_or, 1, idx >> 1, idx & 1, counter, 10,
                               flip());
        }
    };
    if (!reverse)
    {
        for (int k = 0; k < n_hb; ++k) hb_sweep(false);
        for (int k = 0; k < n_or; ++k) or_sweep(false);
    }
    else
    {
        for (int k = 0; k < n_or; ++k) or_sweep(true);
        for (int k = 0; k < n_hb; ++k) hb_sweep(true);
    }
}

int graph_for(lt_ensemble* e, int n_hb, int n_or, int reverse, cudaGraphExec_t* out)
{
    auto key = std::make_tuple(n_hb, n_or, reverse, e->sel_hb, e->sel_or);
    auto it = e->graphs.find(key);
    if (it != e->graphs.end())
    {
        *out = it->second;
        return LT_OK;
    }
    cudaGraph_t g;
    LT_CK(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
    enqueue_round(e, e->stream, n_hb, n_or, reverse, e->sel_hb, e->sel_or, e->d_counter);
    cudaError_t ce = cudaStreamEndCapture(e->stream, &g);
    if (ce != cudaSuccess) return lt::cuda_error(ce, "lt_ensemble: graph capture");
    cudaGraphExec_t x;
    ce = cudaGraphInstantiate(&x, g, 0);
    cudaGraphDestroy(g);
    if (ce != cudaSuccess) return lt::cuda_error(ce, "lt_ensemble: graph instantiation");
    e->graphs[key] = x;
    *out = x;
    return LT_OK;
}

void drop_graphs(lt_ensemble* e)
{
    for (auto& kv : e->graphs) cudaGraphExecDestroy(kv.second);
    e->graphs.clear();
}

// persistent mode: at most this many sweeps (heatbath + overrelaxation) in one round
constexpr int kMaxRoundSweeps = 256;

int persistent_blocks(const lt_ensemble* e)
{
    const int mx = e->be->batch_round_max_blocks_per_sm();
    if (mx < 1) return 0;
    return e->blocks_per_sm > 0 ? std::min(e->blocks_per_sm, mx) : mx;
}

// n_sweep rounds as persistent launches on stream s with the given counter; the barrier words
// start at zero and are left at zero by a completed launch.  A barrier that gave up leaves
// kStatusBarrierTimeout in d_bar[2]: reported as LT_ERR_TIMEOUT after the stream drains, with
// the words reset for the next call.
int persistent_rounds(lt_ensemble* e, cudaStream_t s, int n_sweep, int n_hb, int n_or, int reverse,
                      uint64_t* counter)
{
    const int bps = persistent_blocks(e);
    if (bps < 1) return lt::set_error(LT_ERR_CUDA, "lt_ensemble: the persistent kernel cannot be resident");
    if (n_hb + n_or > kMaxRoundSweeps)
        return lt::set_error(LT_ERR_ARG, "lt_ensemble_sweeps: a persistent round holds at most 256 sweeps");
    const int n_units = e->n_blocks[1];
    for (int k = 0; k < n_sweep; ++k)
    {
        cudaError_t ce = e->be->batch_round(s, e->d_desc, (int)e->lats.size(), n_units, bps, n_hb, n_or, reverse,
                                            counter, 10, e->d_bar, e->polls);
        if (ce != cudaSuccess) return lt::cuda_error(ce, "lt_ensemble: persistent launch");
    }
    unsigned words[3];
    LT_CK(cudaMemcpyAsync(words, e->d_bar, sizeof(words), cudaMemcpyDeviceToHost, s));
    LT_CK(cudaStreamSynchronize(s));
    if (words[2] & lt::kStatusBarrierTimeout)
    {
        LT_CK(cudaMemsetAsync(e->d_bar, 0, 3 * sizeof(unsigned), s));
        LT_CK(cudaStreamSynchronize(s));
        return lt::set_error(LT_ERR_TIMEOUT, "lt_ensemble_sweeps: a grid barrier of the persistent round gave up "
                                             "waiting; the lattices are inconsistent");
    }
    return LT_OK;
}

} // namespace

extern "C" {

int lt_ensemble_create(lt_lattice* const* lattices, const double* betas, int n, uint64_t seed, lt_ensemble** out)
{
    if (!out || !lattices || !betas || n <= 0) return lt::set_error(LT_ERR_ARG, "lt_ensemble_create: bad arguments");
    *out = nullptr;
    for (int k = 0; k < n; ++k)
    {
        if (!lattices[k]) return lt::set_error(LT_ERR_ARG, "lt_ensemble_create: null lattice");
        if (lattices[k]->act_radius != 1)
            return lt::set_error(LT_ERR_ARG, "lt_ensemble_create: ensembles run the Wilson action (radius 1)");
        if (lattices[k]->prec != lattices[0]->prec)
            return lt::set_error(LT_ERR_ARG, "lt_ensemble_create: all lattices need the same storage format");
        if (!(betas[k] > 0.0)) return lt::set_error(LT_ERR_ARG, "lt_ensemble_create: beta must be positive");
        for (int j = 0; j < k; ++j)
            if (lattices[j] == lattices[k]) return lt::set_error(LT_ERR_ARG, "lt_ensemble_create: lattice listed twice");
    }
    for (int k = 1; k < n; ++k)
        if (lattices[k]->device != lattices[0]->device)
            return lt::set_error(LT_ERR_ARG, "lt_ensemble_create: all lattices must live on one device");
    const lt::DeviceScope device_scope(lattices[0]->device);
    auto* e = new (std::nothrow) lt_ensemble();
    if (!e) return lt::set_error(LT_ERR_NOMEM, "lt_ensemble_create: out of host memory");
    e->lats.assign(lattices, lattices + n);
    e->betas.assign(betas, betas + n);
    e->seed = seed;
    e->prec = lattices[0]->prec;
    e->device = lattices[0]->device;
    e->be = lattices[0]->be;
    cudaError_t ce = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking);
    if (ce == cudaSuccess) ce = cudaMalloc((void**)&e->d_desc, sizeof(lt::LatDesc) * n);
    if (ce == cudaSuccess) ce = cudaMalloc((void**)&e->d_counter, sizeof(uint64_t));
    if (ce == cudaSuccess) ce = cudaMalloc((void**)&e->d_bar, (4 + 8 * kMaxRoundSweeps) * sizeof(unsigned));
    if (ce == cudaSuccess) ce = cudaMemsetAsync(e->d_bar, 0, 4 * sizeof(unsigned), e->stream);
    if (ce != cudaSuccess)
    {
        int r = lt::cuda_error(ce, "lt_ensemble_create");
        lt_ensemble_destroy(e);
        return r;
    }
    int r = refresh(e);
    if (r != LT_OK)
    {
        lt_ensemble_destroy(e);
        return r;
    }
    *out = e;
    return LT_OK;
}

int lt_ensemble_destroy(lt_ensemble* e)
{
    if (!e) return LT_OK;
    const lt::DeviceScope device_scope(e->device);
    if (e->stream) cudaStreamSynchronize(e->stream);
    drop_graphs(e);
    if (e->d_desc) cudaFree(e->d_desc);
    if (e->d_counter) cudaFree(e->d_counter);
    if (e->d_bar) cudaFree(e->d_bar);
    if (e->stream) cudaStreamDestroy(e->stream);
    delete e;
    return LT_OK;
}

int lt_ensemble_sweeps(lt_ensemble* e, int n_sweep, int n_hb, int n_or, int reverse, uint64_t* counter)
{
    if (!e || !counter || n_sweep < 0 || n_hb < 0 || n_or < 0)
        return lt::set_error(LT_ERR_ARG, "lt_ensemble_sweeps: bad arguments");
    if (n_sweep == 0 || n_hb + n_or == 0) return LT_OK;
    const lt::DeviceScope device_scope(e->device);
    LT_TRY(join_in(e));
    LT_TRY(refresh(e));
    LT_CK(cudaMemcpyAsync(e->d_counter, counter, sizeof(uint64_t), cudaMemcpyHostToDevice, e->stream));
    if (e->mode == LT_ENSEMBLE_PERSISTENT)
    {
        const int r = persistent_rounds(e, e->stream, n_sweep, n_hb, n_or, reverse ? 1 : 0, e->d_counter);
        if (r != LT_OK)
        {
            join_out(e);
            return r;
        }
    }
    else
    {
        cudaGraphExec_t g;
        LT_TRY(graph_for(e, n_hb, n_or, reverse ? 1 : 0, &g));
        for (int k = 0; k < n_sweep; ++k) LT_CK(cudaGraphLaunch(g, e->stream));
    }
    LT_TRY(launched("lt_ensemble_sweeps"));
    LT_TRY(join_out(e));
    LT_CK(cudaStreamSynchronize(e->stream));
    *counter += (uint64_t)n_sweep * (uint64_t)n_hb;
    return LT_OK;
}

int lt_ensemble_autotune(lt_ensemble* e, int* threads_hb, int* threads_or)
{
    if (!e) return lt::set_error(LT_ERR_ARG, "lt_ensemble_autotune: null ensemble");
    const lt::DeviceScope device_scope(e->device);
    LT_TRY(join_in(e));
    LT_TRY(refresh(e));
    LT_CK(cudaStreamSynchronize(e->stream));
    // scratch copy of every lattice's links: the timing sweeps must not advance the chains
    std::vector<void*> saved(e->lats.size(), nullptr);
    int rc = LT_OK;
    for (size_t k = 0; k < e->lats.size() && rc == LT_OK; ++k)
    {
        const size_t bytes = e->be->gauge_bytes(e->lats[k]->g);
        cudaError_t ce = cudaMalloc(&saved[k], bytes);
        if (ce == cudaSuccess) ce = cudaMemcpyAsync(saved[k], e->lats[k]->U, bytes, cudaMemcpyDeviceToDevice, e->stream);
        if (ce != cudaSuccess) rc = lt::cuda_error(ce, "lt_ensemble_autotune: scratch copy");
    }
    uint64_t* d_scratch_counter = nullptr;
    if (rc == LT_OK)
    {
        cudaError_t ce = cudaMalloc((void**)&d_scratch_counter, sizeof(uint64_t));
        if (ce == cudaSuccess) ce = cudaMemsetAsync(d_scratch_counter, 0, sizeof(uint64_t), e->stream);
        if (ce != cudaSuccess) rc = lt::cuda_error(ce, "lt_ensemble_autotune: counter");
    }
    float best[2] = { 1e30f, 1e30f };
    int pick[2] = { 1, 1 };
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    if (rc == LT_OK && (cudaEventCreate(&t0) != cudaSuccess || cudaEventCreate(&t1) != cudaSuccess))
        rc = lt::set_error(LT_ERR_CUDA, "lt_ensemble_autotune: events");
    for (int op = 0; op < 2 && rc == LT_OK; ++op)
        for (int sel = 0; sel < 3 && rc == LT_OK; ++sel)
        {
            // one untimed sub-sweep, then 8 timed ones
            e->be->batch_sweep(e->stream, e->d_desc, (int)e->lats.size(), e->n_blocks[sel], sel, op, 0, 0,
                               d_scratch_counter, 10, 0);
            cudaEventRecord(t0, e->stream);
            for (int q = 0; q < 8; ++q)
                e->be->batch_sweep(e->stream, e->d_desc, (int)e->lats.size(), e->n_blocks[sel], sel, op, q >> 1,
                                   q & 1, d_scratch_counter, 10, q & 1);
            cudaEventRecord(t1, e->stream);
            cudaError_t ce = cudaEventSynchronize(t1);
            if (ce != cudaSuccess)
            {
                rc = lt::cuda_error(ce, "lt_ensemble_autotune: timing");
                break;
            }
            float ms = 0.f;
            cudaEventElapsedTime(&ms, t0, t1);
            if (ms < best[op])
            {
                best[op] = ms;
                pick[op] = sel;
            }
        }
    // the round as a whole: the graph of batched launches (blocks just chosen) against the
    // persistent cooperative round at each residency from the occupancy limit down to 1 block
    // per SM; one untimed and two timed rounds of 1 heatbath + 1 overrelaxation sweep each
    float best_round = 1e30f;
    int pick_mode = LT_ENSEMBLE_GRAPH, pick_bps = 0;
    if (rc == LT_OK)
    {
        auto time_round = [&](auto&& launch_round, float* ms_out) -> int {
            launch_round();
            cudaEventRecord(t0, e->stream);
            launch_round();
            launch_round();
            cudaEventRecord(t1, e->stream);
            cudaError_t ce = cudaEventSynchronize(t1);
            if (ce != cudaSuccess) return lt::cuda_error(ce, "lt_ensemble_autotune: round timing");
            ce = cudaGetLastError();
            if (ce != cudaSuccess) return lt::cuda_error(ce, "lt_ensemble_autotune: round launch");
            cudaEventElapsedTime(ms_out, t0, t1);
            return LT_OK;
        };
        float ms = 0.f;
        rc = time_round([&] { enqueue_round(e, e->stream, 1, 1, 0, pick[0], pick[1], d_scratch_counter); }, &ms);
        if (rc == LT_OK) best_round = ms;
        const int mx = e->be->batch_round_max_blocks_per_sm();
        for (int bps = mx; bps >= 1 && bps >= mx - 3 && rc == LT_OK; --bps)
        {
            cudaError_t le = cudaSuccess;
            rc = time_round([&] {
                if (le == cudaSuccess)
                    le = e->be->batch_round(e->stream, e->d_desc, (int)e->lats.size(), e->n_blocks[1], bps, 1, 1, 0,
                                            d_scratch_counter, 10, e->d_bar, e->polls);
            }, &ms);
            if (rc == LT_OK && le != cudaSuccess) rc = lt::cuda_error(le, "lt_ensemble_autotune: persistent launch");
            unsigned words[3] = { 0, 0, 0 };
            if (rc == LT_OK && cudaMemcpy(words, e->d_bar, sizeof(words), cudaMemcpyDeviceToHost) != cudaSuccess)
                rc = lt::set_error(LT_ERR_CUDA, "lt_ensemble_autotune: barrier words");
            if (rc == LT_OK && (words[2] & lt::kStatusBarrierTimeout))
            {
                cudaMemset(e->d_bar, 0, sizeof(words));
                rc = lt::set_error(LT_ERR_TIMEOUT, "lt_ensemble_autotune: a grid barrier gave up waiting");
            }
            if (rc == LT_OK && ms < best_round)
            {
                best_round = ms;
                pick_mode = LT_ENSEMBLE_PERSISTENT;
                pick_bps = bps;
            }
        }
    }
    // restore the links whatever happened above
    for (size_t k = 0; k < e->lats.size(); ++k)
        if (saved[k])
        {
            cudaMemcpyAsync(e->lats[k]->U, saved[k], e->be->gauge_bytes(e->lats[k]->g), cudaMemcpyDeviceToDevice,
                            e->stream);
        }
    cudaStreamSynchronize(e->stream);
    for (void* p : saved)
        if (p) cudaFree(p);
    if (d_scratch_counter) cudaFree(d_scratch_counter);
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    if (rc != LT_OK) return rc;
    if (pick[0] != e->sel_hb || pick[1] != e->sel_or) drop_graphs(e);
    e->sel_hb = pick[0];
    e->sel_or = pick[1];
    e->mode = pick_mode;
    e->blocks_per_sm = pick_bps;
    if (threads_hb) *threads_hb = lt::kBatchBlocks[pick[0]];
    if (threads_or) *threads_or = lt::kBatchBlocks[pick[1]];
    LT_TRY(join_out(e));
    return LT_OK;
}

int lt_ensemble_set_mode(lt_ensemble* e, int mode, int blocks_per_sm)
{
    if (!e) return lt::set_error(LT_ERR_ARG, "lt_ensemble_set_mode: null ensemble");
    if ((mode != LT_ENSEMBLE_GRAPH && mode != LT_ENSEMBLE_PERSISTENT) || blocks_per_sm < 0)
        return lt::set_error(LT_ERR_ARG, "lt_ensemble_set_mode: unknown mode or negative block count");
    e->mode = mode;
    e->blocks_per_sm = blocks_per_sm;
    return LT_OK;
}

int lt_ensemble_get_mode(lt_ensemble* e, int* mode, int* blocks_per_sm)
{
    if (!e || !mode || !blocks_per_sm) return lt::set_error(LT_ERR_ARG, "lt_ensemble_get_mode: null pointer");
    const lt::DeviceScope device_scope(e->device);
    *mode = e->mode;
    *blocks_per_sm = e->mode == LT_ENSEMBLE_PERSISTENT ? persistent_blocks(e) : 0;
    return LT_OK;
}

int lt_ensemble_set_barrier_polls(lt_ensemble* e, long long polls)
{
    if (!e || polls < 0) return lt::set_error(LT_ERR_ARG, "lt_ensemble_set_barrier_polls: bad arguments");
    e->polls = polls;
    return LT_OK;
}

int lt_ensemble_set_block(lt_ensemble* e, int threads_hb, int threads_or)
{
    if (!e) return lt::set_error(LT_ERR_ARG, "lt_ensemble_set_block: null ensemble");
    auto sel_of = [](int t) { return t == 64 ? 0 : t == 128 ? 1 : t == 256 ? 2 : -1; };
    const int a = sel_of(threads_hb), b = sel_of(threads_or);
    if (a < 0 || b < 0) return lt::set_error(LT_ERR_ARG, "lt_ensemble_set_block: threads must be 64, 128 or 256");
    if (a != e->sel_hb || b != e->sel_or) drop_graphs(e);
    e->sel_hb = a;
    e->sel_or = b;
    return LT_OK;
}

// Generalised MetadynamicsTemperingKernel::operator() (updates/tempering.hpp:51-72):
// streams a and b sample exp(-S - s_a V) and exp(-S - s_b V); exchanging their
// configurations (CVs q_a, q_b) changes the total weight by
//   dE = (s_a - s_b) (V(q_b) - V(q_a)),
// accepted when u <= exp(-dE) (u uniform in [0, 1)); on acceptance the link storage of the
// two handles is swapped (Swap, lattice.hpp:238-246).  With s_a = 0, s_b = 1 this is the
// reference's two-stream rule dV = V(CV_new) - V(CV_old).
int lt_tempering_swap(lt_lattice* a, lt_lattice* b, const lt_bias* bias, double scale_a, double scale_b, double q_a,
                      double q_b, double u, int* accepted, double* dE_out)
{
    if (!a || !b || !bias || !accepted) return lt::set_error(LT_ERR_ARG, "lt_tempering_swap: null argument");
    const auto* B = reinterpret_cast<const lt::Bias*>(bias);
    const double dE = (scale_a - scale_b) * (B->potential(q_b) - B->potential(q_a));
    if (dE_out) *dE_out = dE;
    *accepted = u <= std::exp(-dE) ? 1 : 0;
    if (*accepted) return lt_swap(a, b);
    return LT_OK;
}

} // extern "C"
