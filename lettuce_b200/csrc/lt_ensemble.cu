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
void enqueue_round(lt_ensemble* e, cudaStream_t s, int n_hb, int n_or, int reverse, int sel_hb, int sel_or,
                   const uint64_t* counter)
{
    const int n = (int)e->lats.size();
    auto hb_sweep = [&](bool rev) {
        for (int q = 0; q < 8; ++q)
        {
            const int idx = rev ? 7 - q : q;
            e->be->batch_sweep(s, e->d_desc, n, e->n_blocks[sel_hb], sel_hb, 0, idx >> 1, idx & 1, counter, 10);
        }
        lt::k_counter_add<<<1, 32, 0, s>>>(const_cast<uint64_t*>(counter), 1);
    };
    auto or_sweep = [&](bool rev) {
        for (int q = 0; q < 8; ++q)
        {
            const int idx = rev ? 7 - q : q;
            e->be->batch_sweep(s, e->d_desc, n, e->n_blocks[sel_or], sel_or, 1, idx >> 1, idx & 1, counter, 10);
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
    cudaGraphExec_t g;
    LT_TRY(graph_for(e, n_hb, n_or, reverse ? 1 : 0, &g));
    LT_CK(cudaMemcpyAsync(e->d_counter, counter, sizeof(uint64_t), cudaMemcpyHostToDevice, e->stream));
    for (int k = 0; k < n_sweep; ++k) LT_CK(cudaGraphLaunch(g, e->stream));
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
                               d_scratch_counter, 10);
            cudaEventRecord(t0, e->stream);
            for (int q = 0; q < 8; ++q)
                e->be->batch_sweep(e->stream, e->d_desc, (int)e->lats.size(), e->n_blocks[sel], sel, op, q >> 1,
                                   q & 1, d_scratch_counter, 10);
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
    if (threads_hb) *threads_hb = lt::kBatchBlocks[pick[0]];
    if (threads_or) *threads_or = lt::kBatchBlocks[pick[1]];
    LT_TRY(join_out(e));
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
