// The lattice handle behind the C ABI's opaque lt_lattice, shared by the translation units
// that implement the ABI (lt_capi.cu, lt_ensemble.cu).
#pragma once
#include <vector>

#include "lettuce_b200.h"
#include "lt_backend.h"
#include "lt_host.h"

namespace lt {
// Records a CUDA error as this thread's last error; returns LT_ERR_NOMEM or LT_ERR_CUDA.
int cuda_error(cudaError_t e, const char* what);

// Makes a handle's device current for one C-ABI call and restores the caller's device after
struct DeviceScope
{
    int prev = -1;
    explicit DeviceScope(int dev)
    {
        int cur;
        if (cudaGetDevice(&cur) == cudaSuccess && cur != dev && cudaSetDevice(dev) == cudaSuccess) prev = cur;
    }
    ~DeviceScope()
    {
        if (prev >= 0) cudaSetDevice(prev);
    }
    DeviceScope(const DeviceScope&) = delete;
    DeviceScope& operator=(const DeviceScope&) = delete;
};
} // namespace lt

#define LT_CK(call)                                                  \
    do {                                                             \
        cudaError_t e_ = (call);                                     \
        if (e_ != cudaSuccess) return lt::cuda_error(e_, #call);     \
    } while (0)

#define LT_TRY(call)                                                 \
    do {                                                             \
        int r_ = (call);                                             \
        if (r_ != LT_OK) return r_;                                  \
    } while (0)

struct lt_lattice
{
    int ext[4];
    int prec;
    int device;
    lt::Geom g;
    const lt::Backend* be;
    cudaStream_t stream = nullptr;
    void* U = nullptr;       // links
    void* U2 = nullptr;      // ping-pong partner for flow / stout
    void* Z = nullptr;       // flow Z (algebra)
    void* P = nullptr;       // HMC momenta (algebra)
    void* F = nullptr;       // metadynamics force / Sigma (algebra)
    void* Ubak = nullptr;    // HMC backup of the links
    void* R = nullptr;       // clover planes
    void* Lam = nullptr;     // Lambda (algebra)
    void* Tloc = nullptr;    // link-local recursion term (full matrix)
    std::vector<void*> levels;   // smeared levels 1..n of the MetaD chain
    std::vector<void*> staples;  // the staples of levels 0..n-1 (full 3x3 per link), for the adjoint
    double* partials = nullptr;
    double* results = nullptr;
    double* h_results = nullptr; // pinned
    void* h_stage = nullptr;     // pinned: FP32 links packed in the device layout on the host (upload)
    int uploads = 0;             // lt_upload_links calls so far (the staging is set up from the second)
    double* d_aos = nullptr;     // staging buffer for host transfers (reference layout)
    unsigned* status = nullptr;  // device status word (lt_status_word) and scratch words
    void* chainA = nullptr;      // straight-line link products of lt_wilson_loop (FP64 full matrices)
    void* chainB = nullptr;
    // the chain kept between lt_wilson_loop_chain calls (the reference's U_chain): the buffer
    // holding it and the product U(x + o mu) ... U(x + (o + n - 1) mu) it holds (n = -1: none)
    void* chain_cur = nullptr;
    int chain_origin = 0, chain_len = -1;
    bool chain_contig = true;
    // gauge action of staples, sweeps, HMC forces / Hamiltonian and flow (lt_set_gauge_action):
    // stencil radius 1 (Wilson, the default) or 2 (plaquettes and 1x2 rectangles)
    int act_radius = 1;
    double act_cp = 1.0, act_cr = 0.0;
    // force of the gradient flow run into this handle (lt_set_flow_action): the gauge action's
    // (LT_FLOW_ACTION_GAUGE, the reference's GradientFlowKernel) or the Zeuthen flow's
    int flow_action = LT_FLOW_ACTION_GAUGE;
    void* Xz = nullptr;          // Luescher-Weisz force of a Zeuthen flow stage (algebra)
    double* tensor = nullptr;    // FullTensor4D of lt_clover_tensor (FP64, reference layout)
    mutable unsigned order = 0;  // launches of the order-alternating sweep and flow kernels

    lt::Ctx ctx() const
    {
        lt::Ctx c;
        c.g = g;
        c.stream = stream;
        c.partials = partials;
        c.results = results;
        c.status = status;
        c.rect = act_radius == 2;
        c.cp = act_cp;
        c.cr = act_cr;
        c.order = &order;
        return c;
    }
};
