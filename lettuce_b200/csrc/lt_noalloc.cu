// lt_plaquette_sum_noalloc: the plaquette sum of a caller-owned device field, computed
// without any device allocation.
//
// Who needs this: callers that may not call cudaMalloc/cudaFree themselves or have the
// library do it for them.  A framework that hands out all device memory from its own pool
// (allocator-managed tensors) forbids raw allocations, because memory taken behind the pool's
// back is invisible to its accounting and can make its own allocations fail; and a timing or
// monitoring loop cannot afford one, because cudaMalloc/cudaFree synchronise the device and
// would stall the work it measures.  Every other entry point of this library allocates its
// scratch lazily per lattice handle.
//
// The block partial sums live in the file-scope array g_partials below: kMaxBlocks
// doubles (128 KiB), resident on every GPU that loads the library until the process exits.
// Each block covers kSitesPerBlock sites, so the largest accepted lattice has
// kMaxBlocks * kSitesPerBlock = 16,777,216 sites (64^4); larger volumes are rejected
// with LT_ERR_ARG.  Every call overwrites the partials it reads (one per block, written
// before the final pass reads them), so nothing has to be cleared between calls; calls
// that overlap on the GPU (different streams, or different host threads on one device)
// race on the shared array and must be serialised by the caller.
//
// Set-up: host code cannot pass g_partials itself to a kernel (its name on the host is a
// stand-in, not a device address).  The first call on each device looks up the array's
// device address with cudaGetSymbolAddress, with that device current, and caches it; that
// first call should therefore come before any stream capture on the device.
#include <cstdio>
#include <mutex>
#include <string>

#include "lettuce_b200.h"
#include "lt_host.h"
#include "lt_kernels.cuh"

namespace {

constexpr int kNoallocThreads = 256;
constexpr int kSitesPerThread = 4;
constexpr int kSitesPerBlock = kNoallocThreads * kSitesPerThread;   // 1024
constexpr int kMaxBlocks = 16384;
constexpr int kMaxDevices = 64;

__device__ __align__(256) double g_partials[kMaxBlocks];

// Per-device address of g_partials, looked up once per device with that device current.
double* g_scratch[kMaxDevices] = {};
std::mutex g_scratch_mutex;

// One site of the plaquette sum on a field in the reference layout double[V][4][3][3][2]
// (PlaquetteSum, observables/plaquette.hpp:26-43).
__device__ __forceinline__ lt::M3<double> ld_aos(const double* __restrict__ links, int site, int mu)
{
    const double* p = links + (size_t)18 * (4 * (size_t)site + mu);
    lt::M3<double> m;
#pragma unroll
    for (int k = 0; k < 9; ++k) m.e[k / 3][k % 3] = lt::mkc(p[2 * k], p[2 * k + 1]);
    return m;
}

__global__ void __launch_bounds__(kNoallocThreads) k_plaq_aos(const double* __restrict__ links, lt::Geom g,
                                                                double* __restrict__ partials)
{
    __shared__ double sh[32];
    lt::Kahan k;
    const int base = blockIdx.x * kSitesPerBlock + threadIdx.x;
#pragma unroll 1
    for (int j = 0; j < kSitesPerThread; ++j)
    {
        const int i = base + j * kNoallocThreads;
        if (i >= g.V) break;
        int c[4];
        int r = i;
        c[3] = r % g.n[3]; r /= g.n[3];
        c[2] = r % g.n[2]; r /= g.n[2];
        c[1] = r % g.n[1]; c[0] = r / g.n[1];
        double acc = 0.0;
#pragma unroll 1
        for (int mu = 0; mu < 4; ++mu)
        {
            const int imu = i + lt::step_up(g, mu, c[mu]);
            const lt::M3<double> umu = ld_aos(links, i, mu);
#pragma unroll 1
            for (int nu = mu + 1; nu < 4; ++nu)
            {
                const int inu = i + lt::step_up(g, nu, c[nu]);
                lt::M3<double> a = lt::mul(umu, ld_aos(links, imu, nu));
                lt::M3<double> b = lt::mul(ld_aos(links, i, nu), ld_aos(links, inu, mu));
                acc += lt::retr_nd(a, b);
            }
        }
        k.add(acc);
    }
    double s = lt::block_sum(k.s - k.c, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

int scratch_for_current_device(double** out)
{
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return lt::set_error(LT_ERR_CUDA, (std::string("lt_plaquette_sum_noalloc: cudaGetDevice: ") + cudaGetErrorString(e)).c_str());
    if (dev < 0 || dev >= kMaxDevices) return lt::set_error(LT_ERR_ARG, "lt_plaquette_sum_noalloc: device index out of range");
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch[dev])
    {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_partials);
        if (e != cudaSuccess || !p)
            return lt::set_error(LT_ERR_CUDA, (std::string("lt_plaquette_sum_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e)).c_str());
        g_scratch[dev] = static_cast<double*>(p);
    }
    *out = g_scratch[dev];
    return LT_OK;
}

} // namespace

extern "C" int lt_plaquette_sum_noalloc(const double* links_dev, const int ext[4], double* out_dev, void* stream)
{
    if (!links_dev || !ext || !out_dev) return lt::set_error(LT_ERR_ARG, "lt_plaquette_sum_noalloc: null pointer");
    // the volume is checked after every factor, so no product of huge extents can wrap past the limit
    long long V = 1;
    for (int d = 0; d < 4; ++d)
    {
        if (ext[d] < 2 || ext[d] % 2)
            return lt::set_error(LT_ERR_ARG, "lt_plaquette_sum_noalloc: extents must be even and >= 2");
        V *= ext[d];
        if (V > (long long)kMaxBlocks * kSitesPerBlock)
            return lt::set_error(LT_ERR_ARG, "lt_plaquette_sum_noalloc: lattice volume exceeds the 16,777,216-site "
                                             "(64^4) limit of the static scratch");
    }
    double* scratch = nullptr;
    int r = scratch_for_current_device(&scratch);
    if (r != LT_OK) return r;
    const lt::Geom g = lt::make_geom(ext);
    const int nblk = (int)((V + kSitesPerBlock - 1) / kSitesPerBlock);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_plaq_aos<<<nblk, kNoallocThreads, 0, s>>>(links_dev, g, scratch);
    lt::k_reduce_final<<<1, lt::kRedThreads, 0, s>>>(scratch, nblk, out_dev);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return lt::set_error(LT_ERR_CUDA, (std::string("lt_plaquette_sum_noalloc: launch: ") + cudaGetErrorString(e)).c_str());
    return LT_OK;
}
