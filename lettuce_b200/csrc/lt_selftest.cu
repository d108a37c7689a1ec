// Test-only entry points: the device SU(3) exponential on caller-given matrices, branch by
// branch, and the architecture the kernels were compiled for.  They exist so the tests can
// feed the exponential the edge cases of the reference's SU3::exp (generic, Taylor, sign-flip
// and zero inputs, math/su3_exp.hpp:21-52, :204-283, :419-432) directly, instead of only
// through flow, stout and HMC steps.
#include <string>

#include "lettuce_b200.h"
#include "lt_host.h"
#include "lt_math.cuh"

namespace {

// exp(iQ) of one traceless Hermitian matrix (18 doubles, row-major re/im) in arithmetic type T
// by one branch of the device exponential:
//   LT_EXP_DISPATCH  exp_ah as the flow, stout and HMC kernels call it (series below the
//                    spectral bound, closed form above it)
//   LT_EXP_CLOSED    the closed form (FP64 scalar chain, matrices in T)
//   LT_EXP_SERIES_TINY / _SHORT / _LONG  the Cayley-Hamilton series with the tiny
//                    (c1 <= 1/512), short (c1 <= 1/32) or long (c1 <= 1/2) term count of exp_ah
template <typename T>
__global__ void k_exp_test(const double* __restrict__ in, double* __restrict__ out, int n, int path)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const double* p = in + 18 * (size_t)k;
    lt::M3<T> Q;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) Q.e[i][j] = lt::mkc<T>((T)p[6 * i + 2 * j], (T)p[6 * i + 2 * j + 1]);
    lt::M3<T> r;
    if (path == LT_EXP_DISPATCH)
    {
        // exp_ah(X, c) = exp(c X) = SU3::exp(-i c X): X = i Q and c = 1 give exp(iQ)
        lt::M3<T> X;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) X.e[i][j] = lt::timesi(Q.e[i][j]);
        r = lt::exp_ah(X, (T)1);
    }
    else
    {
        const lt::M3<T> Q2 = lt::herm_sq(Q);
        if (path == LT_EXP_CLOSED)
        {
            const lt::ExpScalars e = lt::exp_scalars(Q, Q2);
            r = lt::exp_from(e, Q, Q2);
        }
        else
        {
            const T c1 = (T)0.5 * (Q2.e[0][0].r + Q2.e[1][1].r + Q2.e[2][2].r);
            const T c0 = lt::retr_mul(Q, Q2) * (T)(1.0 / 3.0);
            lt::cx<T> g0, g1, g2;
            if (path == LT_EXP_SERIES_TINY)
            {
                if (sizeof(T) == 8) lt::exp_series<9>(c0, c1, g0, g1, g2);
                else lt::exp_series<4>(c0, c1, g0, g1, g2);
            }
            else if (path == LT_EXP_SERIES_SHORT)
            {
                if (sizeof(T) == 8) lt::exp_series<12>(c0, c1, g0, g1, g2);
                else lt::exp_series<6>(c0, c1, g0, g1, g2);
            }
            else
            {
                if (sizeof(T) == 8) lt::exp_series<18>(c0, c1, g0, g1, g2);
                else lt::exp_series<11>(c0, c1, g0, g1, g2);
            }
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) r.e[i][j] = lt::lincomb2(g1, Q.e[i][j], g2, Q2.e[i][j]);
            r.e[0][0] = r.e[0][0] + g0;
            r.e[1][1] = r.e[1][1] + g0;
            r.e[2][2] = r.e[2][2] + g0;
        }
    }
    double* o = out + 18 * (size_t)k;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
        {
            o[6 * i + 2 * j] = (double)r.e[i][j].r;
            o[6 * i + 2 * j + 1] = (double)r.e[i][j].i;
        }
}

int fail(cudaError_t e, const char* what)
{
    return lt::set_error(e == cudaErrorMemoryAllocation ? LT_ERR_NOMEM : LT_ERR_CUDA,
                         (std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")").c_str());
}

} // namespace

extern "C" int lt_su3_exp_test(const double* q_in, double* out, int n, int prec, int path)
{
    if (!q_in || !out || n < 0) return lt::set_error(LT_ERR_ARG, "lt_su3_exp_test: null pointer or negative count");
    if (prec != LT_PREC_FP64 && prec != LT_PREC_FP32 && prec != LT_PREC_FP32_12)
        return lt::set_error(LT_ERR_ARG, "lt_su3_exp_test: unknown precision");
    if (path < LT_EXP_DISPATCH || path > LT_EXP_SERIES_TINY) return lt::set_error(LT_ERR_ARG, "lt_su3_exp_test: unknown path");
    if (n == 0) return LT_OK;
    if ((long long)n * 18 > (1LL << 28)) return lt::set_error(LT_ERR_ARG, "lt_su3_exp_test: too many matrices");
    const size_t bytes = sizeof(double) * 18 * (size_t)n;
    double *d_in = nullptr, *d_out = nullptr;
    cudaError_t e = cudaMalloc(&d_in, bytes);
    if (e == cudaSuccess) e = cudaMalloc(&d_out, bytes);
    if (e == cudaSuccess) e = cudaMemcpy(d_in, q_in, bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
    {
        const int threads = 128, blocks = (n + threads - 1) / threads;
        if (prec == LT_PREC_FP64) k_exp_test<double><<<blocks, threads>>>(d_in, d_out, n, path);
        else k_exp_test<float><<<blocks, threads>>>(d_in, d_out, n, path);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out, d_out, bytes, cudaMemcpyDeviceToHost);
    const cudaError_t e_free = d_in ? cudaFree(d_in) : cudaSuccess;
    if (d_out) cudaFree(d_out);
    if (e != cudaSuccess) return fail(e, "lt_su3_exp_test");
    if (e_free != cudaSuccess) return fail(e_free, "lt_su3_exp_test: cudaFree");
    return LT_OK;
}

extern "C" int lt_device_arch(int* binary_version, int* ptx_version)
{
    if (!binary_version || !ptx_version) return lt::set_error(LT_ERR_ARG, "lt_device_arch: null pointer");
    cudaFuncAttributes a;
    const cudaError_t e = cudaFuncGetAttributes(&a, k_exp_test<double>);
    if (e != cudaSuccess) return fail(e, "lt_device_arch: cudaFuncGetAttributes");
    *binary_version = a.binaryVersion;
    *ptx_version = a.ptxVersion;
    return LT_OK;
}
