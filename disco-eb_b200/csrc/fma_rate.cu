// FP64 FMA throughput of the current GPU: the roofline denominator of the solver kernels, whose
// arithmetic runs on the FP64 pipe (fused multiply-adds, no tensor-core form).
//
// Every thread runs kChains independent FMA chains a <- a * b + c for `iters` iterations; with
// enough resident warps the chains' latency is hidden and the pipe issues every cycle.  b and c
// are kernel arguments (nothing folds at compile time) and every chain's end value is written,
// so no FMA is dead code.  With |b| < 1 the chains converge to c / (1 - b): values stay finite.
#include <cuda_runtime.h>

#include <cstdint>

#include "discoeb.h"

namespace {

constexpr int kChains = 8;
constexpr int kThreads = 256;

__global__ void __launch_bounds__(kThreads) fma_chain_kernel(int64_t iters, double b, double c, double* out)
{
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    double a[kChains];
#pragma unroll
    for (int j = 0; j < kChains; ++j) a[j] = 1e-3 * (tid % 97) + j;
    for (int64_t i = 0; i < iters; ++i) {
#pragma unroll
        for (int j = 0; j < kChains; ++j) a[j] = fma(a[j], b, c);
    }
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < kChains; ++j) s += a[j];
    out[tid] = s;
}

}  // namespace

extern "C" {

int64_t discoeb_fma_rate_threads(void)
{
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return DISCOEB_ECUDA;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0)
        return DISCOEB_ECUDA;
    return (int64_t)sms * 4 * kThreads;
}

int32_t discoeb_fma_rate(int64_t iters, double* out, int64_t n_out, double* flops, void* stream)
{
    if (iters < 1 || !out || !flops) return DISCOEB_EINVAL;
    const int64_t threads = discoeb_fma_rate_threads();
    if (threads < 0) return (int32_t)threads;
    if (n_out < threads) return DISCOEB_EINVAL;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    fma_chain_kernel<<<(unsigned)(threads / kThreads), kThreads, 0, s>>>(iters, 0.9999999, 1e-7, out);
    *flops = 2.0 * kChains * (double)iters * (double)threads;
    return cudaGetLastError() == cudaSuccess ? DISCOEB_SUCCESS : DISCOEB_ECUDA;
}

}  // extern "C"
