// FP64 FMA throughput microbenchmark (the roofline denominator of the chemistry
// kernels, which run on the FP64 CUDA-core pipe).
#include <cuda_runtime.h>

#include "gf_internal.h"

namespace {

constexpr int kChains = 8;

__global__ void __launch_bounds__(256) dfma_kernel(int iters, double a, double b, double* sink) {
    double x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = threadIdx.x * 1e-3 + c;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < kChains; ++c) x[c] = fma(x[c], a, b);
    }
    double s = 0;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += x[c];
    if (s == 12345.678) sink[0] = s;  // keeps the chains live
}

}  // namespace

extern "C" int gf_measure_fp64_peak(double ms, double* tflops) {
    if (!tflops || !(ms > 0)) return GF_ERR_INVALID_ARGUMENT;
    const int sms = gf::device_sm_count();
    if (sms <= 0) return GF_ERR_NO_DEVICE;
    double* sink = nullptr;
    if (cudaMalloc(&sink, sizeof(double)) != cudaSuccess) return GF_ERR_CUDA;
    const int blocks = sms * 8, threads = 256;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int iters = 1 << 12;
    float t = 0;
    // warm up, then scale the iteration count to the requested duration
    for (int rep = 0; rep < 4; ++rep) {
        cudaEventRecord(e0);
        dfma_kernel<<<blocks, threads>>>(iters, 0.999999, 1e-7, sink);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(&t, e0, e1);
        if (t < ms * 0.5 && iters < (1 << 26)) iters *= 2;
    }
    float best = 1e30f;
    for (int rep = 0; rep < 3; ++rep) {
        cudaEventRecord(e0);
        dfma_kernel<<<blocks, threads>>>(iters, 0.999999, 1e-7, sink);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(&t, e0, e1);
        if (t < best) best = t;
    }
    const cudaError_t err = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    if (err != cudaSuccess) return GF_ERR_CUDA;
    const double flops = 2.0 * kChains * (double)iters * blocks * threads;
    *tflops = flops / (best * 1e-3) / 1e12;
    return GF_OK;
}
