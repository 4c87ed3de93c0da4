// peak.cu — FP64 fused multiply-add throughput of the current device.
//
// The denominator of the FP64 rooflines: every thread runs eight independent
// chains of fma(a, b, c) (DFMA, two flops each) long enough that launch cost
// is noise, on a grid of four 256-thread CTAs per SM.  The chains' sum is
// written only when it equals an impossible value, which keeps the compiler
// from removing them.
#include <cuda_runtime.h>

#include "../../include/nxd.h"

namespace {

constexpr int kPeakThreads = 256;
constexpr int kPeakChains = 8;

__global__ void __launch_bounds__(kPeakThreads) k_dfma_peak(double* sink, int iters) {
    double a[kPeakChains];
#pragma unroll
    for (int k = 0; k < kPeakChains; ++k) a[k] = 1e-3 * (threadIdx.x + k);
    const double b = 0.9999999, c = 1e-9;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < kPeakChains; ++k) a[k] = fma(a[k], b, c);
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < kPeakChains; ++k) s += a[k];
    if (s == -1.0) sink[blockIdx.x] = s;
}

}  // namespace

extern "C" nxd_status nxd_fp64_peak(void* stream, double* tflops, double* ms_out) {
    if (!tflops) return NXD_INVALID_ARGUMENT;
    int dev = 0, nsm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return NXD_NO_DEVICE;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return NXD_CUDA_ERROR;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int blocks = 4 * nsm, iters = 1 << 14;
    double* sink = nullptr;
    if (cudaMalloc(&sink, sizeof(double) * blocks) != cudaSuccess) return NXD_CUDA_ERROR;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    for (int rep = 0; rep < 6; ++rep) {
        cudaEventRecord(e0, s);
        k_dfma_peak<<<blocks, kPeakThreads, 0, s>>>(sink, iters);
        cudaEventRecord(e1, s);
        cudaEventSynchronize(e1);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && ms < best) best = ms;   // the first launch warms up
    }
    const cudaError_t err = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    if (err != cudaSuccess) return NXD_CUDA_ERROR;
    const double flops = 2.0 * kPeakChains * (double)iters * blocks * kPeakThreads;
    *tflops = flops / (best * 1e-3) / 1e12;
    if (ms_out) *ms_out = best;
    return NXD_OK;
}
