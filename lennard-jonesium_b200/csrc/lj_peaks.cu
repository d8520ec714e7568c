// lj_peaks.cu -- FMA throughput microbenchmark for the roofline denominators.
//
// The pair kernels run on the CUDA-core FP64 and FP32 pipes (no tensor
// cores), whose peaks are not among the driver's measured peaks, so they are
// measured here: every thread runs 8 independent FMA chains, enough blocks to
// fill every SM several times over, timed with CUDA events.  flops = 2 per FMA.

#include <cuda_runtime.h>

#include "../../include/lj_gpu.h"

namespace {

constexpr int kChains = 8;

template <typename T>
__global__ void __launch_bounds__(256) fma_kernel(T* out, int iters, T a, T b) {
    T x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = (T)(threadIdx.x + c) * (T)1e-3;
    for (int it = 0; it < iters; ++it)
#pragma unroll
        for (int c = 0; c < kChains; ++c) x[c] = x[c] * a + b;
    T s = 0;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += x[c];
    if (s == (T)12345.678) out[0] = s;  // keeps the chains live
}

template <typename T>
int time_fma(int blocks, int iters, double* tflops) {
    T* out = nullptr;
    cudaEvent_t e0, e1;
    if (cudaMalloc(&out, sizeof(T)) != cudaSuccess) return LJ_ERR_CUDA;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    fma_kernel<T><<<blocks, 256>>>(out, iters / 8, (T)0.999999, (T)1e-7);  // warm-up
    cudaEventRecord(e0);
    fma_kernel<T><<<blocks, 256>>>(out, iters, (T)0.999999, (T)1e-7);
    cudaEventRecord(e1);
    cudaError_t e = cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (e != cudaSuccess || ms <= 0) return LJ_ERR_CUDA;
    *tflops = 2.0 * kChains * (double)iters * blocks * 256 / (ms * 1e-3) / 1e12;
    return LJ_OK;
}

}  // namespace

extern "C" int lj_gpu_fma_peaks(int device, double* fp64_tflops, double* fp32_tflops) {
    if (!fp64_tflops || !fp32_tflops) return LJ_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return LJ_ERR_CUDA;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    int blocks = sms * 8;
    int rc = time_fma<double>(blocks, 1 << 14, fp64_tflops);
    if (rc) return rc;
    return time_fma<float>(blocks, 1 << 15, fp32_tflops);
}
