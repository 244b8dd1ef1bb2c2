// Measured FP32 and MUFU peaks of the current device, for the roofline of the
// system-matrix kernels (which are FP32/MUFU bound, not HBM or tensor-core bound).
//
// fp32: each thread runs 8 independent FMA chains; one FMA = 2 flops.
// mufu: each thread runs 8 independent ex2.approx chains (one MUFU op each).
// Both grids fill every SM with 8 resident blocks of 256 threads; times come from CUDA
// events around one launch after a warm-up launch.
#include <cuda_runtime.h>

#include "../../include/sysmat.h"

namespace {

constexpr int kIters = 4096;

__global__ void fma_peak(float* out, float seed)
{
    float a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = seed + (float)(threadIdx.x + k);
    const float m = 0.999999f, c = 1e-7f;
    for (int i = 0; i < kIters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) a[k] = fmaf(a[k], m, c);
    }
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += a[k];
    if (s == 12345.678f) out[threadIdx.x] = s;     // keeps the chains alive
}

__device__ __forceinline__ float ex2_approx(float x)
{
    float y;
    asm volatile("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__global__ void mufu_peak(float* out, float seed)
{
    float a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = seed * (float)(k + 1) * 1e-3f;
    for (int i = 0; i < kIters / 4; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) a[k] = ex2_approx(a[k]) * -0.5f;
    }
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += a[k];
    if (s == 12345.678f) out[threadIdx.x] = s;
}

template <typename K>
float time_kernel(K kernel, int blocks, float* out)
{
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    kernel<<<blocks, 256>>>(out, 1.0f);
    cudaEventRecord(e0);
    kernel<<<blocks, 256>>>(out, 1.0f);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return ms;
}

}  // namespace

extern "C" SYSMAT_API int sysmat_measure_peaks(double* fp32_tflops, double* mufu_tops)
{
    int dev = 0;
    cudaDeviceProp prop;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&prop, dev) != cudaSuccess)
        return SYSMAT_ERR_CUDA;
    float* out = nullptr;
    if (cudaMalloc(&out, 256 * sizeof(float)) != cudaSuccess) return SYSMAT_ERR_NOMEM;
    const int blocks = prop.multiProcessorCount * 8;
    const double threads = (double)blocks * 256.0;
    const float ms_f = time_kernel(fma_peak, blocks, out);
    const float ms_m = time_kernel(mufu_peak, blocks, out);
    cudaError_t err = cudaGetLastError();
    cudaFree(out);
    if (err != cudaSuccess || ms_f <= 0.0f || ms_m <= 0.0f) return SYSMAT_ERR_CUDA;
    if (fp32_tflops) *fp32_tflops = threads * kIters * 8.0 * 2.0 / (ms_f * 1e-3) / 1e12;
    if (mufu_tops) *mufu_tops = threads * (kIters / 4) * 8.0 / (ms_m * 1e-3) / 1e12;
    return SYSMAT_OK;
}
