// qem_diag.cu -- measured throughput peaks used as roofline denominators.
//
// The QEM kernels are bound by the FP32 FMA pipe and the MUFU (SFU) pipe, not
// by HBM or tensor cores, so their roofline needs the device's own FP32 FMA
// and MUFU rates: these kernels measure them with CUDA events (dependent-free
// chains of 8 independent accumulators per thread, enough warps to fill every
// SM); the FP32 rate is the larger of scalar and packed FP32x2 FMA chains.
#include <algorithm>

#include "qem_internal.cuh"

namespace {

__global__ void k_fma_peak(int iters, float seed, float *out)
{
    float a0 = seed + threadIdx.x, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3, a4 = a0 + 4, a5 = a0 + 5, a6 = a0 + 6,
          a7 = a0 + 7;
    const float m = 0.9999999f, c = 1e-7f;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int u = 0; u < 16; u++) {
            a0 = fmaf(a0, m, c); a1 = fmaf(a1, m, c); a2 = fmaf(a2, m, c); a3 = fmaf(a3, m, c);
            a4 = fmaf(a4, m, c); a5 = fmaf(a5, m, c); a6 = fmaf(a6, m, c); a7 = fmaf(a7, m, c);
        }
    }
    const float s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
    if (s == 1234.5f) out[0] = s;  // keeps the chain alive
}

// the same chains as packed FP32x2 instructions (sm_100: one instruction
// issues two FMAs), so that the FP32 denominator also covers kernels that use them
__global__ void k_fma2_peak(int iters, float seed, float *out)
{
    float2 a[8];
#pragma unroll
    for (int j = 0; j < 8; j++) a[j] = make_float2(seed + threadIdx.x + j, seed + threadIdx.x + j + 0.5f);
    const float2 m = make_float2(0.9999999f, 0.9999999f), c = make_float2(1e-7f, 1e-7f);
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int u = 0; u < 8; u++) {
#pragma unroll
            for (int j = 0; j < 8; j++) a[j] = __ffma2_rn(a[j], m, c);
        }
    }
    float s = 0;
#pragma unroll
    for (int j = 0; j < 8; j++) s += a[j].x + a[j].y;
    if (s == 1234.5f) out[0] = s;
}

__global__ void k_mufu_peak(int iters, float seed, float *out)
{
    float a0 = seed * threadIdx.x * 1e-6f, a1 = a0 + 0.1f, a2 = a0 + 0.2f, a3 = a0 + 0.3f;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int u = 0; u < 16; u++) {
            asm volatile("ex2.approx.ftz.f32 %0, %0;" : "+f"(a0));
            asm volatile("ex2.approx.ftz.f32 %0, %0;" : "+f"(a1));
            asm volatile("ex2.approx.ftz.f32 %0, %0;" : "+f"(a2));
            asm volatile("ex2.approx.ftz.f32 %0, %0;" : "+f"(a3));
        }
    }
    const float s = a0 + a1 + a2 + a3;
    if (s == 1234.5f) out[0] = s;
}

// FP64 FMA chains (the roofline denominator of the FP64 path and the adjoint)
__global__ void k_dfma_peak(int iters, double seed, double *out)
{
    double a0 = seed + threadIdx.x, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3, a4 = a0 + 4, a5 = a0 + 5, a6 = a0 + 6,
           a7 = a0 + 7;
    const double m = 0.9999999999, c = 1e-10;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int u = 0; u < 16; u++) {
            a0 = fma(a0, m, c); a1 = fma(a1, m, c); a2 = fma(a2, m, c); a3 = fma(a3, m, c);
            a4 = fma(a4, m, c); a5 = fma(a5, m, c); a6 = fma(a6, m, c); a7 = fma(a7, m, c);
        }
    }
    const double s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
    if (s == 1234.5) out[0] = s;
}

}  // namespace

extern "C" qem_status qem_measure_fp64_peak(int32_t device, double *fp64_tflops)
{
    if (!fp64_tflops) return QEM_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return QEM_ERR_CUDA;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return QEM_ERR_CUDA;
    double *d = nullptr;
    if (cudaMalloc(&d, 64) != cudaSuccess) return QEM_ERR_CUDA;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    const int blocks = prop.multiProcessorCount * 8, threads = 256, iters = 1024;
    float best = 1e30f;
    for (int rep = 0; rep < 4; rep++) {
        float t = 0;
        cudaEventRecord(a);
        k_dfma_peak<<<blocks, threads>>>(iters, 1.0, d);
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        cudaEventElapsedTime(&t, a, b);
        if (rep > 0) best = std::min(best, t);
    }
    const cudaError_t e = cudaGetLastError();
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(d);
    if (e != cudaSuccess) return QEM_ERR_CUDA;
    *fp64_tflops = 2.0 * (double)blocks * threads * iters * 16 * 8 / (best * 1e-3) * 1e-12;
    return QEM_OK;
}

extern "C" qem_status qem_measure_peaks(int32_t device, double *fp32_tflops, double *mufu_tops)
{
    if (cudaSetDevice(device) != cudaSuccess) return QEM_ERR_CUDA;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return QEM_ERR_CUDA;
    float *d = nullptr;
    if (cudaMalloc(&d, 64) != cudaSuccess) return QEM_ERR_CUDA;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    const int blocks = prop.multiProcessorCount * 8, threads = 256;
    const int it_fma = 4096, it_mufu = 1024;
    float best_f = 1e30f, best_f2 = 1e30f, best_m = 1e30f;
    for (int rep = 0; rep < 4; rep++) {
        float t = 0;
        cudaEventRecord(a);
        k_fma_peak<<<blocks, threads>>>(it_fma, 1.0f, d);
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        cudaEventElapsedTime(&t, a, b);
        if (rep > 0) best_f = std::min(best_f, t);
        cudaEventRecord(a);
        k_fma2_peak<<<blocks, threads>>>(it_fma, 1.0f, d);
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        cudaEventElapsedTime(&t, a, b);
        if (rep > 0) best_f2 = std::min(best_f2, t);
        cudaEventRecord(a);
        k_mufu_peak<<<blocks, threads>>>(it_mufu, 1.0f, d);
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        cudaEventElapsedTime(&t, a, b);
        if (rep > 0) best_m = std::min(best_m, t);
    }
    cudaError_t e = cudaGetLastError();
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(d);
    if (e != cudaSuccess) return QEM_ERR_CUDA;
    const double nthr = (double)blocks * threads;
    // scalar: 16 x 8 FMAs per iteration; packed: 8 x 8 instructions of two FMAs
    const double f1 = 2.0 * nthr * it_fma * 16 * 8 / (best_f * 1e-3) * 1e-12;
    const double f2 = 2.0 * nthr * it_fma * 8 * 8 * 2 / (best_f2 * 1e-3) * 1e-12;
    if (fp32_tflops) *fp32_tflops = std::max(f1, f2);
    if (mufu_tops) *mufu_tops = nthr * it_mufu * 16 * 4 / (best_m * 1e-3) * 1e-12;
    return QEM_OK;
}
