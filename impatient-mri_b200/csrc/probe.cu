// Measured FP32 FMA and SFU (sin/cos) throughput of the current GPU: the
// denominators of the NUDFT roofline, which is bound by FP32 FMA and MUFU
// issue rather than by memory.
#include "../../include/impatient_b200.h"
#include <cuda_runtime.h>

namespace {

constexpr int kIters = 4096;

__global__ void __launch_bounds__(256) k_ffma(float *out, float a, float b) {
    float v[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) v[j] = threadIdx.x * 1e-3f + j;
    for (int i = 0; i < kIters; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) v[j] = fmaf(v[j], a, b);
    float s = 0.f;
#pragma unroll
    for (int j = 0; j < 8; ++j) s += v[j];
    if (s == 12345.f) out[0] = s;  // keeps the chains alive
}

__global__ void __launch_bounds__(256) k_mufu(float *out, float a) {
    float v[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) v[j] = threadIdx.x * 1e-3f + j;
    for (int i = 0; i < kIters; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) v[j] = __sinf(v[j]) + a;
    float s = 0.f;
#pragma unroll
    for (int j = 0; j < 4; ++j) s += v[j];
    if (s == 12345.f) out[0] = s;
}

}  // namespace

extern "C" imp_status imp_measure_alu_peaks(int device, double *fp32_tflops, double *sfu_gops) {
    if (!fp32_tflops || !sfu_gops) return IMP_ERR_INVALID_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return IMP_ERR_CUDA;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    float *out = nullptr;
    if (cudaMalloc(&out, sizeof(float)) != cudaSuccess) return IMP_ERR_NOMEM;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int blocks = sms * 8;
    float best_f = 1e30f, best_m = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
        float ms;
        cudaEventRecord(e0);
        k_ffma<<<blocks, 256>>>(out, 0.999f, 1e-4f);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep) best_f = ms < best_f ? ms : best_f;
        cudaEventRecord(e0);
        k_mufu<<<blocks, 256>>>(out, 0.25f);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep) best_m = ms < best_m ? ms : best_m;
    }
    const cudaError_t err = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (err != cudaSuccess) return IMP_ERR_CUDA;
    const double threads = (double)blocks * 256;
    *fp32_tflops = threads * kIters * 8 * 2.0 / (best_f * 1e-3) / 1e12;
    *sfu_gops = threads * kIters * 4 / (best_m * 1e-3) / 1e9;
    return IMP_OK;
}
