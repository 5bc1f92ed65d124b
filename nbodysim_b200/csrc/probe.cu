// FP32 FMA-pipe throughput probe (include/nbody_b200_probe.h).
#include <cuda_runtime.h>

#include "../../include/nbody_b200.h"
#include "../../include/nbody_b200_probe.h"

namespace {

constexpr int kChains = 8;
constexpr int kIters = 4096;

__global__ void __launch_bounds__(256) k_fma_probe(float *out, float a, float b) {
    float x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; c++) x[c] = (float)(threadIdx.x + c) * 1e-3f;
#pragma unroll 16
    for (int i = 0; i < kIters; i++) {
#pragma unroll
        for (int c = 0; c < kChains; c++) x[c] = fmaf(x[c], a, b);
    }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < kChains; c++) s += x[c];
    if (s == 12345.678f) out[blockIdx.x * blockDim.x + threadIdx.x] = s;  // keeps the chains live
}

}  // namespace

extern "C" int nbody_probe_fp32_peak(int device, double *tflops, double *ms) {
    if (!tflops || !ms) return NBODY_ERR_INVALID;
    if (cudaSetDevice(device) != cudaSuccess) return NBODY_ERR_NO_DEVICE;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return NBODY_ERR_CUDA;
    const int blocks = sms * 8, threads = 256;
    float *out = nullptr;
    if (cudaMalloc(&out, sizeof(float) * blocks * threads) != cudaSuccess) return NBODY_ERR_OOM;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    k_fma_probe<<<blocks, threads>>>(out, 0.9999999f, 1e-7f);  // warm-up
    float best = 1e30f;
    for (int r = 0; r < 5; r++) {
        cudaEventRecord(e0);
        k_fma_probe<<<blocks, threads>>>(out, 0.9999999f, 1e-7f);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float t = 0.f;
        cudaEventElapsedTime(&t, e0, e1);
        if (t < best) best = t;
    }
    cudaError_t err = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (err != cudaSuccess) return NBODY_ERR_CUDA;
    const double flops = 2.0 * (double)blocks * threads * kIters * kChains;
    *ms = best;
    *tflops = flops / (best * 1e-3) / 1e12;
    return NBODY_OK;
}
