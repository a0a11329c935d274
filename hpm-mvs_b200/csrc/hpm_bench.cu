/*
 * FP32 peak probe: the roofline denominator for the PatchMatch kernels,
 * which are FP32-pipe work (no tensor cores).  Every thread runs 8
 * independent FMA chains so the FMA pipe, not latency, is the limit; the
 * grid is a multiple of the SM count.  Reported as TFLOP/s (2 flops per FMA).
 */
#include <cuda_runtime.h>

#include "hpm_b200.h"

namespace {

__global__ void __launch_bounds__(256) k_fma_peak(float *out, int iters, float a, float b)
{
    float x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6,
          x7 = x0 + 7;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            x0 = fmaf(x0, a, b);
            x1 = fmaf(x1, a, b);
            x2 = fmaf(x2, a, b);
            x3 = fmaf(x3, a, b);
            x4 = fmaf(x4, a, b);
            x5 = fmaf(x5, a, b);
            x6 = fmaf(x6, a, b);
            x7 = fmaf(x7, a, b);
        }
    }
    const float s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (s == 1234.5f) out[blockIdx.x * blockDim.x + threadIdx.x] = s; /* keeps the chains alive */
}

}  // namespace

extern "C" int hpm_fp32_peak(int device, float *tflops, float *sm_clock_mhz_hint)
{
    if (!tflops) return HPM_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return HPM_ERR_CUDA;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    float *out = nullptr;
    const int blocks = sms * 8, threads = 256, iters = 4096;
    if (cudaMalloc(&out, sizeof(float) * blocks * threads) != cudaSuccess) return HPM_ERR_NOMEM;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    k_fma_peak<<<blocks, threads>>>(out, 256, 0.999f, 0.001f); /* warm-up */
    cudaEventRecord(e0);
    for (int r = 0; r < 4; ++r) k_fma_peak<<<blocks, threads>>>(out, iters, 0.999f, 0.001f);
    cudaEventRecord(e1);
    cudaError_t e = cudaEventSynchronize(e1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (e != cudaSuccess || ms <= 0.0f) return HPM_ERR_CUDA;
    const double flops = 4.0 * blocks * threads * (double)iters * 16 * 8 * 2;
    *tflops = (float)(flops / (ms * 1e-3) / 1e12);
    if (sm_clock_mhz_hint) {
        int khz = 0;
        cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, device);
        *sm_clock_mhz_hint = khz / 1000.0f;
    }
    return HPM_OK;
}
