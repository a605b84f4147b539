// FP32 FMA throughput probe: every thread runs 8 independent FMA chains held in
// registers (no memory traffic in the loop), one wave of 8 CTAs per SM. The
// result is written only if it is non-zero-sum so the compiler keeps the chains.
#include <cuda_runtime.h>

#include "context.hpp"
#include "kernels.hpp"

namespace glued {

__global__ void __launch_bounds__(256) k_fma_chain(float* out, int iters, float a, float b) {
    float x0 = threadIdx.x * 1e-7f, x1 = x0 + 1e-7f, x2 = x0 + 2e-7f, x3 = x0 + 3e-7f;
    float x4 = x0 + 4e-7f, x5 = x0 + 5e-7f, x6 = x0 + 6e-7f, x7 = x0 + 7e-7f;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 16; k++) {
            x0 = fmaf(x0, a, b); x1 = fmaf(x1, a, b); x2 = fmaf(x2, a, b); x3 = fmaf(x3, a, b);
            x4 = fmaf(x4, a, b); x5 = fmaf(x5, a, b); x6 = fmaf(x6, a, b); x7 = fmaf(x7, a, b);
        }
    }
    float s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (s == 1234.5f) out[0] = s;
}

double measureFp32Peak() {
    int dev = 0, sms = 0;
    cudaCheck(cudaGetDevice(&dev), "device");
    cudaCheck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "attr");
    DBuf out;
    out.alloc(16);
    const int blocks = sms * 8, threads = 256, iters = 4096;
    cudaEvent_t e0, e1;
    cudaCheck(cudaEventCreate(&e0), "event");
    cudaCheck(cudaEventCreate(&e1), "event");
    k_fma_chain<<<blocks, threads>>>(out.as<float>(), 64, 0.999999f, 1e-6f);
    double best = 0;
    for (int r = 0; r < 5; r++) {
        cudaCheck(cudaEventRecord(e0), "event");
        k_fma_chain<<<blocks, threads>>>(out.as<float>(), iters, 0.999999f, 1e-6f);
        cudaCheck(cudaEventRecord(e1), "event");
        cudaCheck(cudaEventSynchronize(e1), "event");
        float ms = 0;
        cudaCheck(cudaEventElapsedTime(&ms, e0, e1), "event");
        double flops = 2.0 * 8 * 16 * (double)iters * threads * blocks;
        double t = flops / (ms * 1e-3) / 1e12;
        if (t > best) best = t;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return best;
}

}  // namespace glued
