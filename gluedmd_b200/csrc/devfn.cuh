// Device helpers: position fetch through the user -> GPU-slot map, minimum image,
// deterministic block reductions.
#pragma once

#include "dev.hpp"

namespace glued {

struct F3 { float x, y, z; };

__device__ __forceinline__ F3 f3(float x, float y, float z) { F3 r; r.x = x; r.y = y; r.z = z; return r; }
__device__ __forceinline__ F3 sub3(F3 a, F3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float dot3(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ F3 cross3(F3 a, F3 b) {
    return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

__device__ __forceinline__ F3 loadPos(const float4* __restrict__ posq, const int* __restrict__ u2g, int userAtom) {
    float4 p = __ldg(posq + __ldg(u2g + userAtom));
    return f3(p.x, p.y, p.z);
}

// Minimum image, z -> y -> x (CommonGluedKernels.cpp:74-90). floor(t + 0.5)
// matches the reference's rounding of exact halves.
__device__ __forceinline__ F3 minImage(F3 d, const BoxDev& b) {
    if (b.kind == 0) return d;
    if (b.kind == 1) {
        d.z -= floorf(d.z * b.inv[2] + 0.5f) * b.c[2];
        d.y -= floorf(d.y * b.inv[1] + 0.5f) * b.b[1];
        d.x -= floorf(d.x * b.inv[0] + 0.5f) * b.a[0];
        return d;
    }
    float s3 = floorf(d.z * b.inv[2] + 0.5f);
    d.x -= s3 * b.c[0]; d.y -= s3 * b.c[1]; d.z -= s3 * b.c[2];
    float s2 = floorf(d.y * b.inv[1] + 0.5f);
    d.x -= s2 * b.b[0]; d.y -= s2 * b.b[1];
    float s1 = floorf(d.x * b.inv[0] + 0.5f);
    d.x -= s1 * b.a[0];
    return d;
}

__device__ __forceinline__ double warpSum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ float warpSumF(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sum of NV doubles over the block, fixed reduction tree (deterministic).
// Result valid in every thread. scratch: >= 32 * NV doubles of shared memory.
template <int NV>
__device__ __forceinline__ void blockSum(double (&v)[NV], double* scratch) {
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int k = 0; k < NV; k++) v[k] = warpSum(v[k]);
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; k++) scratch[w * NV + k] = v[k];
    __syncthreads();
    if (w == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) {
            double t = lane < nw ? scratch[lane * NV + k] : 0.0;
            t = warpSum(t);
            if (lane == 0) scratch[k] = t;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; k++) v[k] = scratch[k];
    __syncthreads();
}

// Rational switch (1 - x^n)/(1 - x^m) for positive integer n, m evaluated as
// S_n(x)/S_m(x), S_k(x) = 1 + x + ... + x^(k-1), with derivative
// (S_n' S_m - S_n S_m') / S_m^2. Equal to the quotient for x != 1 and to its
// limit n/m at x = 1, without cancellation anywhere on x >= 0.
__device__ __forceinline__ void ratioSwitch(float x, int n, int m, float& f, float& dfdx) {
    float sn = 0.0f, dsn = 0.0f, sm = 0.0f, dsm = 0.0f;
    for (int j = n - 1; j >= 0; j--) { dsn = dsn * x + sn; sn = sn * x + 1.0f; }
    for (int j = m - 1; j >= 0; j--) { dsm = dsm * x + sm; sm = sm * x + 1.0f; }
    float ism = 1.0f / sm;
    f = sn * ism;
    dfdx = (dsn * sm - sn * dsm) * ism * ism;
}

}  // namespace glued
