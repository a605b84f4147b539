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

// u2g == nullptr means the identity map (walker buffers of the batched path).
__device__ __forceinline__ F3 loadPos(const float4* __restrict__ posq, const int* __restrict__ u2g, int userAtom) {
    int slot = u2g ? __ldg(u2g + userAtom) : userAtom;
    float4 p = __ldg(posq + slot);
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

// Fire-and-forget 64-bit integer add into global memory (fixed-point forces and
// gradient sums). Written as red.global so that a pointer the compiler cannot
// prove global (loaded from a struct or shared memory) does not turn into a
// returning atomic that the thread then waits for.
__device__ __forceinline__ void redAddGlobal(unsigned long long* p, unsigned long long v) {
    asm volatile("red.relaxed.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
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

// Sums each of 32 slots over the warp's lanes with a fixed butterfly (31
// shuffles for all slots instead of 5 per slot): in the round with offset o a
// lane keeps the half of its live slots selected by lane bit o and adds the
// partner's copy of that half. Returns the sum of slot `lane`; v is clobbered.
__device__ __forceinline__ float warpTransposeSum32(float (&v)[32]) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
        const bool up = (lane & o) != 0;
#pragma unroll
        for (int i = 0; i < o; i++) {
            const float send = up ? v[i] : v[i + o];
            const float keep = up ? v[i + o] : v[i];
            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, o);
        }
    }
    return v[0];
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

// Distance / angle / dihedral value and Jacobian rows (jac[k] for atom k) from the
// positions p[0..3] of its atoms, the
// reference's formulas (CommonGluedKernels.cpp:177-444). jac may be null.
__device__ __forceinline__ float simpleCVFromPos(int type, const F3* p, const BoxDev& box, F3* jac) {
    if (type == 1) {  // distance
        F3 d = minImage(sub3(p[1], p[0]), box);
        float dist = sqrtf(dot3(d, d));
        float inv = dist > 1e-10f ? 1.0f / dist : 0.0f;
        if (jac) { jac[0] = f3(-d.x * inv, -d.y * inv, -d.z * inv); jac[1] = f3(d.x * inv, d.y * inv, d.z * inv); }
        return dist;
    }
    if (type == 2) {  // angle at atoms[1]
        F3 pb = p[1];
        F3 d1 = minImage(sub3(p[0], pb), box);
        F3 d2 = minImage(sub3(p[2], pb), box);
        float r1 = sqrtf(dot3(d1, d1)), r2 = sqrtf(dot3(d2, d2));
        float i1 = r1 > 1e-10f ? 1.0f / r1 : 0.0f, i2 = r2 > 1e-10f ? 1.0f / r2 : 0.0f;
        F3 n1 = f3(d1.x * i1, d1.y * i1, d1.z * i1), n2 = f3(d2.x * i2, d2.y * i2, d2.z * i2);
        float ct = fmaxf(-1.0f, fminf(1.0f, dot3(n1, n2)));
        float th = acosf(ct);
        if (jac) {
            float st = sqrtf(1.0f - ct * ct);
            float is = st > 1e-6f ? 1.0f / st : 0.0f;
            float s1 = i1 * is, s2 = i2 * is;
            F3 jA = f3(-(n2.x - ct * n1.x) * s1, -(n2.y - ct * n1.y) * s1, -(n2.z - ct * n1.z) * s1);
            F3 jC = f3(-(n1.x - ct * n2.x) * s2, -(n1.y - ct * n2.y) * s2, -(n1.z - ct * n2.z) * s2);
            jac[0] = jA; jac[1] = f3(-(jA.x + jC.x), -(jA.y + jC.y), -(jA.z + jC.z)); jac[2] = jC;
        }
        return th;
    }
    // dihedral, Blondel-Karplus
    F3 pa = p[0], pb = p[1];
    F3 pc = p[2], pd = p[3];
    F3 b1 = minImage(sub3(pb, pa), box), b2 = minImage(sub3(pc, pb), box), b3 = minImage(sub3(pd, pc), box);
    F3 t = cross3(b1, b2), u = cross3(b2, b3);
    float d = sqrtf(dot3(b2, b2));
    float phi = atan2f(d * dot3(b1, u), dot3(t, u));
    if (jac) {
        float t2 = dot3(t, t), u2 = dot3(u, u);
        float it2 = t2 > 1e-10f ? 1.0f / t2 : 0.0f;
        float iu2 = u2 > 1e-10f ? 1.0f / u2 : 0.0f;
        float id = d > 1e-10f ? 1.0f / d : 0.0f;
        float c1 = dot3(b1, b2) * id, c2 = dot3(b3, b2) * id;
        float aT = d * it2, aU = d * iu2, bTB = (d + c1) * it2, bUB = c2 * iu2;
        F3 jA = f3(-aT * t.x, -aT * t.y, -aT * t.z);
        F3 jD = f3(aU * u.x, aU * u.y, aU * u.z);
        F3 jB = f3(bTB * t.x + bUB * u.x, bTB * t.y + bUB * u.y, bTB * t.z + bUB * u.z);
        jac[0] = jA; jac[1] = jB;
        jac[2] = f3(-(jA.x + jB.x + jD.x), -(jA.y + jB.y + jD.y), -(jA.z + jB.z + jD.z));
        jac[3] = jD;
    }
    return phi;
}

// The same from posq (atoms are user indices, mapped through u2g).
__device__ __forceinline__ float simpleCV(int type, const int* atoms, const float4* __restrict__ posq,
                                         const int* __restrict__ u2g, const BoxDev& box, F3* jac) {
    const int na = type == 1 ? 2 : type == 2 ? 3 : 4;
    F3 p[4];
    for (int k = 0; k < 4; k++) p[k] = k < na ? loadPos(posq, u2g, atoms[k]) : f3(0.f, 0.f, 0.f);
    return simpleCVFromPos(type, p, box, jac);
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
