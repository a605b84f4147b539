// Partial-sum coordination tile used by the allocation-free entry point
// (noalloc.cu): one CTA takes TA = 8*RA A atoms against a split of group B;
// warp w holds A atoms {w, w+8, ...} in registers (all lanes share them), lane l
// walks B atoms {l, l+32, l+64, l+96} of each 128-atom chunk; A gradients are
// reduced over lanes by a fixed shuffle tree, B gradients of a chunk over the 8
// warps in fixed order, and both are written as float partials per (tile,
// split); the CN partial of each CTA is a double. The context and batched paths
// use the step runs of coord_run.cuh instead.
#pragma once

#include "devfn.cuh"

namespace glued {

namespace coordc {
constexpr int NY = 8;     // warps per CTA
constexpr int NX = 32;    // lanes
constexpr int RB = 4;     // B atoms per lane per chunk
constexpr int TB = NX * RB;  // B chunk (128 atoms)
}  // namespace coordc
using namespace coordc;

// Minimum image with the rounding done by adding and removing 1.5 * 2^23: the
// FFMA rounds d/L to the nearest integer (exact halves to even; the reference's
// floor(d/L + 0.5) differs only on exact halves, where both images are equally
// near), valid for |d/L| < 2^22. Three full-rate FP32 operations per axis.
constexpr float kRound = 12582912.0f;
template <int BOX>
__device__ __forceinline__ void imageT(float& dx, float& dy, float& dz, const BoxDev& b) {
    if (BOX == 1) {
        dx -= (fmaf(dx, b.inv[0], kRound) - kRound) * b.a[0];
        dy -= (fmaf(dy, b.inv[1], kRound) - kRound) * b.b[1];
        dz -= (fmaf(dz, b.inv[2], kRound) - kRound) * b.c[2];
    } else if (BOX == 2) {
        float s3 = fmaf(dz, b.inv[2], kRound) - kRound;
        dx -= s3 * b.c[0]; dy -= s3 * b.c[1]; dz -= s3 * b.c[2];
        float s2 = fmaf(dy, b.inv[1], kRound) - kRound;
        dx -= s2 * b.b[0]; dy -= s2 * b.b[1];
        float s1 = fmaf(dx, b.inv[0], kRound) - kRound;
        dx -= s1 * b.a[0];
    }
}

struct SwitchConst {
    float ir0, ir0sq, c;           // 1/r0, 1/r0^2, -n/r0^2
    float n, m;
    float r2hi;                    // pairs need r2 < r2hi: min(cutoff^2, (1000 r0)^2)
    int ni, mi;
};

// f and g = (df/dr)/r of one pair; pairs that are not valid contribute zero.
// Validity (reference: r2 >= 1e-20, x <= 1000, CommonGluedKernels.cpp:983-987;
// optional cutoff) is folded into the denominator: 1/inf = 0 makes f and g zero.
template <int NH>
__device__ __forceinline__ void pairSwitch(float r2, bool valid, const SwitchConst& s, float& f, float& g) {
    valid = valid && (r2 >= 1e-20f) && (r2 < s.r2hi);
    if (NH > 0) {
        float x2 = r2 * s.ir0sq;
        float p = 1.0f;
#pragma unroll
        for (int k = 1; k < NH; k++) p *= x2;
        float y = valid ? fmaf(p, x2, 1.0f) : __int_as_float(0x7f800000);
        float ff;
        asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(ff) : "f"(y));  // 1 ulp; rcp(inf) = 0
        f = ff;
        g = s.c * p * ff * ff;
    } else if (NH < 0) {
        float r = sqrtf(r2);
        float x = r * s.ir0;
        float ff, dfdx;
        ratioSwitch(x, s.ni, s.mi, ff, dfdx);
        f = valid ? ff : 0.0f;
        g = valid ? dfdx * s.ir0 / r : 0.0f;
    } else {
        // Non-integer exponents: the reference formula with its Taylor branch
        // within 1e-4 of x = 1 (CommonGluedKernels.cpp:983-1003), in FP64: in FP32
        // the quotient (1 - x^n)/(1 - x^m) loses up to ~1e-2 relative accuracy
        // through cancellation just outside the Taylor window.
        const double r = sqrt((double)r2);
        const double x = r * (double)s.ir0;
        const double n = s.n, m = s.m;
        double ff, dfdx;
        const double dx1 = x - 1.0;
        if (fabs(dx1) < 1e-4) {
            const double pre = n / m, df = 0.5 * n * (n - m) / m;
            const double sec = n * (m * m - 3.0 * m * (n - 1.0) + n * (2.0 * n - 3.0)) / (6.0 * m);
            ff = pre + dx1 * (df + 0.5 * dx1 * sec);
            dfdx = df + dx1 * sec;
        } else if (x < 1e-10) {
            ff = 1.0; dfdx = 0.0;
        } else {
            const double xn = pow(x, n), xm = pow(x, m);
            const double den = 1.0 - xm;
            ff = (1.0 - xn) / den;
            dfdx = (m * (xm / x) - n * (xn / x) + (n - m) * (xn * xm / x)) / (den * den);
        }
        f = valid ? (float)ff : 0.0f;
        g = valid ? (float)(dfdx * (double)s.ir0 / r) : 0.0f;
    }
}

template <int RA, int BOX, int NH>
__device__ __forceinline__ void coordTile(const float4* __restrict__ posq, const int* __restrict__ u2g,
                                          const CoordDev& C, const CoordItem& it, int ta, int sb,
                                          const BoxDev& box, float (*sB)[TB * 3], double* red) {
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int TA = NY * RA;
    SwitchConst s;
    s.ir0 = 1.0f / it.r0; s.ir0sq = s.ir0 * s.ir0; s.c = -it.n * s.ir0sq;
    s.n = it.n; s.m = it.m;
    s.ni = (int)it.n; s.mi = (int)it.m;
    {
        float xmax = 1000.0f * it.r0;
        float hi = xmax * xmax * 1.0000002f;
        s.r2hi = it.rc2 > 0.0f ? fminf(it.rc2, hi) : hi;
    }

    float ax[RA], ay[RA], az[RA], gax[RA], gay[RA], gaz[RA];
    bool aval[RA];
#pragma unroll
    for (int k = 0; k < RA; k++) {
        int i = ta * TA + ty + NY * k;
        aval[k] = i < it.nA;
        F3 p = aval[k] ? loadPos(posq, u2g, C.atoms[it.a0 + i]) : f3(0.f, 0.f, 0.f);
        ax[k] = p.x; ay[k] = p.y; az[k] = p.z;
        gax[k] = gay[k] = gaz[k] = 0.0f;
    }
    bool aFull = true;
#pragma unroll
    for (int k = 0; k < RA; k++) aFull = aFull && aval[k];
    aFull = __syncthreads_and(aFull);
    double cn = 0.0;
    const int bBeg = sb * C.bSplit;
    const int bEnd = min(it.nB, bBeg + C.bSplit);

    // software pipeline: positions of the next chunk are fetched before the
    // current chunk is computed
    float nbx[RB], nby[RB], nbz[RB];
#pragma unroll
    for (int j = 0; j < RB; j++) {
        int i = bBeg + tx + NX * j;
        F3 p = i < bEnd ? loadPos(posq, u2g, C.atoms[it.b0 + i]) : f3(0.f, 0.f, 0.f);
        nbx[j] = p.x; nby[j] = p.y; nbz[j] = p.z;
    }
    for (int c0 = bBeg; c0 < bEnd; c0 += TB) {
        float bx[RB], by[RB], bz[RB], gbx[RB], gby[RB], gbz[RB];
        bool bval[RB];
#pragma unroll
        for (int j = 0; j < RB; j++) {
            bx[j] = nbx[j]; by[j] = nby[j]; bz[j] = nbz[j];
            bval[j] = (c0 + tx + NX * j) < bEnd;
            gbx[j] = gby[j] = gbz[j] = 0.0f;
            int i = c0 + TB + tx + NX * j;
            F3 p = i < bEnd ? loadPos(posq, u2g, C.atoms[it.b0 + i]) : f3(0.f, 0.f, 0.f);
            nbx[j] = p.x; nby[j] = p.y; nbz[j] = p.z;
        }
        float cnc = 0.0f;
        // edge chunks / tiles carry the validity of each pair; full ones do not
        const bool full = aFull && (c0 + TB <= bEnd);
#define GL_PAIR_LOOP(MASKED)                                                                   \
        _Pragma("unroll") for (int k = 0; k < RA; k++) {                                      \
            _Pragma("unroll") for (int j = 0; j < RB; j++) {                                  \
                float dx = ax[k] - bx[j], dy = ay[k] - by[j], dz = az[k] - bz[j];             \
                imageT<BOX>(dx, dy, dz, box);                                                 \
                float r2 = dx * dx + dy * dy + dz * dz;                                       \
                float f, g;                                                                   \
                pairSwitch<NH>(r2, MASKED ? (aval[k] && bval[j]) : true, s, f, g);            \
                cnc += f;                                                                     \
                gax[k] += g * dx; gay[k] += g * dy; gaz[k] += g * dz;                         \
                gbx[j] -= g * dx; gby[j] -= g * dy; gbz[j] -= g * dz;                         \
            }                                                                                 \
        }
        if (full) { GL_PAIR_LOOP(false) } else { GL_PAIR_LOOP(true) }
#undef GL_PAIR_LOOP
        cn += (double)cnc;
        // B gradients: fixed-order sum over the 8 warps.
#pragma unroll
        for (int j = 0; j < RB; j++) {
            int o = (tx + NX * j) * 3;
            sB[ty][o] = gbx[j]; sB[ty][o + 1] = gby[j]; sB[ty][o + 2] = gbz[j];
        }
        __syncthreads();
        float* out = C.partB + 3 * ((size_t)it.partB + (size_t)ta * it.nB);
        for (int v = threadIdx.x; v < TB * 3; v += NX * NY) {
            int atom = c0 + v / 3;
            if (atom < bEnd) {
                float acc = 0.0f;
#pragma unroll
                for (int y = 0; y < NY; y++) acc += sB[y][v];
                out[(size_t)c0 * 3 + v] = acc;
            }
        }
        __syncthreads();
    }
    // A gradients: fixed xor-shuffle tree over the 32 lanes.
    float* outA = C.partA + 3 * ((size_t)it.partA + (size_t)sb * it.nA);
#pragma unroll
    for (int k = 0; k < RA; k++) {
        float x = warpSumF(gax[k]), y = warpSumF(gay[k]), z = warpSumF(gaz[k]);
        int i = ta * TA + ty + NY * k;
        if (tx == 0 && aval[k]) { outA[3 * i] = x; outA[3 * i + 1] = y; outA[3 * i + 2] = z; }
    }
    double v[1] = {cn};
    blockSum<1>(v, red);
    if (threadIdx.x == 0) C.cnPart[it.cn0 + ta * it.splitsB + sb] = v[0];
}

}  // namespace glued
