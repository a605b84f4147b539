// Coordination number CV (CommonGluedKernels.cpp:899-1031): all ng1 x ng2
// minimum-image pairs of the rational switch f = (1 - x^n) / (1 - x^m), x = r/r0.
//
// The reference evaluates every pair of a CV in one GPU thread. Here one CTA
// takes a tile of TA = 8*RA group-A atoms against a split of group B:
//   - warp w holds A atoms {w, w+8, ...} in registers (all lanes share them),
//   - lane l walks B atoms {l, l+32, l+64, l+96} of each 128-atom chunk,
//   - per-pair force factor g = (df/dr)/r; A gradients accumulate in registers
//     and are reduced over lanes by a fixed shuffle tree at the end; B gradients
//     of a chunk are reduced over the 8 warps through shared memory in fixed
//     order and written once per (A tile, B atom);
//   - the CN partial of each CTA is a double written to its own slot.
// k_coord_finalize then sums the partials over splits / tiles in a fixed order,
// so results are bitwise reproducible run to run (no float atomics).
//
// Switch kinds:
//   k > 0 : m == 2n with n == 2k:  f = 1/(1 + x^n),  g = -n x^(n-2) f^2 / r0^2,
//           no square root and no pow;
//   -1    : integer n, m (1..64):   f = S_n(x) / S_m(x),  S_k(x) = sum_{j<k} x^j,
//           the same rational function without the cancellation of
//           (1 - x^n)/(1 - x^m) near x = 1, which in FP32 costs up to ~1e-3
//           relative force error outside the reference's |x-1| < 1e-4 Taylor
//           window (CommonGluedKernels.cpp:983-1003);
//   0     : non-integer exponents: the reference formula (pow, Taylor branch).
#include "devfn.cuh"
#include "kernels.hpp"

namespace glued {

namespace {
constexpr int NY = 8;     // warps per CTA
constexpr int NX = 32;    // lanes
constexpr int RB = 4;     // B atoms per lane per chunk
constexpr int TB = NX * RB;  // B chunk (128 atoms)
}

template <int BOX>
__device__ __forceinline__ void imageT(float& dx, float& dy, float& dz, const BoxDev& b) {
    if (BOX == 1) {
        dx -= floorf(dx * b.inv[0] + 0.5f) * b.a[0];
        dy -= floorf(dy * b.inv[1] + 0.5f) * b.b[1];
        dz -= floorf(dz * b.inv[2] + 0.5f) * b.c[2];
    } else if (BOX == 2) {
        float s3 = floorf(dz * b.inv[2] + 0.5f);
        dx -= s3 * b.c[0]; dy -= s3 * b.c[1]; dz -= s3 * b.c[2];
        float s2 = floorf(dy * b.inv[1] + 0.5f);
        dx -= s2 * b.b[0]; dy -= s2 * b.b[1];
        float s1 = floorf(dx * b.inv[0] + 0.5f);
        dx -= s1 * b.a[0];
    }
}

struct SwitchConst {
    float ir0, ir0sq, c;           // 1/r0, 1/r0^2, -n/r0^2
    float n, m, preRes, preDf, preSec;
    float rc2;
    int ni, mi;
};

// Returns f and g = (df/dr)/r for one pair; valid == false -> no contribution.
template <int NH>
__device__ __forceinline__ void pairSwitch(float r2, const SwitchConst& s, float& f, float& g) {
    bool valid = (r2 >= 1e-20f) && (s.rc2 == 0.0f || r2 < s.rc2);
    if (NH > 0) {
        float x2 = r2 * s.ir0sq;
        valid = valid && (x2 <= 1e6f);
        float p = 1.0f;
#pragma unroll
        for (int k = 1; k < NH; k++) p *= x2;
        float xn = p * x2;
        float ff = __fdividef(1.0f, 1.0f + xn);
        f = valid ? ff : 0.0f;
        g = valid ? s.c * p * ff * ff : 0.0f;
    } else if (NH < 0) {
        float r = sqrtf(r2);
        float x = r * s.ir0;
        valid = valid && (x <= 1000.0f);
        float ff, dfdx;
        ratioSwitch(x, s.ni, s.mi, ff, dfdx);
        f = valid ? ff : 0.0f;
        g = valid ? dfdx * s.ir0 / r : 0.0f;
    } else {
        float r = sqrtf(r2);
        float x = r * s.ir0;
        valid = valid && (x <= 1000.0f);
        float ff, dfdr;
        float dx1 = x - 1.0f;
        if (fabsf(dx1) < 1e-4f) {
            ff = s.preRes + dx1 * (s.preDf + 0.5f * dx1 * s.preSec);
            dfdr = (s.preDf + dx1 * s.preSec) * s.ir0;
        } else if (x < 1e-10f) {
            ff = 1.0f; dfdr = 0.0f;
        } else {
            float xn = powf(x, s.n), xm = powf(x, s.m);
            float den = 1.0f - xm;
            ff = (1.0f - xn) / den;
            float dfx = (s.m * (xm / x) - s.n * (xn / x) + (s.n - s.m) * (xn * xm / x)) / (den * den);
            dfdr = dfx * s.ir0;
        }
        f = valid ? ff : 0.0f;
        g = valid ? dfdr / r : 0.0f;
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
    s.n = it.n; s.m = it.m; s.rc2 = it.rc2;
    s.ni = (int)it.n; s.mi = (int)it.m;
    s.preRes = s.n / s.m;
    s.preDf = 0.5f * s.n * (s.n - s.m) / s.m;
    s.preSec = s.n * (s.m * s.m - 3.0f * s.m * (s.n - 1.0f) + s.n * (2.0f * s.n - 3.0f)) / (6.0f * s.m);

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
#pragma unroll
        for (int k = 0; k < RA; k++) {
#pragma unroll
            for (int j = 0; j < RB; j++) {
                float dx = ax[k] - bx[j], dy = ay[k] - by[j], dz = az[k] - bz[j];
                imageT<BOX>(dx, dy, dz, box);
                float r2 = dx * dx + dy * dy + dz * dz;
                float f, g;
                pairSwitch<NH>(r2, s, f, g);
                if (!(aval[k] && bval[j])) { f = 0.0f; g = 0.0f; }
                cnc += f;
                gax[k] += g * dx; gay[k] += g * dy; gaz[k] += g * dz;
                gbx[j] -= g * dx; gby[j] -= g * dy; gbz[j] -= g * dz;
            }
        }
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

template <int RA, int BOX>
__global__ void __launch_bounds__(256) k_coord_pairs(const float4* __restrict__ posq, const int* __restrict__ u2g,
                                                     CoordDev C, const BoxDev* __restrict__ boxp) {
    __shared__ float sB[NY][TB * 3];
    __shared__ double red[32];
    const CoordItem it = C.items[C.blockItem[blockIdx.x]];
    const BoxDev box = *boxp;
    int local = blockIdx.x - it.block0;
    int ta = local / it.splitsB, sb = local % it.splitsB;
    switch (it.kind) {
        case 1: coordTile<RA, BOX, 1>(posq, u2g, C, it, ta, sb, box, sB, red); break;
        case 2: coordTile<RA, BOX, 2>(posq, u2g, C, it, ta, sb, box, sB, red); break;
        case 3: coordTile<RA, BOX, 3>(posq, u2g, C, it, ta, sb, box, sB, red); break;
        case 4: coordTile<RA, BOX, 4>(posq, u2g, C, it, ta, sb, box, sB, red); break;
        case -1: coordTile<RA, BOX, -1>(posq, u2g, C, it, ta, sb, box, sB, red); break;
        default: coordTile<RA, BOX, 0>(posq, u2g, C, it, ta, sb, box, sB, red); break;
    }
}

// Sum partials in fixed order: A atoms over B splits, B atoms over A tiles,
// CN over the item's CTAs. Writes Jacobian gradients and cvValues.
__global__ void k_coord_finalize(CoordDev C, JacDev J, double* __restrict__ cvv, int totalRows) {
    int gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid < totalRows) {
        int ii = 0, base = 0;
        while (ii < C.numItems - 1 && gid >= base + C.items[ii].nA + C.items[ii].nB) {
            base += C.items[ii].nA + C.items[ii].nB;
            ii++;
        }
        const CoordItem& it = C.items[ii];
        int i = gid - base;
        double x = 0, y = 0, z = 0;
        if (i < it.nA) {
            const float* p = C.partA + 3 * ((size_t)it.partA + i);
            for (int sb = 0; sb < it.splitsB; sb++) {
                const float* q = p + 3 * (size_t)sb * it.nA;
                x += q[0]; y += q[1]; z += q[2];
            }
        } else {
            int b = i - it.nA;
            const float* p = C.partB + 3 * ((size_t)it.partB + b);
            for (int ta = 0; ta < it.tilesA; ta++) {
                const float* q = p + 3 * (size_t)ta * it.nB;
                x += q[0]; y += q[1]; z += q[2];
            }
        }
        int r = it.jac0 + i;
        J.gx[r] = (float)x; J.gy[r] = (float)y; J.gz[r] = (float)z;
    }
    if (blockIdx.x == 0 && threadIdx.x < 32) {
        for (int ii = 0; ii < C.numItems; ii++) {
            const CoordItem& it = C.items[ii];
            int nb = it.tilesA * it.splitsB;
            double s = 0;
            for (int k = threadIdx.x; k < nb; k += 32) s += C.cnPart[it.cn0 + k];
            s = warpSum(s);
            if (threadIdx.x == 0) cvv[it.cv] = s;
        }
    }
}

void launchCoord(cudaStream_t s, const float4* posq, const int* u2g, const CoordDev& C, int numBlocks,
                 int totalRows, int boxKind, int ra, const BoxDev* box, const JacDev& J, double* cvv) {
    if (C.numItems == 0) return;
#define GL_COORD(RA_, BX_) k_coord_pairs<RA_, BX_><<<numBlocks, 256, 0, s>>>(posq, u2g, C, box)
    if (ra == 8) {
        if (boxKind == 0) GL_COORD(8, 0); else if (boxKind == 1) GL_COORD(8, 1); else GL_COORD(8, 2);
    } else {
        if (boxKind == 0) GL_COORD(4, 0); else if (boxKind == 1) GL_COORD(4, 1); else GL_COORD(4, 2);
    }
#undef GL_COORD
    k_coord_finalize<<<(totalRows + 255) / 256, 256, 0, s>>>(C, J, cvv, totalRows);
}

}  // namespace glued
