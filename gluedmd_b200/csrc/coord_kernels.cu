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
#include "coord_tile.cuh"
#include "kernels.hpp"

namespace glued {

// One instantiation per switch kind (all items of a launch share it): kind 3 is
// n = 6, m = 12; -1 any other integer pair; 0 non-integer exponents.
template <int RA, int BOX, int NH>
__global__ void __launch_bounds__(256, 2) k_coord_pairs(const float4* __restrict__ posq, const int* __restrict__ u2g,
                                                        CoordDev C, const BoxDev* __restrict__ boxp) {
    __shared__ float sB[NY][TB * 3];
    __shared__ double red[32];
    const CoordItem it = C.items[C.blockItem[blockIdx.x]];
    const BoxDev box = *boxp;
    int local = blockIdx.x - it.block0;
    int ta = local / it.splitsB, sb = local % it.splitsB;
    coordTile<RA, BOX, NH>(posq, u2g, C, it, ta, sb, box, sB, red);
}

// Sum partials in fixed order: A atoms over B splits, B atoms over A tiles,
// CN over the item's CTAs. One thread per (row, component); the partial loads of
// a thread are independent and issued together.
__global__ void k_coord_finalize(CoordDev C, JacDev J, double* __restrict__ cvv, int totalRows) {
    int gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid < 3 * totalRows) {
        const int comp = gid % 3;
        const int row = gid / 3;
        int ii = 0, base = 0;
        while (ii < C.numItems - 1 && row >= base + C.items[ii].nA + C.items[ii].nB) {
            base += C.items[ii].nA + C.items[ii].nB;
            ii++;
        }
        const CoordItem& it = C.items[ii];
        const int i = row - base;
        const float* p;
        int n;
        size_t stride;
        if (i < it.nA) {
            p = C.partA + 3 * ((size_t)it.partA + i) + comp;
            n = it.splitsB;
            stride = 3 * (size_t)it.nA;
        } else {
            p = C.partB + 3 * ((size_t)it.partB + (i - it.nA)) + comp;
            n = it.tilesA;
            stride = 3 * (size_t)it.nB;
        }
        double acc = 0.0;
        int k = 0;
        for (; k + 8 <= n; k += 8) {
            float v[8];
#pragma unroll
            for (int u = 0; u < 8; u++) v[u] = __ldg(p + (size_t)(k + u) * stride);
#pragma unroll
            for (int u = 0; u < 8; u++) acc += v[u];
        }
        for (; k < n; k++) acc += __ldg(p + (size_t)k * stride);
        float* out = comp == 0 ? J.gx : comp == 1 ? J.gy : J.gz;
        out[it.jac0 + i] = (float)acc;
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
                 int totalRows, int boxKind, int ra, int kind, const BoxDev* box, const JacDev& J, double* cvv,
                 int parts) {
    if (C.numItems == 0) return;
    if (parts & 1) {
#define GL_K(RA_, BX_, NH_) k_coord_pairs<RA_, BX_, NH_><<<numBlocks, 256, 0, s>>>(posq, u2g, C, box)
#define GL_KB(RA_, NH_) \
        if (boxKind == 0) GL_K(RA_, 0, NH_); else if (boxKind == 1) GL_K(RA_, 1, NH_); else GL_K(RA_, 2, NH_)
#define GL_KN(RA_) \
        if (kind == 3) { GL_KB(RA_, 3); } else if (kind == -1) { GL_KB(RA_, -1); } else { GL_KB(RA_, 0); }
        if (ra == 8) { GL_KN(8) } else { GL_KN(4) }
#undef GL_KN
#undef GL_KB
#undef GL_K
    }
    if (parts & 2) k_coord_finalize<<<(3 * totalRows + 255) / 256, 256, 0, s>>>(C, J, cvv, totalRows);
}

}  // namespace glued
