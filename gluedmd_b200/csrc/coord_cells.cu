// Cutoff coordination (CV_COORDINATION_CUTOFF, an extension with no reference
// counterpart; the pair terms are the reference's, CommonGluedKernels.cpp:969-1027,
// restricted to pairs closer than rc) through a cell list on the device instead
// of all-pairs tiles with a mask.
//
// Decisions. A pair (A atom, B atom) counts when 1e-20 <= r^2 < rc^2, with r^2
// formed in FP64 from the FP32 positions exactly as the FP64 oracle forms it
// (difference, minimum image floor(d inv + 1/2) along c, b, a, then
// x^2 + y^2 + z^2, every operation rounded on its own), so the pair list equals
// the oracle's bit for bit. The pair terms themselves are FP32, as on the tile
// path (scaled units, the same switch functions).
//
// Cells. In a rectangular periodic box each dimension gets
// n_d = min(CELL_MAX_DIM, floor(L_d / rc)) cells (of width >= rc), or 1 cell
// when that is below 3 (the 27-cell stencil would visit a cell twice). Any pair
// closer than rc is then in neighbouring cells. Other boxes (triclinic, or no
// periodicity) use one cell: every B atom is a candidate.
//
// k_cell_bin (one CTA per item) sorts the B atoms by cell with a stable
// counting sort: counts, a scan, then chunks of 1024 atoms in index order, each
// atom's slot = the cell's cursor + same-cell atoms of earlier warps in the chunk
// + same-cell lanes before it in its warp (match_any). Within a cell the atoms
// stay in index order, so the candidate order is fixed.
//
// k_cell_pairs (CELL_SPLIT warps per A atom, one z slice of the stencil each)
// visits the slice's cells in a fixed order, lanes striding over each cell's
// atoms. CN partial of the (A atom, slice): lane sums in FP64, fixed butterfly,
// stored to its own cnPiece slot (the finalize adds the item's slots in order).
// Gradients: A sums over lanes (FP32 butterfly) and every B term go to the
// 64-bit fixed-point accumulator rows, as on the tile path, so k_coord_finalize
// turns them into Jacobian rows unchanged. EMIT = 1 counts the pairs of every
// warp, EMIT = 2 writes them (test and diagnostic use).
#include "coord_run.cuh"
#include "kernels.hpp"
#include "pdl.cuh"

namespace glued {

namespace {

struct D3 {
    double x, y, z;
};

__device__ __forceinline__ D3 cellImage(D3 d, const CellBox& b) {
    const double s3 = floor(__dadd_rn(__dmul_rn(d.z, b.inv[2]), 0.5));
    d.x = __dsub_rn(d.x, __dmul_rn(s3, b.c[0]));
    d.y = __dsub_rn(d.y, __dmul_rn(s3, b.c[1]));
    d.z = __dsub_rn(d.z, __dmul_rn(s3, b.c[2]));
    const double s2 = floor(__dadd_rn(__dmul_rn(d.y, b.inv[1]), 0.5));
    d.x = __dsub_rn(d.x, __dmul_rn(s2, b.b[0]));
    d.y = __dsub_rn(d.y, __dmul_rn(s2, b.b[1]));
    const double s1 = floor(__dadd_rn(__dmul_rn(d.x, b.inv[0]), 0.5));
    d.x = __dsub_rn(d.x, __dmul_rn(s1, b.a[0]));
    return d;
}

__device__ __forceinline__ void cellDims(const CellBox& b, double rc, int (&nc)[3]) {
    nc[0] = nc[1] = nc[2] = 1;
    if (b.kind != 1) return;
    const double L[3] = {b.a[0], b.b[1], b.c[2]};
#pragma unroll
    for (int d = 0; d < 3; d++) {
        int k = (int)floor(L[d] / (rc * (1.0 + 1e-9)));
        k = k < CELL_MAX_DIM ? k : CELL_MAX_DIM;
        nc[d] = k >= 3 ? k : 1;
    }
}

__device__ __forceinline__ int cellCoord(double x, double inv, int n) {
    if (n == 1) return 0;
    double f = x * inv;
    f -= floor(f);
    const int c = (int)(f * (double)n);
    return c >= n ? n - 1 : (c < 0 ? 0 : c);
}

__device__ __forceinline__ int cellOf(const float4& p, const CellBox& b, const int (&nc)[3]) {
    const int cx = cellCoord((double)p.x, b.inv[0], nc[0]);
    const int cy = cellCoord((double)p.y, b.inv[1], nc[1]);
    const int cz = cellCoord((double)p.z, b.inv[2], nc[2]);
    return (cz * nc[1] + cy) * nc[0] + cx;
}

}  // namespace

constexpr int BIN_THREADS = 1024;
constexpr int BIN_PER = 8;   // atoms per thread held in registers between the two passes

__global__ void __launch_bounds__(BIN_THREADS) k_cell_bin(const CellItemDev* __restrict__ items,
                                                          const int* __restrict__ slots,
                                                          const float4* __restrict__ posq,
                                                          const CellBox* __restrict__ boxp) {
    __shared__ int cnt[CELL_MAX], cursor[CELL_MAX];
    __shared__ unsigned char wc[BIN_THREADS / 32][CELL_MAX];
    pdlEnter();
    const CellItemDev& it = items[blockIdx.x];
    const CellBox box = *boxp;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nB = it.nB;
    int nc[3];
    cellDims(box, it.rc, nc);
    const int ncell = nc[0] * nc[1] * nc[2];
    for (int c = tid; c < ncell; c += BIN_THREADS) cnt[c] = 0;
    for (int i = tid; i < (BIN_THREADS / 32) * CELL_MAX; i += BIN_THREADS) (&wc[0][0])[i] = 0;
    __syncthreads();
    const int* bs = slots + it.b0;
    constexpr int GROUP = BIN_PER * BIN_THREADS;
    float4 P[BIN_PER];
    int C[BIN_PER];
    // positions and cells of one group of atoms, every load issued before any use
    auto load = [&](int g0) {
        int sl[BIN_PER];
#pragma unroll
        for (int k = 0; k < BIN_PER; k++) {
            const int j = g0 + k * BIN_THREADS + tid;
            sl[k] = j < nB ? bs[j] : -1;
        }
#pragma unroll
        for (int k = 0; k < BIN_PER; k++) P[k] = sl[k] >= 0 ? posq[sl[k]] : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int k = 0; k < BIN_PER; k++) C[k] = sl[k] >= 0 ? cellOf(P[k], box, nc) : -1;
    };
    for (int g0 = 0; g0 < nB; g0 += GROUP) {
        load(g0);
#pragma unroll
        for (int k = 0; k < BIN_PER; k++)
            if (C[k] >= 0) atomicAdd(&cnt[C[k]], 1);
    }
    __syncthreads();
    if (tid == 0) {
        int s = 0;
        for (int c = 0; c < ncell; c++) {
            it.cellStart[c] = s;
            cursor[c] = s;
            s += cnt[c];
        }
        it.cellStart[ncell] = s;
        it.grid[0] = nc[0]; it.grid[1] = nc[1]; it.grid[2] = nc[2]; it.grid[3] = ncell;
    }
    __syncthreads();
    // stable scatter, chunks of BIN_THREADS atoms in index order
    const unsigned lt = (1u << lane) - 1u;
    for (int g0 = 0; g0 < nB; g0 += GROUP) {
        if (nB > GROUP) load(g0);   // one group: still in registers
#pragma unroll
        for (int k = 0; k < BIN_PER; k++) {
            if (g0 + k * BIN_THREADS >= nB) break;   // uniform
            const int c = C[k];
            const unsigned m = __match_any_sync(0xffffffffu, c);
            const bool leader = (m & lt) == 0;
            if (c >= 0 && leader) wc[warp][c] = (unsigned char)__popc(m);
            __syncthreads();
            if (c >= 0) {
                int cross = 0;
                for (int w = 0; w < warp; w++) cross += wc[w][c];
                const int slot = cursor[c] + cross + __popc(m & lt);
                it.sortedB[slot] = g0 + k * BIN_THREADS + tid;
                it.sortedPos[slot] = P[k];
            }
            __syncthreads();
            if (c >= 0 && leader) {
                atomicAdd(&cursor[c], __popc(m));
                wc[warp][c] = 0;
            }
            __syncthreads();
        }
    }
}

// Warps (CELL_SPLIT w + z) of the grid take A atom w of the cell items
// (item-major), z-slice z of its stencil (dz = z - 1; slices 1 and 2 are empty
// when the box has one cell along z). Candidates pass a loose FP32 test first
// (r^2 below rc^2 (1 + 1e-3) + 1e-6 L^2, far above the FP32 rounding of r^2);
// the decision is then the FP64 one. EMIT: 0 evaluate; 1 pairCount[warp] = pairs
// found; 2 write them as (a, b) at pairs[2 * (pairOffset[warp] + k)], in
// candidate order.
template <int NH, int EMIT>
__global__ void __launch_bounds__(256) k_cell_pairs(const CellItemDev* __restrict__ items, int numItems,
                                                    const int* __restrict__ slots, const float4* __restrict__ posq,
                                                    const CellBox* __restrict__ boxp, unsigned long long* __restrict__ acc,
                                                    double* __restrict__ cnPiece, int* __restrict__ pairCount,
                                                    const long long* __restrict__ pairOffset,
                                                    int* __restrict__ pairs) {
    const int lane = threadIdx.x & 31;
    const int gw = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
    const int zs = gw % CELL_SPLIT;
    int a = gw / CELL_SPLIT;
    int wi = 0;
    while (wi < numItems && a >= items[wi].nA) { a -= items[wi].nA; wi++; }
    pdlEnter();
    if (wi >= numItems) return;   // warp-uniform
    const CellItemDev& it = items[wi];
    const CellBox box = *boxp;
    const float4 pa = posq[slots[it.a0 + a]];
    const D3 A = {(double)pa.x, (double)pa.y, (double)pa.z};
    const int nx = it.grid[0], ny = it.grid[1], nz = it.grid[2];
    const int cx = cellCoord(A.x, box.inv[0], nx), cy = cellCoord(A.y, box.inv[1], ny),
              cz = cellCoord(A.z, box.inv[2], nz);
    RunConst K;
    K.n = it.n; K.m = it.m; K.ni = (int)it.n; K.mi = (int)it.m; K.ir0 = 1.0f / it.r0;
    const double ir0 = 1.0 / (double)it.r0, ir02 = ir0 * ir0;
    const double rc2 = it.rc2;
    const bool periodic = box.kind != 0;
    // FP32 copy of the box for the pre-test
    const float fa0 = (float)box.a[0], fb0 = (float)box.b[0], fb1 = (float)box.b[1];
    const float fc0 = (float)box.c[0], fc1 = (float)box.c[1], fc2 = (float)box.c[2];
    const float fi0 = (float)box.inv[0], fi1 = (float)box.inv[1], fi2 = (float)box.inv[2];
    const double Lm = fmax(fmax(fabs(box.a[0]), fabs(box.b[1])), fabs(box.c[2]));
    const float loose = (float)(rc2 * (1.0 + 1e-3) + 1e-6 * Lm * Lm);
    double cn = 0.0;
    float gx = 0.f, gy = 0.f, gz = 0.f;
    int found = 0;
    long long out = EMIT == 2 ? pairOffset[gw] : 0;
    const bool sliceLive = nz >= 3 || zs == 0;
    const int dz = nz >= 3 ? zs - 1 : 0;
    const int oy = ny >= 3 ? -1 : 0, ey = ny >= 3 ? 1 : 0;
    const int ox = nx >= 3 ? -1 : 0, ex = nx >= 3 ? 1 : 0;
    if (sliceLive)
        for (int dy = oy; dy <= ey; dy++)
            for (int dx = ox; dx <= ex; dx++) {
                const int c = (((cz + dz + nz) % nz) * ny + (cy + dy + ny) % ny) * nx + (cx + dx + nx) % nx;
                const int s = it.cellStart[c], e = it.cellStart[c + 1];
                for (int k0 = s; k0 < e; k0 += 32) {
                    const int k = k0 + lane;
                    bool in = false;
                    D3 d = {0.0, 0.0, 0.0};
                    double r2 = 0.0;
                    if (k < e) {
                        const float4 pb = it.sortedPos[k];
                        float ux = pa.x - pb.x, uy = pa.y - pb.y, uz = pa.z - pb.z;
                        if (periodic) {
                            const float s3 = floorf(fmaf(uz, fi2, 0.5f));
                            ux = fmaf(-s3, fc0, ux); uy = fmaf(-s3, fc1, uy); uz = fmaf(-s3, fc2, uz);
                            const float s2 = floorf(fmaf(uy, fi1, 0.5f));
                            ux = fmaf(-s2, fb0, ux); uy = fmaf(-s2, fb1, uy);
                            const float s1 = floorf(fmaf(ux, fi0, 0.5f));
                            ux = fmaf(-s1, fa0, ux);
                        }
                        if (fmaf(uz, uz, fmaf(uy, uy, ux * ux)) < loose) {
                            d = {__dsub_rn(A.x, (double)pb.x), __dsub_rn(A.y, (double)pb.y),
                                 __dsub_rn(A.z, (double)pb.z)};
                            if (periodic) d = cellImage(d, box);
                            r2 = __dadd_rn(__dadd_rn(__dmul_rn(d.x, d.x), __dmul_rn(d.y, d.y)), __dmul_rn(d.z, d.z));
                            in = !(r2 < 1e-20) && r2 < rc2;
                        }
                    }
                    if (EMIT == 1) {
                        found += __popc(__ballot_sync(0xffffffffu, in));
                        continue;
                    }
                    if (EMIT == 2) {
                        const unsigned bm = __ballot_sync(0xffffffffu, in);
                        if (in) {
                            const long long o = out + __popc(bm & ((1u << lane) - 1u));
                            pairs[2 * o] = a;
                            pairs[2 * o + 1] = it.sortedB[k];
                        }
                        out += __popc(bm);
                        continue;
                    }
                    if (in) {
                        const float sx = (float)(d.x * ir0), sy = (float)(d.y * ir0), sz = (float)(d.z * ir0);
                        const float x2 = (float)(r2 * ir02);
                        float f, h;
                        switchX2<NH>(x2, true, K, f, h);
                        cn += (double)f;
                        const float hx = h * sx, hy = h * sy, hz = h * sz;
                        gx += hx; gy += hy; gz += hz;
                        unsigned long long* rb = acc + 3 * (size_t)(it.row0 + it.nA + it.sortedB[k]);
                        redAddI64(rb, __float2ll_rn(-hx * crun::FX));
                        redAddI64(rb + 1, __float2ll_rn(-hy * crun::FX));
                        redAddI64(rb + 2, __float2ll_rn(-hz * crun::FX));
                    }
                }
            }
    if (EMIT == 1) {
        if (lane == 0) pairCount[gw] = found;
        return;
    }
    if (EMIT == 2) return;
    gx = warpSumF(gx); gy = warpSumF(gy); gz = warpSumF(gz);
    cn = warpSum(cn);
    if (lane == 0) {
        if (sliceLive) {
            unsigned long long* ra = acc + 3 * (size_t)(it.row0 + a);
            redAddI64(ra, __float2ll_rn(gx * crun::FX));
            redAddI64(ra + 1, __float2ll_rn(gy * crun::FX));
            redAddI64(ra + 2, __float2ll_rn(gz * crun::FX));
        }
        cnPiece[it.pieceBegin + CELL_SPLIT * a + zs] = cn;   // every slot written, empty slices 0
    }
}

template <int EMIT>
static void launchPairs(cudaStream_t s, int kind, int totalA, const CellItemDev* items, int numItems,
                        const int* slots, const float4* posq, const CellBox* box, unsigned long long* acc,
                        double* cnPiece, int* pairCount, const long long* pairOffset, int* pairs) {
    const dim3 grid((unsigned)((CELL_SPLIT * (long long)totalA * 32 + 255) / 256)), block(256);
    if (kind == 3)
        launchPdl(k_cell_pairs<3, EMIT>, grid, block, 0, s, items, numItems, slots, posq, box, acc, cnPiece, pairCount,
                  pairOffset, pairs);
    else if (kind == -1)
        launchPdl(k_cell_pairs<-1, EMIT>, grid, block, 0, s, items, numItems, slots, posq, box, acc, cnPiece,
                  pairCount, pairOffset, pairs);
    else
        launchPdl(k_cell_pairs<0, EMIT>, grid, block, 0, s, items, numItems, slots, posq, box, acc, cnPiece, pairCount,
                  pairOffset, pairs);
}

void launchCellCoord(cudaStream_t s, const CellItemDev* items, int numItems, int totalA, int kind, const int* slots,
                     const float4* posq, const CellBox* box, unsigned long long* acc, double* cnPiece) {
    if (numItems == 0 || totalA == 0) return;
    launchPdl(k_cell_bin, dim3(numItems), dim3(BIN_THREADS), 0, s, items, slots, posq, box);
    launchPairs<0>(s, kind, totalA, items, numItems, slots, posq, box, acc, cnPiece, nullptr, nullptr, nullptr);
}

void launchCellPairList(cudaStream_t s, const CellItemDev* items, int numItems, int totalA, int kind, const int* slots,
                        const float4* posq, const CellBox* box, int* pairCount, const long long* pairOffset,
                        int* pairs, int pass) {
    if (numItems == 0 || totalA == 0) return;
    if (pass == 1) {
        launchPdl(k_cell_bin, dim3(numItems), dim3(BIN_THREADS), 0, s, items, slots, posq, box);
        launchPairs<1>(s, kind, totalA, items, numItems, slots, posq, box, nullptr, nullptr, pairCount, nullptr,
                       nullptr);
    } else {
        launchPairs<2>(s, kind, totalA, items, numItems, slots, posq, box, nullptr, nullptr, nullptr, pairOffset,
                       pairs);
    }
}

}  // namespace glued
