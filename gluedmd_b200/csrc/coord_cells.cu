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
// Binning, a counting sort of the B atoms by cell in three launches:
// k_cell_count (one thread per B atom) writes every atom's cell and position and
// counts the cells with integer atomics; k_cell_scan turns the counts into cell
// starts and write cursors; k_cell_scatter places every atom at its cell's next
// slot. The order within a cell follows the atomics, which is why every sum of
// the pairs kernel is formed in 64-bit fixed point (exact, order-independent):
// the results are bitwise reproducible all the same. The pairs kernel clears
// the counts after its wait.
//
// k_cell_pairs (CELL_SPLIT warps per A atom, one z slice of the stencil each)
// visits the slice's cells, lanes striding over each cell's atoms. Every pair
// term (switch value, gradient components) is converted to 64-bit fixed point
// (value * 2^32) and summed exactly: the CN per CTA into the item's one CN
// accumulator (k_coord_finalize converts and clears it), the A sums and every B
// term to the fixed-point accumulator rows, as on the tile path, so
// k_coord_finalize turns them into Jacobian rows unchanged. EMIT = 1
// counts the pairs of every warp, EMIT = 2 writes them (test and diagnostic
// use; the host sorts the list).
#include <algorithm>

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

constexpr int COUNT_THREADS = 256;

// Binning, first half (grid: B atoms x items): the cell of every B atom and its
// position into cellId / posB, per-cell counts with integer atomics (one per
// distinct cell of a warp), and the cell grid.
__global__ void __launch_bounds__(COUNT_THREADS) k_cell_count(const CellItemDev* __restrict__ items,
                                                              const int* __restrict__ slots,
                                                              const float4* __restrict__ posq,
                                                              const CellBox* __restrict__ boxp) {
    pdlEnter();
    const CellItemDev& it = items[blockIdx.y];
    const CellBox box = *boxp;
    int nc[3];
    cellDims(box, it.rc, nc);
    const int j = blockIdx.x * COUNT_THREADS + threadIdx.x;
    int c = -1;
    if (j < it.nB) {
        const float4 p = posq[slots[it.b0 + j]];
        c = cellOf(p, box, nc);
        it.cellId[j] = c;
        it.posB[j] = p;
    }
    const unsigned m = __match_any_sync(0xffffffffu, c);
    if (c >= 0 && (m & ((1u << (threadIdx.x & 31)) - 1u)) == 0) atomicAdd(it.counts + c, __popc(m));
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        it.grid[0] = nc[0]; it.grid[1] = nc[1]; it.grid[2] = nc[2]; it.grid[3] = nc[0] * nc[1] * nc[2];
    }
}

// Binning, second step (one CTA per item): exclusive scan of the counts into
// cellStart; the counts become the cells' write cursors.
__global__ void __launch_bounds__(CELL_MAX) k_cell_scan(const CellItemDev* __restrict__ items) {
    __shared__ int wsum[CELL_MAX / 32];
    pdlEnter();
    const CellItemDev& it = items[blockIdx.x];
    const int ncell = it.grid[3];
    const int c = threadIdx.x, lane = c & 31, warp = c >> 5;
    const int v = c < ncell ? it.counts[c] : 0;
    int x = v;   // inclusive warp scan
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    int before = 0;
    for (int w = 0; w < warp; w++) before += wsum[w];
    const int start = before + x - v;
    if (c < ncell) {
        it.cellStart[c] = start;
        it.counts[c] = start;
    }
    if (c == 0) it.cellStart[ncell] = it.nB;
}

// Binning, third step (one thread per B atom): each atom takes the next slot of
// its cell (one atomic per distinct cell of a warp). The order within a cell
// depends on the atomics' order; every sum the pairs kernel forms is in 64-bit
// fixed point, so the results do not.
__global__ void __launch_bounds__(COUNT_THREADS) k_cell_scatter(const CellItemDev* __restrict__ items) {
    pdlEnter();
    const CellItemDev& it = items[blockIdx.y];
    const int j = blockIdx.x * COUNT_THREADS + threadIdx.x;
    const int c = j < it.nB ? it.cellId[j] : -1;
    const unsigned m = __match_any_sync(0xffffffffu, c);
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(m) - 1;
    int base = 0;
    if (c >= 0 && lane == leader) base = atomicAdd(it.counts + c, __popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (c >= 0) {
        const int slot = base + __popc(m & ((1u << lane) - 1u));
        it.sortedB[slot] = j;
        it.sortedPos[slot] = it.posB[j];
    }
}

// Warps (CELL_SPLIT w + z) of the grid take A atom w of the cell items
// (item-major), z-slice z of its stencil (dz = z - 1; slices 1 and 2 are empty
// when the box has one cell along z). Every candidate's r^2 is formed in FP32
// first; only those within a margin (1e-3 rc^2 + 1e-6 L^2, far above the FP32
// rounding of r^2) of the cutoff or near the lower bound are decided in FP64,
// the rest are inside or outside beyond any rounding, so the decisions are the
// FP64 oracle's. Pair terms use the FP32 difference, or the FP64 one where it
// was formed. EMIT: 0 evaluate; 1 pairCount[warp] = pairs
// found; 2 write them as (a, b) at pairs[2 * (pairOffset[warp] + k)], in
// candidate order.
template <int NH, int EMIT>
__global__ void __launch_bounds__(256) k_cell_pairs(const CellItemDev* __restrict__ items, int numItems,
                                                    const int* __restrict__ slots, const float4* __restrict__ posq,
                                                    const CellBox* __restrict__ boxp, unsigned long long* __restrict__ acc,
                                                    int* __restrict__ pairCount,
                                                    const long long* __restrict__ pairOffset,
                                                    int* __restrict__ pairs) {
    const int lane = threadIdx.x & 31;
    const int gw = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
    const int zs = gw % CELL_SPLIT;
    int a = gw / CELL_SPLIT;
    int wi = 0;
    while (wi < numItems && a >= items[wi].nA) { a -= items[wi].nA; wi++; }
    pdlEnter();
    if (blockIdx.x == 0)   // the binning of this step is complete: clear its counts for the next one
        for (int i = 0; i < numItems; i++)
            for (int k = threadIdx.x; k < CELL_MAX; k += blockDim.x) items[i].counts[k] = 0;
    const bool live = wi < numItems;   // warp-uniform
    if (!live && EMIT != 0) return;   // (the EMIT passes have no CTA barrier)
    if (!live) { wi = 0; a = 0; }     // evaluates nothing, joins the CTA's CN reduction
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
    // |FP32 r^2 - FP64 r^2| stays far below this margin (the FP32 rounding of a
    // difference and its image is ~1e-7 L per component)
    const double margin = rc2 * 1e-3 + 1e-6 * Lm * Lm;
    const float sureIn = (float)(rc2 - margin), sureOut = (float)(rc2 + margin);
    const float ir0f = 1.0f / it.r0;
    // CN and A-gradient sums in 64-bit fixed point (value * 2^32): exact, so
    // independent of the candidate order
    long long cnq = 0, gqx = 0, gqy = 0, gqz = 0;
    int found = 0;
    long long out = EMIT == 2 ? pairOffset[gw] : 0;
    const bool sliceLive = live && (nz >= 3 || zs == 0);
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
                    float ex = 0.f, ey = 0.f, ez = 0.f, x2e = 0.f;   // the pair's scaled difference and x^2
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
                        const float r2f = fmaf(uz, uz, fmaf(uy, uy, ux * ux));
                        if (r2f < sureIn && r2f > 1e-10f) {
                            // inside beyond any rounding: the FP64 decision is "in"
                            in = true;
                            ex = ux * ir0f; ey = uy * ir0f; ez = uz * ir0f;
                            x2e = r2f * (ir0f * ir0f);
                        } else if (r2f < sureOut) {
                            // near the cutoff (or the lower bound): the decision in FP64
                            D3 d = {__dsub_rn(A.x, (double)pb.x), __dsub_rn(A.y, (double)pb.y),
                                    __dsub_rn(A.z, (double)pb.z)};
                            if (periodic) d = cellImage(d, box);
                            const double r2 =
                                __dadd_rn(__dadd_rn(__dmul_rn(d.x, d.x), __dmul_rn(d.y, d.y)), __dmul_rn(d.z, d.z));
                            in = !(r2 < 1e-20) && r2 < rc2;
                            ex = (float)(d.x * ir0); ey = (float)(d.y * ir0); ez = (float)(d.z * ir0);
                            x2e = (float)(r2 * ir02);
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
                        const float sx = ex, sy = ey, sz = ez;
                        float f, h;
                        switchX2<NH>(x2e, true, K, f, h);
                        const long long qx = __float2ll_rn(h * sx * crun::FX);
                        const long long qy = __float2ll_rn(h * sy * crun::FX);
                        const long long qz = __float2ll_rn(h * sz * crun::FX);
                        cnq += __float2ll_rn(f * crun::FX);
                        gqx += qx; gqy += qy; gqz += qz;
                        unsigned long long* rb = acc + 3 * (size_t)(it.row0 + it.nA + it.sortedB[k]);
                        redAddI64(rb, -qx);
                        redAddI64(rb + 1, -qy);
                        redAddI64(rb + 2, -qz);
                    }
                }
            }
    if (EMIT == 1) {
        if (lane == 0) pairCount[gw] = found;
        return;
    }
    if (EMIT == 2) return;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        gqx += __shfl_xor_sync(0xffffffffu, gqx, o);
        gqy += __shfl_xor_sync(0xffffffffu, gqy, o);
        gqz += __shfl_xor_sync(0xffffffffu, gqz, o);
        cnq += __shfl_xor_sync(0xffffffffu, cnq, o);
    }
    __shared__ long long sCn[8];
    __shared__ int sItem[8];
    const int warp = threadIdx.x >> 5;
    if (lane == 0) {
        if (sliceLive) {
            unsigned long long* ra = acc + 3 * (size_t)(it.row0 + a);
            redAddI64(ra, gqx);
            redAddI64(ra + 1, gqy);
            redAddI64(ra + 2, gqz);
        }
        sCn[warp] = cnq;
        sItem[warp] = sliceLive ? wi : -1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        // one fixed-point CN addition per (CTA, item): integer, so order-independent
        long long run = 0;
        int cur = -1;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
            if (sItem[w] != cur) {
                if (cur >= 0) redAddI64(items[cur].cn, run);
                cur = sItem[w];
                run = 0;
            }
            run += sCn[w];
        }
        if (cur >= 0) redAddI64(items[cur].cn, run);
    }
}

template <int EMIT>
static void launchPairs(cudaStream_t s, int kind, int totalA, const CellItemDev* items, int numItems,
                        const int* slots, const float4* posq, const CellBox* box, unsigned long long* acc,
                        int* pairCount, const long long* pairOffset, int* pairs) {
    const dim3 grid((unsigned)((CELL_SPLIT * (long long)totalA * 32 + 255) / 256)), block(256);
    if (kind == 3)
        launchPdl(k_cell_pairs<3, EMIT>, grid, block, 0, s, items, numItems, slots, posq, box, acc, pairCount,
                  pairOffset, pairs);
    else if (kind == -1)
        launchPdl(k_cell_pairs<-1, EMIT>, grid, block, 0, s, items, numItems, slots, posq, box, acc,
                  pairCount, pairOffset, pairs);
    else
        launchPdl(k_cell_pairs<0, EMIT>, grid, block, 0, s, items, numItems, slots, posq, box, acc, pairCount,
                  pairOffset, pairs);
}

// maxB: the largest B group of the items
static void launchBin(cudaStream_t s, const CellItemDev* items, int numItems, int maxB, const int* slots,
                      const float4* posq, const CellBox* box) {
    const dim3 grid((unsigned)((std::max(1, maxB) + COUNT_THREADS - 1) / COUNT_THREADS), numItems);
    launchPdl(k_cell_count, grid, dim3(COUNT_THREADS), 0, s, items, slots, posq, box);
    launchPdl(k_cell_scan, dim3(numItems), dim3(CELL_MAX), 0, s, items);
    launchPdl(k_cell_scatter, grid, dim3(COUNT_THREADS), 0, s, items);
}

void launchCellCoord(cudaStream_t s, const CellItemDev* items, int numItems, int totalA, int maxB, int kind,
                     const int* slots,
                     const float4* posq, const CellBox* box, unsigned long long* acc) {
    if (numItems == 0 || totalA == 0) return;
    launchBin(s, items, numItems, maxB, slots, posq, box);
    launchPairs<0>(s, kind, totalA, items, numItems, slots, posq, box, acc, nullptr, nullptr, nullptr);
}

void launchCellPairList(cudaStream_t s, const CellItemDev* items, int numItems, int totalA, int maxB, int kind,
                        const int* slots,
                        const float4* posq, const CellBox* box, int* pairCount, const long long* pairOffset,
                        int* pairs, int pass) {
    if (numItems == 0 || totalA == 0) return;
    if (pass == 1) {
        launchBin(s, items, numItems, maxB, slots, posq, box);
        launchPairs<1>(s, kind, totalA, items, numItems, slots, posq, box, nullptr, pairCount, nullptr, nullptr);
    } else {
        launchPairs<2>(s, kind, totalA, items, numItems, slots, posq, box, nullptr, nullptr, pairOffset, pairs);
    }
}

}  // namespace glued
