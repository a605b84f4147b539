// Coordination number CV (CommonGluedKernels.cpp:899-1031): all ng1 x ng2
// minimum-image pairs of the rational switch f = (1 - x^n) / (1 - x^m), x = r/r0.
//
// The reference evaluates every pair of a CV in one GPU thread. Here the pairs
// of every coordination CV of the context are one list of (A tile, B chunk)
// steps spread evenly over a persistent grid (coord_run.cuh):
//   - one 16-warp CTA per SM; warp w holds A atoms {w, w+16, ...} of the tile in
//     registers (all lanes share them), lane l takes B atoms {l, l+32, l+64,
//     l+96} of each chunk,
//   - per-pair force factor h = (df/dx)/x in units of r0; A sums over lanes at
//     the end of a tile's run, B sums over the 16 warps per chunk, both added as
//     64-bit fixed point (bitwise reproducible, independent of the grid),
//   - k_coord_finalize converts the sums to the float Jacobian rows and the CN
//     values and clears the accumulators for the next evaluation.
//
// Switch kinds:
//   k > 0 : m == 2n with n == 2k:  f = 1/(1 + x^n),  h = -n x^(n-2) f^2 (times 1/r0),
//           no square root and no pow;
//   -1    : integer n, m (1..64):   f = S_n(x) / S_m(x),  S_k(x) = sum_{j<k} x^j,
//           the same rational function without the cancellation of
//           (1 - x^n)/(1 - x^m) near x = 1, which in FP32 costs up to ~1e-3
//           relative force error outside the reference's |x-1| < 1e-4 Taylor
//           window (CommonGluedKernels.cpp:983-1003);
//   0     : non-integer exponents: the reference formula (pow, Taylor branch).
#include <algorithm>
#include <map>
#include <mutex>
#include <set>
#include <utility>

#include "context.hpp"
#include "coord_run.cuh"
#include "kernels.hpp"
#include "pdl.cuh"

namespace glued {

// One CTA of COORD_NW warps per SM: its warps meet at a barrier every step, so
// none of them runs ahead; buffers in dynamic shared memory (above the 48 KB
// static limit).
template <int RA, int BOX, int NH, bool HI, bool BLK>
__global__ void __launch_bounds__(COORD_NW * 32, 1) k_coord_run(CoordRunDev R) {
    pdlEnter();
    extern __shared__ __align__(16) unsigned char dsm[];
    CoordRunSmem<RA, COORD_CH / 32>& sm = *reinterpret_cast<CoordRunSmem<RA, COORD_CH / 32>*>(dsm);
    const int s0 = coordRange(R.numSteps, gridDim.x, blockIdx.x), s1 = coordRange(R.numSteps, gridDim.x, blockIdx.x + 1);
    if (s0 < s1) coordRun<RA, COORD_CH / 32, BOX, NH, HI, BLK>(R, s0, s1, sm, NoPieceHook());
}

// Fixed-point sums -> float Jacobian rows (one thread per row and component),
// every accumulator read is cleared; CN values = sums of the run pieces' partials
// in step order. The item of each row comes from the item table, written when
// the plan is built, and is looked up before the wait.
__global__ void k_coord_finalize(CoordRunDev R, int numItems, JacDev J, double* __restrict__ cvv, int totalRows) {
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    int ii = 0, base = 0;
    if (gid < 3 * totalRows)
        while (ii < numItems - 1 && gid / 3 >= base + R.items[ii].nA + R.items[ii].nB) {
            base += R.items[ii].nA + R.items[ii].nB;
            ii++;
        }
    pdlEnter();
    if (gid < 3 * totalRows) {
        const int comp = gid % 3;
        const int row = gid / 3;
        const CoordItem& it = R.items[ii];
        unsigned long long* a = R.acc + 3 * (size_t)row + comp;
        const long long v = (long long)*a;
        *a = 0ull;
        float* out = comp == 0 ? J.gx : comp == 1 ? J.gy : J.gz;
        out[it.jac0 + (row - base)] = (float)((double)v * crun::IFXD * coordAccScale(it));
    }
    if (blockIdx.x == 0) {
        // CN of each item: thread t sums the item's pieces t, t + 256, ... (in
        // order), then the fixed block tree
        __shared__ double red[32];
        for (int i = 0; i < numItems; i++) {
            if (R.items[i].cells) {
                // cell-list item: one exact fixed-point sum
                if (threadIdx.x == 0) {
                    cvv[R.items[i].cv] = (double)(long long)R.cellCn[i] * crun::IFXD;
                    R.cellCn[i] = 0ull;
                }
                continue;
            }
            double t = 0.0;
            for (int k = R.items[i].pieceBegin + (int)threadIdx.x; k < R.items[i].pieceEnd; k += blockDim.x)
                t += R.cnPiece[k];
            double v[1] = {t};
            blockSum<1>(v, red);
            if (threadIdx.x == 0) cvv[R.items[i].cv] = v[0];
            __syncthreads();
        }
    }
}

// slots[k] = u2g[atoms[k]]: the posq row of every coordination atom, rebuilt
// whenever OpenMM reorders atoms.
__global__ void k_compose_slots(const int* __restrict__ atoms, const int* __restrict__ u2g, int* __restrict__ slots,
                                int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) slots[i] = u2g[atoms[i]];
}

void launchComposeSlots(cudaStream_t s, const int* atoms, const int* u2g, int* slots, int n) {
    if (n > 0) k_compose_slots<<<(n + 255) / 256, 256, 0, s>>>(atoms, u2g, slots, n);
}

// Per-step gather tables of the coordination runs (CoordRunDev::gB, gA) from the
// step list and the atoms' posq rows (slots), one thread per (step, lane of the
// chunk / tile); rebuilt whenever the rows change. A step gathers its tile's A
// atoms when it starts a tile run: the tile's first chunk, or the first step of
// a CTA's range in a grid of `grid` CTAs.
__global__ void k_step_gathers(const CoordStep* __restrict__ steps, int numSteps, int grid,
                               const int* __restrict__ slots, int* __restrict__ gB, int* __restrict__ gA, int ta,
                               int ch) {
    // one thread per (step, lane), lane < max(ta, ch)
    const int w = ta > ch ? ta : ch;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)numSteps * w) return;
    const int s = (int)(i / w), t = (int)(i % w);
    const CoordStep d = steps[s];
    const int nAv = stepNA(d.packed), nBv = stepNB(d.packed), fl = stepFlags(d.packed);
    if (t < ch) gB[(size_t)s * ch + t] = t < nBv ? slots[d.bStart + t] : -1;
    if (t < ta) {
        // smallest CTA whose range could start at s
        const long long b = ((long long)s * grid + numSteps - 1) / numSteps;
        const bool rangeStart = b < grid && coordRange(numSteps, grid, (int)b) == s;
        gA[(size_t)s * ta + t] = ((fl & COORD_F_FIRST) || rangeStart) ? (t < nAv ? slots[d.aStart + t] : -2) : -1;
    }
}

// Pair constants of every step (runConst of its item and system box), for runs
// whose items and boxes are fixed: the runs kernel then copies them with the
// step records instead of computing them from two more dependent loads.
__global__ void k_step_consts(const CoordStep* __restrict__ steps, int numSteps, const CoordItem* __restrict__ items,
                              const BoxDev* __restrict__ sysBox, RunConst* __restrict__ out) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < numSteps) out[s] = runConst(items[steps[s].item], sysBox[steps[s].sys]);
}

void launchStepConsts(cudaStream_t s, const CoordStep* steps, int numSteps, const CoordItem* items,
                      const BoxDev* sysBox, RunConst* out) {
    if (numSteps > 0) k_step_consts<<<(numSteps + 255) / 256, 256, 0, s>>>(steps, numSteps, items, sysBox, out);
}

size_t runConstBytes() { return sizeof(RunConst); }

void launchStepGathers(cudaStream_t s, const CoordStep* steps, int numSteps, int grid, const int* slots, int* gB,
                       int* gA, int ta, int ch) {
    const long long n = (long long)numSteps * (ta > ch ? ta : ch);
    if (n > 0) k_step_gathers<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(steps, numSteps, grid, slots, gB, gA, ta, ch);
}

// The dynamic shared-memory limit is a per-function maximum: it only ever grows
// (a smaller request after a larger one must not lower it under a batch that
// still launches with the larger size).
void runKernelSetup(const void* fn, size_t dynSmem) {
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, size_t> limit;
    int dev = 0;
    cudaCheck(cudaGetDevice(&dev), "device");
    std::lock_guard<std::mutex> lock(mu);
    auto it = limit.find({fn, dev});
    if (it != limit.end() && it->second >= dynSmem) return;
    cudaCheck(cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                                   (int)cudaSharedmemCarveoutMaxShared), "carveout");
    cudaCheck(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dynSmem), "smem");
    limit[{fn, dev}] = dynSmem;
}

template <int RA, int BOX, int NH, bool HI, bool BLK>
static void launchRun(cudaStream_t s, int grid, const CoordRunDev& R) {
    const size_t dyn = sizeof(CoordRunSmem<RA, COORD_CH / 32>);
    runKernelSetup((const void*)k_coord_run<RA, BOX, NH, HI, BLK>, dyn);
    // plain launch: the persistent grid fills every SM, nothing to overlap
    k_coord_run<RA, BOX, NH, HI, BLK><<<grid, COORD_NW * 32, dyn, s>>>(R);
}

template <int BOX, bool BLK>
static void launchRunB(cudaStream_t s, int grid, int kind, bool hi, const CoordRunDev& R) {
    if (kind == 3) {
        if (hi) launchRun<8, BOX, 3, true, BLK>(s, grid, R);
        else launchRun<8, BOX, 3, false, BLK>(s, grid, R);
    } else if (kind == -1) {
        launchRun<8, BOX, -1, true, BLK>(s, grid, R);
    } else {
        launchRun<8, BOX, 0, true, BLK>(s, grid, R);
    }
}

template <bool BLK>
static void launchRunK(cudaStream_t s, int grid, int boxKind, int kind, bool hi, const CoordRunDev& R) {
    if (boxKind == 0) launchRunB<0, BLK>(s, grid, kind, true, R);
    else if (boxKind == 1) launchRunB<1, BLK>(s, grid, kind, hi, R);
    else launchRunB<2, BLK>(s, grid, kind, hi, R);
}

void launchCoord(cudaStream_t s, const CoordRunDev& R, int numItems, int grid, int totalRows, int boxKind, int kind,
                 bool hi, const JacDev& J, double* cvv, int parts, bool blocked) {
    if (numItems == 0) return;
    if ((parts & 1) && R.numSteps > 0) {
        if (blocked) launchRunK<true>(s, grid, boxKind, kind, hi, R);
        else launchRunK<false>(s, grid, boxKind, kind, hi, R);
    }
    if (parts & 2) {
        const int n = std::max(3 * totalRows, numItems);
        launchPdl(k_coord_finalize, dim3((n + 255) / 256), dim3(256), 0, s, R, numItems, J, cvv, totalRows);
    }
}

int coordRunOccupancy(int kind, int boxKind, bool hi) {
    const void* fn;
    if (kind == 3) {
        fn = boxKind == 0 ? (const void*)k_coord_run<8, 0, 3, true, false>
             : boxKind == 1 ? (hi ? (const void*)k_coord_run<8, 1, 3, true, false> : (const void*)k_coord_run<8, 1, 3, false, false>)
                            : (hi ? (const void*)k_coord_run<8, 2, 3, true, false> : (const void*)k_coord_run<8, 2, 3, false, false>);
    } else if (kind == -1) {
        fn = boxKind == 0 ? (const void*)k_coord_run<8, 0, -1, true, false>
             : boxKind == 1 ? (const void*)k_coord_run<8, 1, -1, true, false> : (const void*)k_coord_run<8, 2, -1, true, false>;
    } else {
        fn = boxKind == 0 ? (const void*)k_coord_run<8, 0, 0, true, false>
             : boxKind == 1 ? (const void*)k_coord_run<8, 1, 0, true, false> : (const void*)k_coord_run<8, 2, 0, true, false>;
    }
    const size_t dyn = sizeof(CoordRunSmem<8, COORD_CH / 32>);
    runKernelSetup(fn, dyn);
    int perSM = 0;
    cudaCheck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, fn, COORD_NW * 32, dyn), "occupancy");
    return std::max(1, perSM);
}

}  // namespace glued
