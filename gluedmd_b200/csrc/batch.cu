// Batched multi-walker step: every walker's CVs, biases and force scatter in two
// launches per step, captured in one CUDA graph.
//
// The reference steps one OpenMM Context per walker and shares the bias through
// raw device pointers (tests/test_multiwalker.py:156-158,
// platforms/common/src/CommonGluedKernels.cpp:5234-5262). Here all walkers of a
// GPU are evaluated together:
//
//   1. Coordination runs (coord_run.cuh, launched through launchCoord): the
//      (A tile, B chunk) steps of every walker's coordination CVs, walker-major,
//      in equal static ranges over a persistent grid (SMs x resident CTAs);
//      gradients accumulate in 64-bit fixed point, CN partials per run piece.
//   2. k_batch_finalize, walkers x parts CTAs: each part clears and scatters its
//      share of the walker's coordination rows (dU/dCN needs only CN and the
//      harmonic terms: the hill bias acts on distance/angle/dihedral CVs) and
//      evaluates its share of the shared hill table for that walker; the last
//      part to finish sums the hill partials in part order and completes the
//      walker (harmonic terms, energy, the distance/angle/dihedral rows).
//
// Every reduction has a fixed order or is an integer sum, so a step is bitwise
// reproducible. Deposition (updateState at pace): one hill per walker, in walker
// order, with the well-tempered height from that walker's last hill-bias energy.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <string>

#include "batch.hpp"
#include "context.hpp"
#include "coord_run.cuh"
#include "kernels.hpp"

namespace glued {

namespace {
constexpr int MAXCV = 32;      // CV values per walker
constexpr int MAXSIMPLE = 16;  // distance/angle/dihedral CVs per walker
constexpr int MAXHARM = 32;    // harmonic terms per walker
constexpr int FT = 256;        // threads of a finalize CTA
constexpr int ROWS_PER_THREAD = 2;   // coordination rows one finalize thread scatters
constexpr int WBLK = 64;       // walkers per hill item (8 per warp)
constexpr int HC_MAX = 1024;   // hills per hill item, at most (shared-memory staging)
}  // namespace

struct BWalker {
    const float4* posq;
    unsigned long long* force;
    int padded;
    int n;
    BoxDev box;
};
struct BSimple { int type; int cv; int atoms[4]; };
struct BHarm { int cv; float k, at; int periodic; };
struct BHill {
    float4* mirror;
    double* centers;
    double* heights;
    int* count;
    int maxH, D, cv[2], pace, present;
    float a[2], isig2[2], period[2], iperiod[2];
    double h0, hif;
};

struct BatchDev {
    const BWalker* walkers;
    int W, nCV, nS, nC, nH;
    const BSimple* simple;  // [W][nS]
    const BHarm* harm;      // [W][nH]
    const CoordItem* items; // [W][nC]
    CoordRunDev R;          // coordination step runs over all walkers' items
    int rowsPerWalker;      // coordination rows of one walker (all its items)
    int parts;              // finalize CTAs per walker
    BHill hill;
    int nWB;                // walker blocks of <= WBLK walkers
    int hc;                 // hills per hill item (multiple of 32, <= HC_MAX)
    double* hillPart;       // [ceil(maxHills / hc)][W][3]
    double* cvv;            // [W][nCV]
    double* energy;         // [W]
    double* hillEnergy;     // [W]
    unsigned long long* stamps;   // profiling (nullptr = off): runs kernel [grid][4]
    unsigned long long* fstamps;  // profiling (nullptr = off): finalize kernel [W * parts][6]
};

__device__ __forceinline__ unsigned long long globalTimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ double harmonicDU(const BHarm& hm, double v, double& E) {
    const double TWO_PI = 6.283185307179586;
    double ds = v - (double)hm.at;
    if (hm.periodic) ds -= TWO_PI * round(ds / TWO_PI);
    E += 0.5 * (double)hm.k * ds * ds;
    return (double)hm.k * ds;
}

__device__ __forceinline__ void scatterRow(unsigned long long* F, int P, int atom, double g, float gx, float gy,
                                           float gz) {
    const double S = 4294967296.0;
    redAddGlobal(F + atom, (unsigned long long)(long long)(-(g * (double)gx) * S));
    redAddGlobal(F + atom + P, (unsigned long long)(long long)(-(g * (double)gy) * S));
    redAddGlobal(F + atom + 2 * P, (unsigned long long)(long long)(-(g * (double)gz) * S));
}

// ------------------------------------------------------------- hill items
// One item: hc consecutive hills of the shared table against the <= 64 walkers
// of one walker block. The walkers' hill-CV values are computed once per CTA
// (sS, one thread per walker and CV); the chunk is staged in shared memory by
// plain coalesced loads; warp w takes walkers w, w + 8, ...; lane l takes hills
// l, l + 32, ...; FP32 sums per lane, a fixed xor tree per walker, one partial
// per (item, walker), summed by the finalize in item order.
__device__ void hillCVs(const BatchDev& B, int wb, float* sS) {
    const int w0 = wb * WBLK, nw = min(WBLK, B.W - w0);
    const BHill& hb = B.hill;
    const int t = threadIdx.x;
    if (t < 2 * nw) {
        const int w = w0 + t / 2, d = t % 2;
        float v = 0.0f;
        if (d < hb.D) {
            const BWalker& wk = B.walkers[w];
            for (int s = 0; s < B.nS; s++) {
                const BSimple& si = B.simple[w * B.nS + s];
                if (si.cv == hb.cv[d]) v = simpleCV(si.type, si.atoms, wk.posq, nullptr, wk.box, nullptr);
            }
        }
        sS[t] = v;
    }
}

__device__ void hillItem(const BatchDev& B, int item, int itemsPerBlock, const float* sS, float4* sH) {
    const BHill& hb = B.hill;
    const int c = item % itemsPerBlock, wb = item / itemsPerBlock;
    const int w0 = wb * WBLK, nw = min(WBLK, B.W - w0);
    const int count = *hb.count;
    const int hc = B.hc;
    const int k0 = c * hc, n = max(0, min(hc, count - k0));
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    __syncthreads();  // sH free (previous item read), sS written
    for (int k = tid; k < hc; k += blockDim.x)
        sH[k] = k < n ? __ldg(hb.mirror + k0 + k) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    __syncthreads();
    for (int wl = warp; wl < nw; wl += 8) {
        const float s0 = sS[wl * 2], s1 = sS[wl * 2 + 1];
        float V = 0.0f, g0 = 0.0f, g1 = 0.0f;
#pragma unroll 4
        for (int q = 0; q < hc / 32; q++) {
            const float4 hk = sH[lane + 32 * q];   // height 0 past the end of the table
            float dx = s0 - hk.x, dy = s1 - hk.y;
            if (hb.period[0] > 0.0f) dx -= hb.period[0] * rintf(dx * hb.iperiod[0]);
            if (hb.period[1] > 0.0f) dy -= hb.period[1] * rintf(dy * hb.iperiod[1]);
            const float ex = dx * dx * hb.a[0] + dy * dy * hb.a[1];
            const float g = ex <= 8.0f ? hk.z * __expf(-ex) : 0.0f;
            V += g; g0 += g * dx; g1 += g * dy;
        }
        V = warpSumF(V); g0 = warpSumF(g0); g1 = warpSumF(g1);
        if (lane == 0) {
            double* out = B.hillPart + 3 * ((size_t)c * B.W + w0 + wl);
            out[0] = V;
            out[1] = -(double)g0 * hb.isig2[0];
            out[2] = -(double)g1 * hb.isig2[1];
        }
    }
}

// ------------------------------------------------------------- the runs
// Persistent CTAs (grid = SMs x resident CTAs): CTA b runs its static range of
// coordination steps, then its hill items b, b + grid, ... (ranges balanced so
// that CTAs with more hill items get fewer steps).
template <int RA, int BOX, int NH, bool HI>
__global__ void __launch_bounds__(256, 2) k_batch_runs(BatchDev B) {
    __shared__ CoordRunSmem<RA> sm;
    __shared__ float sS[WBLK * 2];
    const int numHill = B.hill.present ? ((*B.hill.count + B.hc - 1) / B.hc) * B.nWB : 0;
    int wbHave = -1;
    unsigned long long* st = B.stamps ? B.stamps + 4 * (size_t)blockIdx.x : nullptr;
    if (st && threadIdx.x == 0) st[0] = globalTimer();
    const int perBlock = numHill / max(B.nWB, 1);
    if ((int)blockIdx.x < numHill) {
        wbHave = blockIdx.x / perBlock;
        hillCVs(B, wbHave, sS);
    }
    if (st) { __syncthreads(); if (threadIdx.x == 0) st[1] = globalTimer(); }
    const int s0 = B.R.begin[blockIdx.x], s1 = B.R.begin[blockIdx.x + 1];
    if (s0 < s1) coordRun<RA, BOX, NH, HI>(B.R, s0, s1, sm, NoPieceHook());
    if (st) { __syncthreads(); if (threadIdx.x == 0) st[2] = globalTimer(); }
    float4* sH = reinterpret_cast<float4*>(&sm.g[0][0][0]);
    for (int item = blockIdx.x; item < numHill; item += gridDim.x) {
        const int wb = item / perBlock;
        if (wb != wbHave) {
            __syncthreads();
            hillCVs(B, wb, sS);
            wbHave = wb;
        }
        hillItem(B, item, perBlock, sS, sH);
    }
    if (st) { __syncthreads(); if (threadIdx.x == 0) st[3] = globalTimer(); }
}

// ------------------------------------------------------------- finalize
// CTA (walker w, part p) after the runs. Every part clears and scatters its share
// of the walker's coordination rows (at most ROWS_PER_THREAD per thread) with
// dU/dCN, which needs only CN (the walker's run-piece partials in step order)
// and the harmonic terms: the hill bias acts only on distance/angle/dihedral
// CVs. Part 0 also computes those CVs and their Jacobians, sums the hill
// partials in item order (fixed tree), evaluates the harmonic terms and the hill
// bias, writes CVs and energies and scatters the distance/angle/dihedral rows.
// Copies n bytes (multiple of 4) from global to shared memory, all threads.
__device__ __forceinline__ void copyWords(void* dst, const void* src, int n) {
    const int* s = static_cast<const int*>(src);
    int* d = static_cast<int*>(dst);
    for (int i = threadIdx.x; i < n / 4; i += blockDim.x) d[i] = __ldg(s + i);
}

constexpr int MAXCOORD = 8;   // coordination CVs per walker

__global__ void __launch_bounds__(FT) k_batch_finalize(BatchDev B) {
    __shared__ double sCV[MAXCV], sdU[MAXCV];
    __shared__ F3 sJac[MAXSIMPLE * 4];
    __shared__ double red[32 * 3];
    // the walker's record: one round of independent loads
    __shared__ BWalker sW;
    __shared__ BSimple sSimple[MAXSIMPLE];
    __shared__ BHarm sHarm[MAXHARM];
    __shared__ CoordItem sItem[MAXCOORD];
    const int w = blockIdx.x / B.parts, part = blockIdx.x % B.parts;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    unsigned long long* st = B.fstamps ? B.fstamps + 6 * (size_t)blockIdx.x : nullptr;
    if (st && tid == 0) st[0] = globalTimer();
    copyWords(&sW, B.walkers + w, sizeof(BWalker));
    copyWords(sSimple, B.simple + (size_t)w * B.nS, sizeof(BSimple) * B.nS);
    copyWords(sHarm, B.harm + (size_t)w * B.nH, sizeof(BHarm) * B.nH);
    copyWords(sItem, B.items + (size_t)w * B.nC, sizeof(CoordItem) * B.nC);
    if (tid < MAXCV) { sCV[tid] = 0.0; sdU[tid] = 0.0; }
    __syncthreads();
    if (st && tid == 0) st[1] = globalTimer();
    // part 0: distance/angle/dihedral values and Jacobians (positions: one round)
    if (part == 0 && tid < B.nS) {
        F3 jac[4];
        const float v = simpleCV(sSimple[tid].type, sSimple[tid].atoms, sW.posq, nullptr, sW.box, jac);
        for (int k = 0; k < 4; k++) sJac[tid * 4 + k] = jac[k];
        sCV[sSimple[tid].cv] = (double)v;
    }
    // the rows of this part: fixed-point sums (cleared as read) and their atoms
    const int r0 = (int)((long long)B.rowsPerWalker * part / B.parts);
    const int r1 = (int)((long long)B.rowsPerWalker * (part + 1) / B.parts);
    // (all loads first, so that they are in flight together; the rows are
    // cleared at the end of the kernel)
    long long vx[ROWS_PER_THREAD], vy[ROWS_PER_THREAD], vz[ROWS_PER_THREAD];
    int rItem[ROWS_PER_THREAD], rAtom[ROWS_PER_THREAD], rRow[ROWS_PER_THREAD];
#pragma unroll
    for (int q = 0; q < ROWS_PER_THREAD; q++) {
        const int r = r0 + tid + FT * q;
        rItem[q] = -1; rAtom[q] = 0; rRow[q] = 0;
        vx[q] = vy[q] = vz[q] = 0;
        if (r < r1) {
            // the walker's rows: item 0's A and B rows, then item 1's, ...
            int c = 0, base = 0;
            while (c < B.nC - 1 && r >= base + sItem[c].nA + sItem[c].nB) {
                base += sItem[c].nA + sItem[c].nB;
                c++;
            }
            const CoordItem& it = sItem[c];
            const int i = r - base;
            rRow[q] = it.row0 + i;
            const unsigned long long* a = B.R.acc + 3 * (size_t)rRow[q];
            vx[q] = (long long)__ldcg(a); vy[q] = (long long)__ldcg(a + 1); vz[q] = (long long)__ldcg(a + 2);
            rItem[q] = c;
            rAtom[q] = __ldg(B.R.slots + (i < it.nA ? it.a0 + i : it.b0 + (i - it.nA)));
        }
    }
    // CN: warp c sums item c's piece partials (lane l: pieces l, l + 32, ..., step
    // order), fixed xor tree
    if (warp < B.nC) {
        double t = 0.0;
        for (int k = sItem[warp].pieceBegin + lane; k < sItem[warp].pieceEnd; k += 32) t += __ldcg(B.R.cnPiece + k);
        t = warpSum(t);
        if (lane == 0) sCV[sItem[warp].cv] = t;
    }
    if (st) { __syncthreads(); if (tid == 0) st[2] = globalTimer(); }
    double hv[3] = {0.0, 0.0, 0.0};
    if (part == 0 && B.hill.present) {
        const int items = (*B.hill.count + B.hc - 1) / B.hc;
        for (int c = tid; c < items; c += FT) {
            const double* q = B.hillPart + 3 * ((size_t)c * B.W + w);
            hv[0] += __ldcg(q); hv[1] += __ldcg(q + 1); hv[2] += __ldcg(q + 2);
        }
    }
    if (part == 0) blockSum<3>(hv, red);   // part-uniform: every thread of part 0 takes part
    else __syncthreads();
    if (st && tid == 0) st[3] = globalTimer();
    // dU/dCV: part 0 everything, the other parts the coordination CVs only
    if (tid == 0) {
        double E = 0.0;
        for (int k = 0; k < B.nH; k++) {
            const BHarm& hm = sHarm[k];
            bool coordCv = false;
            for (int c = 0; c < B.nC; c++) coordCv = coordCv || sItem[c].cv == hm.cv;
            if (part == 0 || coordCv) sdU[hm.cv] += harmonicDU(hm, sCV[hm.cv], E);
        }
        if (part == 0) {
            if (B.hill.present) {
                E += hv[0];
                sdU[B.hill.cv[0]] += hv[1];
                if (B.hill.D > 1) sdU[B.hill.cv[1]] += hv[2];
            }
            for (int k = 0; k < B.nCV; k++) B.cvv[(size_t)w * B.nCV + k] = sCV[k];
            B.energy[w] = E;
            B.hillEnergy[w] = B.hill.present ? hv[0] : 0.0;
        }
    }
    __syncthreads();
    if (st && tid == 0) st[4] = globalTimer();
    unsigned long long* F = sW.force;
    const int P = sW.padded;
#pragma unroll
    for (int q = 0; q < ROWS_PER_THREAD; q++) {
        if (rItem[q] < 0) continue;
        const CoordItem& it = sItem[rItem[q]];
        const double g = sdU[it.cv];
        if (g == 0.0) continue;
        const double sc = coordAccScale(it) * crun::IFXD;
        scatterRow(F, P, rAtom[q], g, (float)((double)vx[q] * sc), (float)((double)vy[q] * sc),
                   (float)((double)vz[q] * sc));
    }
    if (part == 0 && tid < B.nS * 4) {
        const BSimple& si = sSimple[tid / 4];
        const int k = tid % 4;
        const int na = si.type == 1 ? 2 : si.type == 2 ? 3 : 4;
        const double g = sdU[si.cv];
        if (k < na && g != 0.0) {
            const F3 j = sJac[tid];
            scatterRow(F, P, si.atoms[k], g, j.x, j.y, j.z);
        }
    }
    // clear the rows for the next step's runs
#pragma unroll
    for (int q = 0; q < ROWS_PER_THREAD; q++) {
        if (rItem[q] < 0) continue;
        unsigned long long* a = B.R.acc + 3 * (size_t)rRow[q];
        a[0] = 0ull; a[1] = 0ull; a[2] = 0ull;
    }
    if (st) { __syncthreads(); if (tid == 0) st[5] = globalTimer(); }
}

typedef void (*RunsFn)(BatchDev);

template <int NH>
RunsFn runsKernelB(int box, bool hi) {
    if (box == 0) return k_batch_runs<8, 0, NH, true>;
    if (box == 1) return hi ? k_batch_runs<8, 1, NH, true> : k_batch_runs<8, 1, NH, false>;
    return hi ? k_batch_runs<8, 2, NH, true> : k_batch_runs<8, 2, NH, false>;
}

RunsFn runsKernel(int box, int kind, bool hi) {
    return kind == 3 ? runsKernelB<3>(box, hi) : kind == -1 ? runsKernelB<-1>(box, true) : runsKernelB<0>(box, true);
}

__global__ void k_batch_deposit(BatchDev B) {
    // one hill per walker, walker order; height from the walker's last hill energy
    const BHill& hb = B.hill;
    __shared__ int sN;
    if (threadIdx.x == 0) sN = *hb.count;
    __syncthreads();
    const int n0 = sN;
    for (int w = threadIdx.x; w < B.W; w += blockDim.x) {
        const int k = n0 + w;
        if (k >= hb.maxH) continue;
        double h = hb.hif > 0.0 ? hb.h0 * exp(-B.hillEnergy[w] * hb.hif) : hb.h0;
        double c[2] = {0.0, 0.0};
        for (int d = 0; d < hb.D; d++) c[d] = B.cvv[(size_t)w * B.nCV + hb.cv[d]];
        for (int d = 0; d < hb.D; d++) hb.centers[(size_t)k * hb.D + d] = c[d];
        hb.heights[k] = h;
        hb.mirror[k] = make_float4((float)c[0], (float)c[1], (float)h, 0.0f);
    }
    __syncthreads();
    if (threadIdx.x == 0) *hb.count = min(hb.maxH, n0 + B.W);
}

// ================================================================== host
struct Batch::Impl {
    int W = 0, nCV = 0, nS = 0, nC = 0, nH = 0, boxKind = 1, kind = 3;
    std::vector<BWalker> walkersH;
    std::vector<CoordItem> items;
    std::vector<int> coordAtoms;
    std::vector<CoordStep> steps;
    DBuf walkersD, simpleD, harmD, itemsD, atomsD, stepsD, beginD, boxesD, sysPosqD, acc, cnPiece;
    DBuf hillPart, cvv, energy, hillEnergy, status, scratchForce;
    DBuf hMirror, hCenters, hHeights, hCount;
    BHill hill{};
    BatchTuning tune;
    BatchDev dev{};
    int grid = 0;        // coordination runs: SMs x resident CTAs
    int rows = 0;        // coordination rows of one walker
    int parts = 1;       // finalize CTAs per walker
    int nWB = 1;         // walker blocks of the hill items
    int hillCountHost = 0;   // host mirror of the hill count (set_hills + deposits)
    int balancedItems = -1;  // hill items the current ranges were balanced for
    bool hi = true;
    cudaStream_t stream = 0;
    cudaStream_t cap = nullptr;
    cudaGraphExec_t graph = nullptr;
    long long launches = 0;
    int lastUpdateStep = -1;
    bool ready = false;
    float lastMs = 0;

    void destroyGraph() {
        if (graph) { cudaGraphExecDestroy(graph); graph = nullptr; }
    }

    RunsFn runs() const { return runsKernel(boxKind, kind, hi); }
    int hcHill() const { return tune.hillChunk > 0 ? tune.hillChunk : 512; }

    // Per-CTA step ranges: CTA b also evaluates hill items b, b + grid, ...,
    // charged hillWeightPct percent of a step each; run pieces to match. The
    // device copies are rewritten in place (a captured graph keeps their
    // addresses) unless they must grow.
    void balance() {
        const int nItems = hill.present ? ((hillCountHost + hcHill() - 1) / hcHill()) * ((W + WBLK - 1) / WBLK) : 0;
        std::vector<double> pre(grid, 0.0);
        for (int h = 0; h < nItems; h++) pre[h % grid] += tune.hillWeightPct / 100.0;
        std::vector<int> begin = balanceRanges((int)steps.size(), grid, pre);
        const int pieces = buildCoordPieces(steps, begin, items);
        auto put = [&](DBuf& d, const void* src, size_t bytes) {
            if (d.bytes < bytes) { d.alloc(bytes); destroyGraph(); }
            if (bytes) cudaCheck(cudaMemcpy(d.p, src, bytes, cudaMemcpyHostToDevice), "ranges");
        };
        put(beginD, begin.data(), sizeof(int) * begin.size());
        put(stepsD, steps.data(), sizeof(CoordStep) * steps.size());
        put(itemsD, items.data(), sizeof(CoordItem) * items.size());
        if (cnPiece.bytes < sizeof(double) * std::max(1, pieces)) {
            cnPiece.alloc(sizeof(double) * std::max(1, pieces));
            destroyGraph();
        }
        balancedItems = nItems;
        dev.R.begin = beginD.as<int>();
        dev.R.steps = stepsD.as<CoordStep>();
        dev.R.items = itemsD.as<CoordItem>();
        dev.items = itemsD.as<CoordItem>();
        dev.R.cnPiece = cnPiece.as<double>();
    }

    int minParts() const { return std::max(1, (rows + FT * ROWS_PER_THREAD - 1) / (FT * ROWS_PER_THREAD)); }

    void plan() {
        // coordination steps over all walkers' items (walker-major)
        buildCoordSteps(items, 8, steps);
        rows = 0;
        for (int c = 0; c < nC; c++) rows += items[c].nA + items[c].nB;
        std::vector<const float4*> posqOf(W);
        for (int w = 0; w < W; w++) posqOf[w] = walkersH[w].posq;
        sysPosqD.upload(posqOf);
        itemsD.alloc(sizeof(CoordItem) * std::max((size_t)1, items.size()));
        stepsD.alloc(sizeof(CoordStep) * std::max((size_t)1, steps.size()));
        const size_t accRows = (size_t)std::max(1, rows) * W;
        if (acc.bytes < sizeof(unsigned long long) * 3 * accRows) acc.alloc(sizeof(unsigned long long) * 3 * accRows);
        cudaCheck(cudaMemset(acc.p, 0, acc.bytes), "reset");
        std::vector<BoxDev> boxes(W);
        for (int w = 0; w < W; w++) boxes[w] = walkersH[w].box;
        boxesD.upload(boxes);
        hi = false;
        for (int w = 0; w < W && nC > 0; w++) {
            const BoxDev& b = walkersH[w].box;
            double box9[9] = {b.a[0], b.a[1], b.a[2], b.b[0], b.b[1], b.b[2], b.c[0], b.c[1], b.c[2]};
            std::vector<CoordItem> mine(items.begin() + w * nC, items.begin() + (w + 1) * nC);
            if (coordNeedsHi(mine, box9, boxKind != 0)) hi = true;
        }
        int dev_ = 0, sms = 0;
        cudaCheck(cudaGetDevice(&dev_), "device");
        cudaCheck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev_), "attr");
        cudaCheck(cudaFuncSetAttribute((const void*)runs(), cudaFuncAttributePreferredSharedMemoryCarveout,
                                       (int)cudaSharedmemCarveoutMaxShared), "carveout");
        int perSM = 0;
        cudaCheck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, (const void*)runs(), 256, 0), "occupancy");
        if (perSM < 1) throw Error(GLUED_E_CUDA, "batched runs kernel cannot be resident");
        grid = sms * perSM;
        balance();
        parts = tune.parts > 0 ? std::max(minParts(), tune.parts) : minParts();
        nWB = (W + WBLK - 1) / WBLK;
        if (hill.present) hillPart.alloc(sizeof(double) * 3 * (size_t)W * ((hill.maxH + hcHill() - 1) / hcHill()));
        dev.walkers = walkersD.as<BWalker>();
        dev.W = W; dev.nCV = nCV; dev.nS = nS; dev.nC = nC; dev.nH = nH;
        dev.simple = simpleD.as<BSimple>();
        dev.harm = harmD.as<BHarm>();
        dev.items = itemsD.as<CoordItem>();
        dev.R.items = itemsD.as<CoordItem>();
        dev.R.steps = stepsD.as<CoordStep>();
        dev.R.slots = atomsD.as<int>();
        dev.R.sysPosq = sysPosqD.as<const float4*>();
        dev.R.sysBox = boxesD.as<BoxDev>();
        dev.R.itemsPerSys = std::max(nC, 1);
        dev.R.acc = acc.as<unsigned long long>();
        dev.R.cnPiece = cnPiece.as<double>();
        dev.rowsPerWalker = rows;
        dev.parts = parts;
        dev.hill = hill;
        dev.hillPart = hillPart.as<double>();
        dev.nWB = nWB;
        dev.hc = hcHill();
        dev.cvv = cvv.as<double>(); dev.energy = energy.as<double>(); dev.hillEnergy = hillEnergy.as<double>();
        destroyGraph();
    }

    void launchRuns(cudaStream_t s) {
        void* args[] = {&dev};
        cudaCheck(cudaLaunchKernel((const void*)runs(), dim3(grid), dim3(256), args, 0, s), "runs");
    }
    void launchFinalize(cudaStream_t s) {
        void* args[] = {&dev};
        cudaCheck(cudaLaunchKernel((const void*)k_batch_finalize, dim3(W * parts), dim3(FT), args, 0, s), "finalize");
    }
    // The step's launches on stream s: coordination runs, then the finalize.
    void launch(cudaStream_t s) {
        launchRuns(s);
        launchFinalize(s);
        cudaCheck(cudaGetLastError(), "step launch");
    }
    int launchesPerStep() const { return 2; }
};

Batch::Batch(const std::vector<const GluedForce*>& forces, const glued_walker_desc* walkers) : impl_(new Impl()) {
    Impl& I = *impl_;
    I.W = (int)forces.size();
    if (I.W < 1) throw Error(GLUED_E_INVALID, "batch needs at least one walker");
    const GluedForce& f0 = *forces[0];
    I.nCV = f0.numCVValues();
    if (I.nCV > MAXCV) throw Error(GLUED_E_INVALID, "batch: at most 32 CV values per walker");
    // structure of walker 0; every walker must match it
    std::vector<int> types;
    for (auto& c : f0.cvs()) {
        if (c.type != CV_DISTANCE && c.type != CV_ANGLE && c.type != CV_DIHEDRAL && c.type != CV_COORDINATION &&
            c.type != CV_COORDINATION_CUTOFF)
            throw Error(GLUED_E_UNSUPPORTED, "batch: CV type " + std::to_string(c.type) +
                                                 " not supported (distance, angle, dihedral, coordination)");
        types.push_back(c.type);
        if (c.type <= CV_DIHEDRAL) I.nS++;
        else I.nC++;
    }
    if (I.nS > MAXSIMPLE) throw Error(GLUED_E_INVALID, "batch: at most 16 distance/angle/dihedral CVs per walker");
    if (I.nC > MAXCOORD) throw Error(GLUED_E_INVALID, "batch: at most 8 coordination CVs per walker");
    int hillBias = -1;
    for (int b = 0; b < f0.numBiases(); b++) {
        const BiasSpec& bs = f0.bias(b);
        if (bs.type == BIAS_HARMONIC) I.nH += (int)bs.cvs.size();
        else if (bs.type == BIAS_METAD_HILLS) {
            if (hillBias >= 0) throw Error(GLUED_E_UNSUPPORTED, "batch: at most one METAD_HILLS bias");
            hillBias = b;
        } else
            throw Error(GLUED_E_UNSUPPORTED, "batch: bias type " + std::to_string(bs.type) +
                                                 " not supported (HARMONIC, METAD_HILLS)");
    }
    if (I.nH > MAXHARM) throw Error(GLUED_E_INVALID, "batch: too many harmonic terms");
    std::vector<BSimple> simple;
    std::vector<BHarm> harm;
    for (int w = 0; w < I.W; w++) {
        const GluedForce& f = *forces[w];
        const glued_walker_desc& wd = walkers[w];
        if (f.numCVSpecs() != (int)types.size() || f.numBiases() != f0.numBiases())
            throw Error(GLUED_E_INVALID, "batch: walker " + std::to_string(w) + " has a different CV/bias structure");
        if (!wd.posq || !wd.force_buffer || wd.num_atoms < 1 || wd.padded_num_atoms < wd.num_atoms)
            throw Error(GLUED_E_INVALID, "batch: walker " + std::to_string(w) + " has invalid buffers");
        BWalker bw{};
        bw.posq = static_cast<const float4*>(wd.posq);
        bw.force = reinterpret_cast<unsigned long long*>(wd.force_buffer);
        bw.padded = wd.padded_num_atoms;
        bw.n = wd.num_atoms;
        const double* bx = wd.box;
        bool rect = bx[1] == 0 && bx[2] == 0 && bx[3] == 0 && bx[5] == 0 && bx[6] == 0 && bx[7] == 0;
        bool per = f0.usesPBC;
        for (int i = 0; i < 3; i++) { bw.box.a[i] = (float)bx[i]; bw.box.b[i] = (float)bx[3 + i]; bw.box.c[i] = (float)bx[6 + i]; }
        bw.box.inv[0] = (float)(1.0 / bx[0]); bw.box.inv[1] = (float)(1.0 / bx[4]); bw.box.inv[2] = (float)(1.0 / bx[8]);
        bw.box.kind = per ? (rect ? 1 : 2) : 0;
        if (w == 0) I.boxKind = bw.box.kind;
        else if (bw.box.kind != I.boxKind) throw Error(GLUED_E_INVALID, "batch: walkers must share the box kind");
        I.walkersH.push_back(bw);
        int slot = 0;
        for (int i = 0; i < f.numCVSpecs(); i++) {
            const CVSpec& c = f.cv(i);
            if (c.type != types[i]) throw Error(GLUED_E_INVALID, "batch: walker " + std::to_string(w) + " CV " + std::to_string(i) + " type differs");
            auto chk = [&](int a) {
                if (a < 0 || a >= wd.num_atoms) throw Error(GLUED_E_INVALID, "batch: walker " + std::to_string(w) + " atom index " + std::to_string(a) + " out of range");
            };
            if (c.type <= CV_DIHEDRAL) {
                BSimple s{};
                s.type = c.type; s.cv = slot;
                int na = c.type == CV_DISTANCE ? 2 : c.type == CV_ANGLE ? 3 : 4;
                if ((int)c.atoms.size() < na) throw Error(GLUED_E_INVALID, "batch: CV needs more atoms");
                for (int k = 0; k < na; k++) { chk(c.atoms[k]); s.atoms[k] = c.atoms[k]; }
                simple.push_back(s);
            } else {
                if (c.atoms.size() < 2 || c.atoms[0] < 1 || c.atoms[0] >= (int)c.atoms.size() || c.params.size() < 3)
                    throw Error(GLUED_E_INVALID, "batch: invalid coordination spec");
                CoordItem it{};
                it.cv = slot; it.nA = c.atoms[0]; it.nB = (int)c.atoms.size() - 1 - it.nA;
                it.a0 = (int)I.coordAtoms.size(); it.b0 = it.a0 + it.nA;
                for (size_t k = 1; k < c.atoms.size(); k++) { chk(c.atoms[k]); I.coordAtoms.push_back(c.atoms[k]); }
                it.r0 = (float)c.params[0]; it.n = (float)c.params[1]; it.m = (float)c.params[2];
                double rc = (c.type == CV_COORDINATION_CUTOFF && c.params.size() > 3) ? c.params[3] : 0.0;
                it.rc2 = (float)(rc * rc);
                it.kind = coordKind(it.n, it.m);
                I.items.push_back(it);
            }
            slot++;
        }
        int nh = 0;
        for (int b = 0; b < f.numBiases(); b++) {
            const BiasSpec& bs = f.bias(b);
            if (bs.type != f0.bias(b).type) throw Error(GLUED_E_INVALID, "batch: bias types differ between walkers");
            if (bs.type == BIAS_HARMONIC) {
                for (size_t d = 0; d < bs.cvs.size(); d++) {
                    if (bs.params.size() < 2 * (d + 1)) throw Error(GLUED_E_INVALID, "batch: harmonic needs [k, s0] per CV");
                    BHarm h{};
                    h.cv = bs.cvs[d]; h.k = (float)bs.params[2 * d]; h.at = (float)bs.params[2 * d + 1];
                    h.periodic = bs.iparams.empty() ? 0 : bs.iparams[0];
                    harm.push_back(h);
                    nh++;
                }
            }
        }
        if (nh != I.nH) throw Error(GLUED_E_INVALID, "batch: harmonic terms differ between walkers");
    }
    // group sizes must match across walkers (same tiling for every walker)
    for (int w = 1; w < I.W; w++)
        for (int c = 0; c < I.nC; c++)
            if (I.items[w * I.nC + c].nA != I.items[c].nA || I.items[w * I.nC + c].nB != I.items[c].nB ||
                I.items[w * I.nC + c].kind != I.items[c].kind)
                throw Error(GLUED_E_INVALID, "batch: coordination group sizes / exponents differ between walkers");
    // one switch kind per launch (the most general one present)
    if (!I.items.empty()) {
        I.kind = I.items[0].kind;
        for (auto& it : I.items)
            if (it.kind != I.kind) I.kind = (I.kind == 0 || it.kind == 0) ? 0 : -1;
        for (auto& it : I.items) it.kind = I.kind;
    }
    // shared hill bias from walker 0
    I.hill = BHill{};
    if (hillBias >= 0) {
        const BiasSpec& bs = f0.bias(hillBias);
        const int D = (int)bs.cvs.size();
        if (D > 2) throw Error(GLUED_E_UNSUPPORTED, "batch: METAD_HILLS on at most 2 CVs");
        if (bs.params.size() < (size_t)(3 + 3 * D) || bs.iparams.size() < (size_t)(2 + D))
            throw Error(GLUED_E_INVALID, "batch: METAD_HILLS parameters");
        for (int d = 0; d < D; d++) {
            bool simpleCvOk = false;
            for (auto& s : simple) if (s.cv == bs.cvs[d]) simpleCvOk = true;
            if (!simpleCvOk) throw Error(GLUED_E_UNSUPPORTED, "batch: METAD_HILLS must act on distance/angle/dihedral CVs");
        }
        BHill& h = I.hill;
        h.present = 1; h.D = D;
        h.h0 = bs.params[0];
        double gamma = bs.params[1 + D], kT = bs.params[2 + D];
        h.hif = gamma <= 1.0 ? 0.0 : 1.0 / ((gamma - 1.0) * kT);
        h.pace = bs.iparams[0];
        h.maxH = bs.iparams[1];
        for (int d = 0; d < 2; d++) {
            h.cv[d] = d < D ? bs.cvs[d] : 0;
            double sg = d < D ? bs.params[1 + d] : 1.0;
            h.a[d] = d < D ? (float)(1.0 / (2.0 * sg * sg)) : 0.0f;
            h.isig2[d] = d < D ? (float)(1.0 / (sg * sg)) : 0.0f;
            int per = d < D ? bs.iparams[2 + d] : 0;
            double L = d < D ? bs.params[3 + 2 * D + d] - bs.params[3 + D + d] : 0.0;
            h.period[d] = per ? (float)L : 0.0f;
            h.iperiod[d] = per ? (float)(1.0 / L) : 0.0f;
        }
        if (h.maxH < 1) throw Error(GLUED_E_INVALID, "batch: METAD_HILLS maxHills must be >= 1");
        I.hMirror.alloc(sizeof(float4) * (size_t)h.maxH);
        I.hCenters.alloc(sizeof(double) * (size_t)h.maxH * D);
        I.hHeights.alloc(sizeof(double) * (size_t)h.maxH);
        I.hCount.alloc(sizeof(int) * 4);
        h.mirror = I.hMirror.as<float4>(); h.centers = I.hCenters.as<double>();
        h.heights = I.hHeights.as<double>(); h.count = I.hCount.as<int>();
    }
    I.walkersD.upload(I.walkersH);
    I.simpleD.upload(simple);
    I.harmD.upload(harm);
    I.atomsD.upload(I.coordAtoms);
    I.cvv.alloc(sizeof(double) * (size_t)I.W * std::max(I.nCV, 1));
    I.energy.alloc(sizeof(double) * I.W);
    I.hillEnergy.alloc(sizeof(double) * I.W);
    I.status.alloc(sizeof(int) * 4);
    cudaCheck(cudaStreamCreateWithFlags(&I.cap, cudaStreamNonBlocking), "stream");
    I.plan();
}

Batch::~Batch() {
    if (impl_) {
        impl_->destroyGraph();
        if (impl_->cap) cudaStreamDestroy(impl_->cap);
        delete impl_;
    }
}

void Batch::setStream(cudaStream_t s) {
    impl_->stream = s;
}

void Batch::setTuning(const BatchTuning& t) {
    if (t.ra != 8) throw Error(GLUED_E_INVALID, "batch tuning: ra must be 8");
    if (t.parts < 0 || t.parts > 4096) throw Error(GLUED_E_INVALID, "batch tuning: finalize parts must be 0..4096");
    if (t.hillWeightPct < 0 || t.hillWeightPct > 10000)
        throw Error(GLUED_E_INVALID, "batch tuning: hill weight must be 0..10000 percent of a step");
    if (t.hillChunk != 0 && (t.hillChunk < 128 || t.hillChunk > HC_MAX || t.hillChunk % 128))
        throw Error(GLUED_E_INVALID, "batch tuning: hill chunk must be 0 or a multiple of 128 up to 1024");
    cudaCheck(cudaStreamSynchronize(impl_->stream), "sync");
    impl_->tune = t;
    impl_->plan();
}

BatchTuning Batch::tuning() const { return impl_->tune; }

void Batch::execute() {
    Impl& I = *impl_;
    if (!I.graph) {
        cudaGraph_t g = nullptr;
        cudaCheck(cudaStreamBeginCapture(I.cap, cudaStreamCaptureModeThreadLocal), "capture begin");
        try {
            I.launch(I.cap);
        } catch (...) {
            cudaStreamEndCapture(I.cap, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        cudaCheck(cudaStreamEndCapture(I.cap, &g), "capture end");
        cudaError_t ie = cudaGraphInstantiate(&I.graph, g, 0);
        cudaGraphDestroy(g);
        cudaCheck(ie, "graph instantiate");
    }
    cudaCheck(cudaGraphLaunch(I.graph, I.stream), "graph launch");
    I.launches += I.launchesPerStep();
    I.ready = true;
}

// Autotuner: finalize CTAs per walker and the weight of a hill item in the range
// balance are timed on the live walkers with CUDA events (forces go to a scratch
// buffer) and the fastest combination is kept.
BatchTuning Batch::autotune() {
    Impl& I = *impl_;
    cudaCheck(cudaStreamSynchronize(I.stream), "sync");
    size_t maxPad = 0;
    for (auto& w : I.walkersH) maxPad = std::max(maxPad, (size_t)w.padded);
    I.scratchForce.alloc(sizeof(long long) * 3 * maxPad);
    std::vector<BWalker> tmp = I.walkersH;
    for (auto& w : tmp) w.force = I.scratchForce.as<unsigned long long>();
    cudaCheck(cudaMemcpy(I.walkersD.p, tmp.data(), sizeof(BWalker) * tmp.size(), cudaMemcpyHostToDevice), "tune");
    cudaEvent_t a, b;
    cudaCheck(cudaEventCreate(&a), "event");
    cudaCheck(cudaEventCreate(&b), "event");
    BatchTuning best = I.tune;
    float bestMs = 1e30f;
    const BatchTuning saved = I.tune;
    const int base = I.minParts();
    for (int hc : {256, 512, 1024})
        for (int pct : {100, 150, 200, 300})
            for (int mul : {1, 2}) {
                if (!I.hill.present && (hc != 512 || pct != 150)) continue;
                BatchTuning t;
                t.ra = 8; t.parts = base * mul; t.hillWeightPct = pct; t.hillChunk = hc;
                I.tune = t;
                I.plan();
                for (int r = 0; r < 2; r++) I.launch(I.stream);
                cudaCheck(cudaEventRecord(a, I.stream), "event");
                const int reps = 8;
                for (int r = 0; r < reps; r++) I.launch(I.stream);
                cudaCheck(cudaEventRecord(b, I.stream), "event");
                cudaCheck(cudaEventSynchronize(b), "event");
                float ms = 0;
                cudaCheck(cudaEventElapsedTime(&ms, a, b), "event");
                ms /= reps;
                I.launches += (long long)(reps + 2) * I.launchesPerStep();
                if (ms < bestMs) { bestMs = ms; best = t; }
            }
    (void)saved;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaCheck(cudaMemcpy(I.walkersD.p, I.walkersH.data(), sizeof(BWalker) * I.walkersH.size(), cudaMemcpyHostToDevice), "tune");
    I.tune = best;
    I.plan();
    I.lastMs = bestMs;
    int st = status();
    if (st) throw Error(GLUED_E_TIMEOUT, "batch: bounded wait gave up during autotuning (status " + std::to_string(st) + ")");
    return best;
}

// One regular step launched without the graph, with every CTA recording
// %globaltimer at entry, end of phase A, barrier exit and exit, and how many
// coordination / hill items it processed. out[0..7]: phase-A end (earliest,
// latest CTA), barrier exit (latest), exit (latest) in microseconds after the
// earliest entry; coordination items, hill items, most and fewest items per CTA.
// Percentile p (0..100) of v (sorted in place).
static double pct(std::vector<double>& v, double p) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    size_t i = (size_t)std::min((double)v.size() - 1, std::floor(p / 100.0 * (double)(v.size() - 1) + 0.5));
    return v[i];
}

void Batch::phaseTimes(double* out) {
    Impl& I = *impl_;
    const int fg = I.W * I.parts;
    DBuf st;
    st.alloc(sizeof(unsigned long long) * (4 * (size_t)I.grid + 6 * (size_t)fg));
    cudaCheck(cudaMemsetAsync(st.p, 0, st.bytes, I.stream), "stamps");
    I.dev.stamps = st.as<unsigned long long>();
    I.dev.fstamps = st.as<unsigned long long>() + 4 * (size_t)I.grid;
    cudaEvent_t e[3];
    for (auto& x : e) cudaCheck(cudaEventCreate(&x), "event");
    cudaCheck(cudaEventRecord(e[0], I.stream), "event");
    I.launchRuns(I.stream);
    cudaCheck(cudaEventRecord(e[1], I.stream), "event");
    I.launchFinalize(I.stream);
    cudaCheck(cudaEventRecord(e[2], I.stream), "event");
    I.dev.stamps = nullptr;
    I.dev.fstamps = nullptr;
    cudaCheck(cudaEventSynchronize(e[2]), "event");
    float a = 0, b = 0;
    cudaCheck(cudaEventElapsedTime(&a, e[0], e[1]), "event");
    cudaCheck(cudaEventElapsedTime(&b, e[1], e[2]), "event");
    for (auto& x : e) cudaEventDestroy(x);
    I.launches += I.launchesPerStep();
    I.ready = true;
    std::vector<unsigned long long> h(st.bytes / sizeof(unsigned long long));
    cudaCheck(cudaMemcpy(h.data(), st.p, st.bytes, cudaMemcpyDeviceToHost), "stamps");
    unsigned long long t0 = ~0ull, f0 = ~0ull;
    for (int g = 0; g < I.grid; g++) t0 = std::min(t0, h[4 * (size_t)g]);
    for (int g = 0; g < fg; g++) f0 = std::min(f0, h[4 * (size_t)I.grid + 6 * (size_t)g]);
    std::vector<double> cvs, coord, end, fdur, fend, fph[5];
    for (int g = 0; g < I.grid; g++) {
        const unsigned long long* r = h.data() + 4 * (size_t)g;
        cvs.push_back((r[1] - r[0]) * 1e-3);
        coord.push_back((r[2] - t0) * 1e-3);
        end.push_back((r[3] - t0) * 1e-3);
    }
    for (int g = 0; g < fg; g++) {
        const unsigned long long* r = h.data() + 4 * (size_t)I.grid + 6 * (size_t)g;
        fdur.push_back((r[5] - r[0]) * 1e-3);
        fend.push_back((r[5] - f0) * 1e-3);
        for (int k = 0; k < 5; k++) fph[k].push_back((r[k + 1] - r[k]) * 1e-3);
    }
    out[0] = a * 1e3; out[1] = b * 1e3;
    out[2] = pct(cvs, 50); out[3] = pct(cvs, 100);
    out[4] = pct(coord, 0); out[5] = pct(coord, 50); out[6] = pct(coord, 100);
    out[7] = pct(end, 50); out[8] = pct(end, 100);
    out[9] = pct(fdur, 50); out[10] = pct(fdur, 100); out[11] = pct(fend, 100);
    for (int k = 0; k < 5; k++) out[16 + k] = pct(fph[k], 50);
    out[12] = (double)I.steps.size(); out[13] = (double)I.grid; out[14] = (double)I.parts; out[15] = (double)fg;
}

void Batch::updateState(int step) {
    Impl& I = *impl_;
    if (!I.ready || step == I.lastUpdateStep) return;
    if (!I.hill.present) return;
    I.lastUpdateStep = step;
    if (step == 0 || step % I.hill.pace != 0) return;
    k_batch_deposit<<<1, 256, 0, I.stream>>>(I.dev);
    cudaCheck(cudaGetLastError(), "deposit");
    I.launches++;
    I.hillCountHost = std::min(I.hill.maxH, I.hillCountHost + I.W);
    const int nItems = ((I.hillCountHost + I.hcHill() - 1) / I.hcHill()) * ((I.W + WBLK - 1) / WBLK);
    if (nItems != I.balancedItems) I.balance();
}

void Batch::energies(double* out) {
    cudaCheck(cudaStreamSynchronize(impl_->stream), "sync");
    cudaCheck(cudaMemcpy(out, impl_->energy.p, sizeof(double) * impl_->W, cudaMemcpyDeviceToHost), "energies");
}

void Batch::cvValues(double* out) {
    cudaCheck(cudaStreamSynchronize(impl_->stream), "sync");
    cudaCheck(cudaMemcpy(out, impl_->cvv.p, sizeof(double) * (size_t)impl_->W * impl_->nCV, cudaMemcpyDeviceToHost), "cvs");
}

int Batch::numCVs() const { return impl_->nCV; }
int Batch::numWalkers() const { return impl_->W; }

int Batch::numHills() {
    if (!impl_->hill.present) return 0;
    cudaCheck(cudaStreamSynchronize(impl_->stream), "sync");
    int n = 0;
    cudaCheck(cudaMemcpy(&n, impl_->hill.count, sizeof(int), cudaMemcpyDeviceToHost), "hills");
    return n;
}

void Batch::setHills(const double* centers, const double* heights, int n) {
    Impl& I = *impl_;
    if (!I.hill.present) throw Error(GLUED_E_STATE, "batch has no METAD_HILLS bias");
    if (n < 0 || n > I.hill.maxH) throw Error(GLUED_E_INVALID, "batch: hill count out of range");
    cudaCheck(cudaStreamSynchronize(I.stream), "sync");
    const int D = I.hill.D;
    std::vector<float4> m(n);
    for (int k = 0; k < n; k++)
        m[k] = make_float4((float)centers[k * D], D > 1 ? (float)centers[k * D + 1] : 0.0f, (float)heights[k], 0.0f);
    if (n > 0) {
        cudaCheck(cudaMemcpy(I.hill.centers, centers, sizeof(double) * (size_t)n * D, cudaMemcpyHostToDevice), "hills");
        cudaCheck(cudaMemcpy(I.hill.heights, heights, sizeof(double) * n, cudaMemcpyHostToDevice), "hills");
        cudaCheck(cudaMemcpy(I.hill.mirror, m.data(), sizeof(float4) * n, cudaMemcpyHostToDevice), "hills");
    }
    cudaCheck(cudaMemcpy(I.hill.count, &n, sizeof(int), cudaMemcpyHostToDevice), "hills");
    I.hillCountHost = n;
    I.balance();
}

void Batch::getHills(double* centers, double* heights, int n) {
    Impl& I = *impl_;
    int have = numHills();
    if (n > have) throw Error(GLUED_E_INVALID, "batch: fewer hills than requested");
    if (n > 0) {
        cudaCheck(cudaMemcpy(centers, I.hill.centers, sizeof(double) * (size_t)n * I.hill.D, cudaMemcpyDeviceToHost), "hills");
        cudaCheck(cudaMemcpy(heights, I.hill.heights, sizeof(double) * n, cudaMemcpyDeviceToHost), "hills");
    }
}

int Batch::status() {
    cudaCheck(cudaStreamSynchronize(impl_->stream), "sync");
    int s = 0;
    cudaCheck(cudaMemcpy(&s, impl_->status.p, sizeof(int), cudaMemcpyDeviceToHost), "status");
    return s;
}

long long Batch::launchCount() const { return impl_->launches; }
bool Batch::graphed() const { return impl_->graph != nullptr; }

double Batch::lastStepMs() { return impl_->lastMs; }

}  // namespace glued
