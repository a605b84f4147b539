// Batched multi-walker step: every walker's CVs, biases and force scatter in two
// launches per step, captured in one CUDA graph.
//
// The reference steps one OpenMM Context per walker and shares the bias through
// raw device pointers (tests/test_multiwalker.py:156-158,
// platforms/common/src/CommonGluedKernels.cpp:5234-5262). Here all walkers of a
// GPU are evaluated together:
//
//   1. k_batch_runs, a persistent grid (SMs x resident CTAs): every CTA runs an
//      equal static range of the (A tile, B chunk) coordination steps of all
//      walkers (coord_run.cuh; gradients in 64-bit fixed point, CN partials per
//      run piece), then evaluates an equal slice of the shared hill table for
//      every walker (slice and hill-CV atoms staged in shared memory when the
//      CTA starts), one FP64 partial per (CTA, walker).
//   2. k_batch_finalize, walkers x parts CTAs: parts 1, 2, ... clear and scatter
//      their shares of the walker's coordination rows (dU/dCN needs only CN and
//      the harmonic terms: the hill bias acts on distance/angle/dihedral CVs);
//      part 0 sums the hill partials in CTA order and completes the walker
//      (harmonic terms, energy, the distance/angle/dihedral rows), and takes
//      the rows too only when it is the walker's one part.
//
// Every reduction has a fixed order or is an integer sum, so a step is bitwise
// reproducible. Deposition (updateState at pace): one hill per walker, in walker
// order, with the well-tempered height from that walker's last hill-bias energy.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
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
constexpr int RUNS_THREADS = COORD_NW * 32;   // threads of a runs CTA (one CTA per SM)
constexpr int WBLK = 64;       // walkers per hill pass
constexpr int JW = WBLK / COORD_NW;   // walker slots per warp in a hill pass
static_assert(JW * COORD_NW == WBLK && 3 * JW <= 32, "hill walker slots");
constexpr int HS = 512;        // hills staged in shared memory at a time (a slice of the
                               // 50,000-hill table over 148 CTAs is 338)
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
    float* mirror;      // [3][cap]: scaled x, scaled y, height of every hill
    int cap;            // maxH rounded up to a multiple of 4
    double* centers;
    double* heights;
    int* count;
    int maxH, D, cv[2], pace, present;
    // scaled units: s' = u s with u = sqrt(log2(e) / (2 sigma^2)) (0 for an
    // unused dimension); periods pS = u L (0: not periodic), ipS = 1 / pS;
    // a hill counts while dx'^2 + dy'^2 <= cut = 8 log2(e); dV/ds = gsc * sum g dx'
    float u[2], pS[2], ipS[2], gsc[2], cut;
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
    const float4* const* hillCvPos;  // [W][2][4] posq addresses of the hill CVs' atoms (nullptr: unused)
    const int* hillCvType;  // [W][2] CV type of hill dimension d (0: none)
    const int* rowAtom;     // [W * rowsPerWalker] atom of every coordination row
    double* hillPart;       // [hillParts][W][3]: hill sums of every runs CTA
    int hillParts;          // CTAs of the runs grid
    double* cvv;            // [W][nCV]
    double* energy;         // [W]
    double* hillEnergy;     // [W]
    int* status;                  // bit 0: a deposit found the hill table full
    unsigned long long* stamps;   // profiling (nullptr = off): runs kernel [grid][7] (6 times, SM id)
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

// ------------------------------------------------------------- hill slices
// Every CTA of the runs grid owns an equal contiguous slice of the shared hill
// table and evaluates it for all walkers after its coordination steps. Data
// movement stays off the critical path: the CTA's prologue copies (cp.async)
// the tables it needs first (hill count, posq addresses of the hill CVs' atoms,
// boxes of <= 64 walkers); when those have landed, before its first
// coordination step computes, it issues the gathers that depend on them (its
// slice of the table, HS hills at a time, and the atoms' positions), which land
// while that step computes. Arithmetic: CVs and hill centres are stored scaled
// by u = sqrt(log2(e) / (2 sigma^2)) per dimension (the mirror table holds
// scaled centres, as three arrays x, y, height), so a hill is
// exp2(-(dx^2 + dy^2)) of scaled differences; slices start on multiples of 4
// hills so that they move in 16-byte copies. Warp w takes walkers w, w + 16,
// ... (JW at a time in registers), lane l takes the hill pairs (2p, 2p+1),
// p = l, l + 32, ..., in packed FP32 (f32x2: two hills per instruction); FP32
// sums per lane, a fixed butterfly over the lanes, one FP64 partial per (CTA,
// walker), summed by the finalize in CTA order.
struct HillStage {
    float hx[HS], hy[HS], hh[HS];   // the staged chunk: scaled centres, heights
    float4 pos[WBLK * 8];
    BoxDev box[WBLK];
    const float4* ptr[WBLK * 8];
    int count[4];
    float sS[WBLK * 2];
};

// This CTA's hill groups (4 hills each) [g0, g1) of the table.
__device__ __forceinline__ void hillSliceRange(const BatchDev& B, const HillStage& hs, int& g0, int& g1) {
    const int groups = (hs.count[0] + 3) / 4;
    g0 = (int)((long long)groups * blockIdx.x / gridDim.x);
    g1 = (int)((long long)groups * (blockIdx.x + 1) / gridDim.x);
}

// Tables of walker block wb: count, atom addresses, boxes (no dependent loads).
__device__ void hillStageTables(const BatchDev& B, int wb, HillStage& hs) {
    const int w0 = wb * WBLK, nw = min(WBLK, B.W - w0);
    static_assert(sizeof(BoxDev) % 16 == 0, "box record");
    constexpr int BW = sizeof(BoxDev) / 16;
    const float4* ptrSrc = reinterpret_cast<const float4*>(B.hillCvPos + (size_t)w0 * 8);
    for (int t = threadIdx.x; t < nw * 4; t += blockDim.x)
        cpAsync16(reinterpret_cast<float4*>(hs.ptr) + t, ptrSrc + t, true);
    for (int t = threadIdx.x; t < nw * BW; t += blockDim.x)
        cpAsync16(reinterpret_cast<float4*>(&hs.box[t / BW]) + t % BW,
                  reinterpret_cast<const float4*>(B.R.sysBox + w0 + t / BW) + t % BW, true);
    if (threadIdx.x == 0) cpAsync16(hs.count, B.hill.count, true);
}

// Hill groups [c0, min(g1, c0 + HS / 4)) into the chunk arrays; the bytes past
// the table's count and the rest of the chunk are zero (height 0).
__device__ __forceinline__ void hillStageHills(const BatchDev& B, const HillStage& hs, int c0, int g1) {
    const int count = hs.count[0];
    const int ng = min(g1 - c0, HS / 4);
    for (int t = threadIdx.x; t < 3 * (HS / 4); t += blockDim.x) {
        const int c = t / (HS / 4), g = t % (HS / 4);
        const int k = 4 * (c0 + g);
        const int bytes = g < ng ? 4 * max(0, min(4, count - k)) : 0;
        const float* d = c == 0 ? hs.hx : c == 1 ? hs.hy : hs.hh;
        cpAsyncBytes(const_cast<float*>(d) + 4 * g, B.hill.mirror + (size_t)c * B.hill.cap + (bytes ? k : 0), bytes);
    }
}

// Gathers that depend on the tables (after they have landed): the first HS
// hills of the slice and the atoms' positions of walker block wb.
__device__ void hillStageData(const BatchDev& B, int wb, HillStage& hs) {
    const int w0 = wb * WBLK, nw = min(WBLK, B.W - w0);
    int g0, g1;
    hillSliceRange(B, hs, g0, g1);
    hillStageHills(B, hs, g0, g1);
    for (int t = threadIdx.x; t < nw * 8; t += blockDim.x) {
        const float4* a = hs.ptr[t];
        cpAsync16(&hs.pos[t], a ? a : reinterpret_cast<const float4*>(B.hill.mirror), a != nullptr);
    }
}

// Scaled hill-CV values of walker block wb from the staged positions.
__device__ void hillCVs(const BatchDev& B, int wb, HillStage& hs) {
    const int w0 = wb * WBLK, nw = min(WBLK, B.W - w0);
    const int t = threadIdx.x;
    if (t < 2 * nw) {
        const int type = B.hillCvType[(w0 + t / 2) * 2 + t % 2];
        float v = 0.0f;
        if (type) {
            F3 p[4];
            for (int k = 0; k < 4; k++) { const float4 q = hs.pos[t * 4 + k]; p[k] = f3(q.x, q.y, q.z); }
            v = simpleCVFromPos(type, p, hs.box[t / 2], nullptr);
        }
        hs.sS[t] = v * (t % 2 ? B.hill.u[1] : B.hill.u[0]);
    }
}

// The hill pairs p = lane, lane + 32, ... (< np) of the staged chunk against the
// JW walkers of this warp, two hills per packed instruction; acc[j][c]: packed
// partial sums of g, g dx, g dy for walker slot j.
// Packed two-sum: s + c gains b with the rounding error of the addition kept in c.
__device__ __forceinline__ void twoSum2(unsigned long long& s, unsigned long long& c, unsigned long long b) {
    const unsigned long long t = f2::add(s, b), bb = f2::sub(t, s);
    c = f2::add(c, f2::add(f2::sub(s, f2::sub(t, bb)), f2::sub(b, bb)));
    s = t;
}

template <bool P0, bool P1, bool COMP>
__device__ __forceinline__ void hillEval(const HillStage& hs, const BHill& hb, int np, const float (&s0)[JW],
                                         const float (&s1)[JW], unsigned long long (&acc)[JW][3],
                                         unsigned long long (&cmp)[JW][3]) {
    constexpr float R = 12582912.0f;   // 1.5 * 2^23: adding and removing it rounds to an integer
    const int lane = threadIdx.x & 31;
    const unsigned long long R2 = f2::pk(R, R);
    const unsigned long long ip0 = f2::pk(hb.ipS[0], hb.ipS[0]), np0 = f2::pk(-hb.pS[0], -hb.pS[0]);
    const unsigned long long ip1 = f2::pk(hb.ipS[1], hb.ipS[1]), np1 = f2::pk(-hb.pS[1], -hb.pS[1]);
    unsigned long long sx[JW], sy[JW];
#pragma unroll
    for (int j = 0; j < JW; j++) { sx[j] = f2::pk(s0[j], s0[j]); sy[j] = f2::pk(s1[j], s1[j]); }
    const unsigned long long* hx2 = reinterpret_cast<const unsigned long long*>(hs.hx);
    const unsigned long long* hy2 = reinterpret_cast<const unsigned long long*>(hs.hy);
    const unsigned long long* hh2 = reinterpret_cast<const unsigned long long*>(hs.hh);
    for (int p = lane; p < np; p += 32) {
        const unsigned long long hx = hx2[p], hy = hy2[p], hh = hh2[p];   // height 0 past the slice
#pragma unroll
        for (int j = 0; j < JW; j++) {
            unsigned long long dx = f2::sub(sx[j], hx), dy = f2::sub(sy[j], hy);
            if (P0) dx = f2::fma(f2::sub(f2::fma(dx, ip0, R2), R2), np0, dx);
            if (P1) dy = f2::fma(f2::sub(f2::fma(dy, ip1, R2), R2), np1, dy);
            const unsigned long long ex = f2::fma(dx, dx, f2::mul(dy, dy));
            float ea, eb, ga, gb;
            f2::upk(ex, ea, eb);
            asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(ga) : "f"(-ea));
            asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(gb) : "f"(-eb));
            ga = ea <= hb.cut ? ga : 0.0f;
            gb = eb <= hb.cut ? gb : 0.0f;
            const unsigned long long g = f2::mul(hh, f2::pk(ga, gb));
            if (COMP) {
                twoSum2(acc[j][0], cmp[j][0], g);
                twoSum2(acc[j][1], cmp[j][1], f2::mul(g, dx));
                twoSum2(acc[j][2], cmp[j][2], f2::mul(g, dy));
            } else {
                acc[j][0] = f2::add(acc[j][0], g);
                acc[j][1] = f2::fma(g, dx, acc[j][1]);
                acc[j][2] = f2::fma(g, dy, acc[j][2]);
            }
        }
    }
}

// warpTransposeSum32 with a two-sum at every addition: e[] holds the slots'
// compensation terms, which travel (and add up) with them; *err = the result's.
__device__ __forceinline__ float warpTransposeSum32C(float (&v)[32], float (&e)[32], float& err) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
        const bool up = (lane & o) != 0;
#pragma unroll
        for (int i = 0; i < o; i++) {
            const float sv = up ? v[i] : v[i + o], kv = up ? v[i + o] : v[i];
            const float se = up ? e[i] : e[i + o], ke = up ? e[i + o] : e[i];
            const float rv = __shfl_xor_sync(0xffffffffu, sv, o), re = __shfl_xor_sync(0xffffffffu, se, o);
            const float t = __fadd_rn(kv, rv), bb = __fsub_rn(t, kv);
            e[i] = __fadd_rn(__fadd_rn(ke, re), __fadd_rn(__fsub_rn(kv, __fsub_rn(t, bb)), __fsub_rn(rv, bb)));
            v[i] = t;
        }
    }
    err = e[0];
    return v[0];
}

// This CTA's hill slice for every walker. `gathered`: the data of walker block
// 0 was issued during the coordination steps. COMP: two-sum compensated sums
// (per lane, through the lane tree; the walker's value is hi + lo in FP64).
template <bool COMP>
__device__ void hillSlice(const BatchDev& B, HillStage& hs, bool gathered, bool cvsDone, unsigned long long* st) {
    const BHill& hb = B.hill;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nWB = (B.W + WBLK - 1) / WBLK;
    for (int wb = 0; wb < nWB; wb++) {
        const int w0 = wb * WBLK, nw = min(WBLK, B.W - w0);
        if (wb > 0) {
            __syncthreads();   // the previous block's data fully read
            hillStageTables(B, wb, hs);
            cpAsyncCommit();
        }
        if (wb > 0 || !gathered) {
            cpAsyncWaitAll();
            __syncthreads();
            hillStageData(B, wb, hs);
            cpAsyncCommit();
        }
        cpAsyncWaitAll();
        __syncthreads();
        if (st && wb == 0 && threadIdx.x == 0) st[3] = globalTimer();
        if (wb > 0 || !cvsDone) {
            hillCVs(B, wb, hs);
            __syncthreads();
        }
        int g0, g1;
        hillSliceRange(B, hs, g0, g1);
        float s0[JW], s1[JW];
#pragma unroll
        for (int j = 0; j < JW; j++) {
            const int wl = min(warp + COORD_NW * j, nw - 1);
            s0[j] = hs.sS[wl * 2]; s1[j] = hs.sS[wl * 2 + 1];
        }
        unsigned long long pacc[JW][3], pcmp[JW][3];   // pcmp: compensation terms (COMP only)
#pragma unroll
        for (int j = 0; j < JW; j++) {
            pacc[j][0] = pacc[j][1] = pacc[j][2] = 0ull;
            if (COMP) pcmp[j][0] = pcmp[j][1] = pcmp[j][2] = 0ull;
        }
        for (int c0 = g0; c0 < g1; c0 += HS / 4) {
            if (c0 != g0) {
                __syncthreads();
                hillStageHills(B, hs, c0, g1);
                cpAsyncCommit();
                cpAsyncWaitAll();
                __syncthreads();
            }
            const int np = 2 * min(g1 - c0, HS / 4);   // hill pairs staged
            const bool p0 = hb.pS[0] > 0.0f, p1 = hb.pS[1] > 0.0f;
            if (p0 && p1) hillEval<true, true, COMP>(hs, hb, np, s0, s1, pacc, pcmp);
            else if (p0) hillEval<true, false, COMP>(hs, hb, np, s0, s1, pacc, pcmp);
            else if (p1) hillEval<false, true, COMP>(hs, hb, np, s0, s1, pacc, pcmp);
            else hillEval<false, false, COMP>(hs, hb, np, s0, s1, pacc, pcmp);
        }
        if (st && wb == 0 && threadIdx.x == 0) st[4] = globalTimer();
        // lane 3 j + c: component c of walker slot j
        double v;
        if constexpr (COMP) {
            float acc[32], cme[32];
#pragma unroll
            for (int j = 0; j < JW; j++)
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    float a, b, ca, cb;
                    f2::upk(pacc[j][c], a, b);
                    f2::upk(pcmp[j][c], ca, cb);
                    const float t = __fadd_rn(a, b), bb = __fsub_rn(t, a);
                    acc[3 * j + c] = t;
                    cme[3 * j + c] = __fadd_rn(__fadd_rn(ca, cb), __fadd_rn(__fsub_rn(a, __fsub_rn(t, bb)),
                                                                             __fsub_rn(b, bb)));
                }
#pragma unroll
            for (int k = 3 * JW; k < 32; k++) acc[k] = cme[k] = 0.0f;
            float lo;
            const float hi = warpTransposeSum32C(acc, cme, lo);
            v = (double)hi + (double)lo;
        } else {
            float acc[32];
#pragma unroll
            for (int j = 0; j < JW; j++)
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    float a, b;
                    f2::upk(pacc[j][c], a, b);
                    acc[3 * j + c] = a + b;
                }
#pragma unroll
            for (int k = 3 * JW; k < 32; k++) acc[k] = 0.0f;
            v = (double)warpTransposeSum32(acc);
        }
        const int j = lane / 3, c = lane - 3 * j;
        const int wl = warp + COORD_NW * j;
        if (lane < 3 * JW && wl < nw)
            B.hillPart[3 * ((size_t)blockIdx.x * B.W + w0 + wl) + c] = c == 0 ? v : v * (c == 1 ? hb.gsc[0] : hb.gsc[1]);
    }
}

// ------------------------------------------------------------- the runs
// Persistent CTAs (grid = SMs x resident CTAs): CTA b copies its hill tables,
// runs its static range of coordination steps (equal step counts; the hill
// gathers are issued when the first step starts), then evaluates its slice.
template <int RA, int RB, int BOX, int NH, bool HI, bool COMP>
__device__ __forceinline__ void runsBody(const BatchDev& B, CoordRunSmem<RA, RB>& sm, HillStage& hs) {
    unsigned long long* st = B.stamps ? B.stamps + 10 * (size_t)blockIdx.x : nullptr;
    if (st && threadIdx.x == 0) {
        unsigned sm;
        asm volatile("mov.u32 %0, %%smid;" : "=r"(sm));
        st[6] = sm;
        st[0] = globalTimer();
    }
    const bool hills = B.hill.present != 0;
    if (hills) {
        hillStageTables(B, 0, hs);
        cpAsyncCommit();
    }
    if (st && threadIdx.x == 0) st[1] = globalTimer();
    const int s0 = coordRange(B.R.numSteps, gridDim.x, blockIdx.x), s1 = coordRange(B.R.numSteps, gridDim.x, blockIdx.x + 1);
    if (s0 < s1) {
        // profiling stamps 7, 9 and 8: the first step's data has landed / the first
        // step is done / the hill CVs evaluated after it are done
        if (hills)
            coordRun<RA, RB, BOX, NH, HI, COMP>(
                B.R, s0, s1, sm, NoPieceHook(),
                [&]() {
                    if (st && threadIdx.x == 0) st[7] = globalTimer();
                    hillStageData(B, 0, hs);
                    cpAsyncCommit();
                },
                [&]() {
                    if (st && threadIdx.x == 0) st[9] = globalTimer();
                    hillCVs(B, 0, hs);   // read after the barriers of the hill slice
                    if (st && threadIdx.x == 0) st[8] = globalTimer();
                });
        else
            coordRun<RA, RB, BOX, NH, HI, COMP>(
                B.R, s0, s1, sm, NoPieceHook(),
                [&]() { if (st && threadIdx.x == 0) st[7] = globalTimer(); },
                [&]() { if (st && threadIdx.x == 0) st[8] = st[9] = globalTimer(); });
    }
    if (st) { __syncthreads(); if (threadIdx.x == 0) st[2] = globalTimer(); }
    // the finalize (a programmatic dependent launch) may be scheduled once every
    // CTA is here; it waits for this grid's completion before reading its output
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    if (hills) hillSlice<COMP>(B, hs, s0 < s1, s0 < s1, st);
    if (st) {
        __syncthreads();
        if (threadIdx.x == 0) {
            if (!hills) st[3] = st[4] = st[2];
            st[5] = globalTimer();
        }
    }
}

// Dynamic shared memory: the coordination buffers, then (with a hill bias) the
// hill staging area.
template <int RA, int RB>
constexpr size_t hillStageOffset() { return (sizeof(CoordRunSmem<RA, RB>) + 255) / 256 * 256; }

template <int RA, int RB, int BOX, int NH, bool HI, bool COMP>
__global__ void __launch_bounds__(RUNS_THREADS, 1) k_batch_runs(BatchDev B) {
    extern __shared__ __align__(256) unsigned char dsm[];
    runsBody<RA, RB, BOX, NH, HI, COMP>(B, *reinterpret_cast<CoordRunSmem<RA, RB>*>(dsm),
                                        *reinterpret_cast<HillStage*>(dsm + hillStageOffset<RA, RB>()));
}

// ------------------------------------------------------------- finalize
// CTA (walker w, part p) after the runs:
//   - loads whose addresses are known at plan time go first: the part's share of
//     the walker's coordination rows (fixed-point sums, cleared after use) and
//     their atoms, then the walker record;
//   - CN = the walker's run-piece partials in step order; dU/dCN from the
//     harmonic terms (the hill bias acts only on distance/angle/dihedral CVs);
//     the part's coordination rows are scattered (gradient rounded to float as
//     in the per-context Jacobian table);
//   - part 0 completes the walker: distance/angle/dihedral CVs, the hill
//     partials of the runs CTAs summed in CTA order (lane-strided, fixed xor
//     tree), harmonic terms and hill bias, CVs and energies, and the
//     distance/angle/dihedral rows. With more than one part it has no
//     coordination rows: its own chain of dependent steps is the longest, and
//     without the rows' loads and scatter it ends ~0.6 us earlier and the C4
//     step (64 walkers, 1,280 rows each) takes ~1 us less.
// Copies n bytes (multiple of 4) from global to shared memory, all threads.
__device__ __forceinline__ void copyWords(void* dst, const void* src, int n) {
    const int* s = static_cast<const int*>(src);
    int* d = static_cast<int*>(dst);
    for (int i = threadIdx.x; i < n / 4; i += blockDim.x) d[i] = __ldg(s + i);
}

constexpr int MAXCOORD = 8;   // coordination CVs per walker
constexpr int HPU = 8;        // hill partials per lane loaded at a time

struct FinSmem {
    double sCV[MAXCV], sdU[MAXCV];
    double tE[MAXHARM], tdU[MAXHARM];   // harmonic terms: energy, dU/dCV
    F3 sJac[MAXSIMPLE * 4];
    double sHill[3];
    // the walker's record: one round of independent loads
    BWalker sW;
    BSimple sSimple[MAXSIMPLE];
    BHarm sHarm[MAXHARM];
    CoordItem sItem[MAXCOORD];
};

__device__ void finalizeItem(const BatchDev& B, int fi, FinSmem& fs) {
    double* sCV = fs.sCV;
    double* sdU = fs.sdU;
    F3* sJac = fs.sJac;
    BWalker& sW = fs.sW;
    BSimple* sSimple = fs.sSimple;
    BHarm* sHarm = fs.sHarm;
    CoordItem* sItem = fs.sItem;
    const int w = fi / B.parts, part = fi % B.parts;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const BHill& hb = B.hill;
    unsigned long long* st = B.fstamps ? B.fstamps + 6 * (size_t)fi : nullptr;
    if (st && tid == 0) st[0] = globalTimer();
    // coordination rows: with more than one part, part 0 only completes the
    // walker and parts 1, 2, ... share the rows; a single part does both
    const int rowParts = B.parts > 1 ? B.parts - 1 : 1, rp = B.parts > 1 ? part - 1 : 0;
    const int r0 = rp < 0 ? 0 : (int)((long long)B.rowsPerWalker * rp / rowParts);
    const int r1 = rp < 0 ? 0 : (int)((long long)B.rowsPerWalker * (rp + 1) / rowParts);
    long long vx[ROWS_PER_THREAD], vy[ROWS_PER_THREAD], vz[ROWS_PER_THREAD];
    int rItem[ROWS_PER_THREAD], rAtom[ROWS_PER_THREAD];
    const size_t rowBase = (size_t)w * B.rowsPerWalker;
    // loads that do not depend on the runs kernel: atoms of the rows, the record
#pragma unroll
    for (int q = 0; q < ROWS_PER_THREAD; q++) {
        const int r = r0 + tid + FT * q;
        rItem[q] = r < r1 ? 0 : -1;
        rAtom[q] = r < r1 ? __ldg(B.rowAtom + rowBase + r) : 0;
    }
    copyWords(&sW, B.walkers + w, sizeof(BWalker));
    copyWords(sSimple, B.simple + (size_t)w * B.nS, sizeof(BSimple) * B.nS);
    copyWords(sHarm, B.harm + (size_t)w * B.nH, sizeof(BHarm) * B.nH);
    copyWords(sItem, B.items + (size_t)w * B.nC, sizeof(CoordItem) * B.nC);
    // launched as a programmatic dependent of the runs kernel: wait here until
    // it has completed and its writes are visible (no-op otherwise)
    asm volatile("griddepcontrol.wait;" ::: "memory");
#pragma unroll
    for (int q = 0; q < ROWS_PER_THREAD; q++) {
        vx[q] = vy[q] = vz[q] = 0;
        if (rItem[q] == 0) {
            const unsigned long long* a = B.R.acc + 3 * (rowBase + r0 + tid + FT * q);
            vx[q] = (long long)__ldcg(a); vy[q] = (long long)__ldcg(a + 1); vz[q] = (long long)__ldcg(a + 2);
        }
    }
    // part 0: the hill partials of the runs CTAs (warp 2; lane l sums CTAs l,
    // l + 32, ... in that order, HPU of them loaded at a time)
    double hv0 = 0.0, hv1 = 0.0, hv2 = 0.0;
    if (part == 0 && hb.present && warp == 2)
        for (int c0 = lane; c0 < B.hillParts; c0 += 32 * HPU) {
            double a0[HPU], a1[HPU], a2[HPU];
#pragma unroll
            for (int u = 0; u < HPU; u++) {
                const int c = c0 + 32 * u;
                const double* q = B.hillPart + 3 * ((size_t)c * B.W + w);
                a0[u] = c < B.hillParts ? __ldcg(q) : 0.0;
                a1[u] = c < B.hillParts ? __ldcg(q + 1) : 0.0;
                a2[u] = c < B.hillParts ? __ldcg(q + 2) : 0.0;
            }
#pragma unroll
            for (int u = 0; u < HPU; u++) { hv0 += a0[u]; hv1 += a1[u]; hv2 += a2[u]; }
        }
    if (tid < MAXCV) { sCV[tid] = 0.0; sdU[tid] = 0.0; }
    if (part == 0 && warp == 2) {
        hv0 = warpSum(hv0); hv1 = warpSum(hv1); hv2 = warpSum(hv2);
        if (lane == 0) { fs.sHill[0] = hv0; fs.sHill[1] = hv1; fs.sHill[2] = hv2; }
    }
    __syncthreads();
    if (st && tid == 0) st[1] = globalTimer();
    // part 0: distance/angle/dihedral CVs (warp 1)
    if (part == 0 && warp == 1 && lane < B.nS) {
        F3 jac[4];
        const float v = simpleCV(sSimple[lane].type, sSimple[lane].atoms, sW.posq, nullptr, sW.box, jac);
        for (int k = 0; k < 4; k++) sJac[lane * 4 + k] = jac[k];
        sCV[sSimple[lane].cv] = (double)v;
    }
    // the item of every row (item 0's A and B rows, then item 1's, ...)
#pragma unroll
    for (int q = 0; q < ROWS_PER_THREAD; q++) {
        if (rItem[q] < 0) continue;
        const int r = r0 + tid + FT * q;
        int c = 0, base = 0;
        while (c < B.nC - 1 && r >= base + sItem[c].nA + sItem[c].nB) {
            base += sItem[c].nA + sItem[c].nB;
            c++;
        }
        rItem[q] = c;
    }
    // CN: warps 2..7 take items warp - 2, warp + 4, ...; lane l sums pieces l,
    // l + 32, ... (step order), fixed xor tree
    for (int c = warp - 2; c >= 0 && c < B.nC; c += FT / 32 - 2) {
        const CoordItem& it = sItem[c];
        double t = 0.0;
        for (int k = it.pieceBegin + lane; k < it.pieceEnd; k += 32) t += __ldcg(B.R.cnPiece + k);
        t = warpSum(t);
        if (lane == 0) sCV[it.cv] = t;
    }
    __syncthreads();
    if (st && tid == 0) st[2] = globalTimer();
    // dU/dCN (coordination CVs); part 0: all CVs, energies. Lane k of warp 0
    // evaluates harmonic term k; lane 0 adds them in term order.
    if (warp == 0) {
        if (lane < B.nH) {
            const BHarm& hm = sHarm[lane];
            bool coordCv = false;
            for (int c = 0; c < B.nC; c++) coordCv = coordCv || sItem[c].cv == hm.cv;
            double e = 0.0, du = 0.0;
            if (part == 0 || coordCv) du = harmonicDU(hm, sCV[hm.cv], e);
            fs.tE[lane] = e;
            fs.tdU[lane] = du;
        }
        __syncwarp();
    }
    if (tid == 0) {
        double E = 0.0;
        for (int k = 0; k < B.nH; k++) {
            E += fs.tE[k];
            sdU[sHarm[k].cv] += fs.tdU[k];
        }
        if (part == 0) {
            if (hb.present) {
                E += fs.sHill[0];
                sdU[hb.cv[0]] += fs.sHill[1];
                if (hb.D > 1) sdU[hb.cv[1]] += fs.sHill[2];
            }
            for (int k = 0; k < B.nCV; k++) B.cvv[(size_t)w * B.nCV + k] = sCV[k];
            B.energy[w] = E;
            B.hillEnergy[w] = hb.present ? fs.sHill[0] : 0.0;
        }
    }
    __syncthreads();
    if (st && tid == 0) st[3] = globalTimer();
    unsigned long long* F = sW.force;
    const int P = sW.padded;
#pragma unroll
    for (int q = 0; q < ROWS_PER_THREAD; q++) {
        if (rItem[q] < 0) continue;
        const CoordItem& it = sItem[rItem[q]];
        const double g = sdU[it.cv];
        unsigned long long* a = B.R.acc + 3 * (rowBase + r0 + tid + FT * q);
        a[0] = 0ull; a[1] = 0ull; a[2] = 0ull;
        if (g == 0.0) continue;
        const double sc = coordAccScale(it) * crun::IFXD;
        scatterRow(F, P, rAtom[q], g, (float)((double)vx[q] * sc), (float)((double)vy[q] * sc),
                   (float)((double)vz[q] * sc));
    }
    if (st && tid == 0) st[4] = globalTimer();
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
    if (st) { __syncthreads(); if (tid == 0) st[5] = globalTimer(); }
}

__global__ void __launch_bounds__(FT) k_batch_finalize(BatchDev B) {
    __shared__ FinSmem fs;
    finalizeItem(B, blockIdx.x, fs);
}

typedef void (*RunsFn)(BatchDev);

template <int NH, bool COMP>
RunsFn runsKernelB(int box, bool hi) {
    if (box == 0) return k_batch_runs<8, 4, 0, NH, true, COMP>;
    if (box == 1) return hi ? k_batch_runs<8, 4, 1, NH, true, COMP> : k_batch_runs<8, 4, 1, NH, false, COMP>;
    return hi ? k_batch_runs<8, 4, 2, NH, true, COMP> : k_batch_runs<8, 4, 2, NH, false, COMP>;
}

template <bool COMP>
RunsFn runsKernelK(int box, int kind, bool hi) {
    return kind == 3    ? runsKernelB<3, COMP>(box, hi)
           : kind == -1 ? runsKernelB<-1, COMP>(box, true)
                        : runsKernelB<0, COMP>(box, true);
}

// Other tile shapes (RA A atoms per warp, RB B atoms per lane) for the
// autotuner: the n = 6, m = 12 switch in rectangular or no boxes, plain sums.
template <int RA, int RB>
RunsFn runsKernelShape(int box, bool hi) {
    if (box == 0) return k_batch_runs<RA, RB, 0, 3, true, false>;
    return hi ? k_batch_runs<RA, RB, 1, 3, true, false> : k_batch_runs<RA, RB, 1, 3, false, false>;
}

bool shapeAvailable(int box, int kind, bool comp, int ra, int ch) {
    if (ra == 8 && ch == 128) return true;
    return kind == 3 && !comp && box != 2 && (ra == 4 || ra == 8) && (ch == 128 || ch == 256);
}

// comp: two-sum compensated hill sums and blocked coordination A sums.
RunsFn runsKernel(int box, int kind, bool hi, bool comp, int ra, int ch) {
    if (ra == 4 && ch == 128) return runsKernelShape<4, 4>(box, hi);
    if (ra == 8 && ch == 256) return runsKernelShape<8, 8>(box, hi);
    if (ra == 4 && ch == 256) return runsKernelShape<4, 8>(box, hi);
    return comp ? runsKernelK<true>(box, kind, hi) : runsKernelK<false>(box, kind, hi);
}

size_t runsSmemOffset(int ra, int ch) {
    if (ra == 4 && ch == 128) return hillStageOffset<4, 4>();
    if (ra == 8 && ch == 256) return hillStageOffset<8, 8>();
    if (ra == 4 && ch == 256) return hillStageOffset<4, 8>();
    return hillStageOffset<8, 4>();
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
        hb.mirror[k] = (float)(c[0] * hb.u[0]);
        hb.mirror[hb.cap + k] = (float)(c[1] * hb.u[1]);
        hb.mirror[2 * hb.cap + k] = (float)h;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        *hb.count = min(hb.maxH, n0 + B.W);
        if (n0 + B.W > hb.maxH) atomicOr(B.status, 1);
    }
}

// ================================================================== host
struct Batch::Impl {
    int W = 0, nCV = 0, nS = 0, nC = 0, nH = 0, boxKind = 1, kind = 3;
    std::vector<BWalker> walkersH;
    std::vector<CoordItem> items;
    std::vector<int> coordAtoms;
    std::vector<CoordStep> steps;
    DBuf walkersD, simpleD, harmD, itemsD, atomsD, stepsD, gBD, gAD, stepPosqD, boxesD, sysPosqD, acc, cnPiece;
    DBuf hillCvPosD, hillCvTypeD, rowAtomD, stepConstD;
    std::vector<BSimple> simpleH;
    DBuf hillPart, cvv, energy, hillEnergy, status, scratchForce;
    DBuf hMirror, hCenters, hHeights, hCount;
    BHill hill{};
    BatchTuning tune;
    int sumMode = SUM_FP32;   // SUM_FP32: plain FP32 sums; SUM_FP32C: two-sum hills, blocked coordination
    bool cachedTune = false;  // the last autotune returned a cached choice
    // autotuner cache key: walker count, coordination group sizes, hill count
    // (power-of-two bucket), box kind, switch kind, sum precision
    int hostHillCount() const {
        int n = 0;
        cudaCheck(cudaMemcpy(&n, hill.count, sizeof(int), cudaMemcpyDeviceToHost), "hills");
        return n;
    }
    std::string signature() const {
        std::string k = std::to_string(W) + "|" + std::to_string(nC);
        for (int c = 0; c < nC; c++) k += "|" + std::to_string(items[c].nA) + "x" + std::to_string(items[c].nB);
        int hb = 0;
        for (int n = hill.present ? hostHillCount() : 0; n > 0; n >>= 1) hb++;
        return k + "|h" + std::to_string(hb) + "|b" + std::to_string(boxKind) + "|k" + std::to_string(kind) + "|s" +
               std::to_string(sumMode);
    }
    BatchDev dev{};
    int grid = 0;        // coordination runs: SMs x resident CTAs
    int rows = 0;        // coordination rows of one walker
    int parts = 1;       // finalize CTAs per walker
    bool hi = true;
    cudaStream_t stream = 0;
    cudaStream_t cap = nullptr;
    cudaGraphExec_t graph = nullptr;
    long long launches = 0;
    int lastUpdateStep = -1;
    std::vector<unsigned long long> lastStamps;   // raw records of the last phaseTimes call
    bool ready = false;
    float lastMs = 0;

    void destroyGraph() {
        if (graph) { cudaGraphExecDestroy(graph); graph = nullptr; }
    }

    RunsFn runs() const { return runsKernel(boxKind, kind, hi, sumMode == SUM_FP32C, tune.ra, tune.ch); }

    // Per-CTA step ranges (equal step counts) and the run pieces to match. The
    // device copies are rewritten in place (a captured graph keeps their
    // addresses) unless they must grow.
    void balance() {
        std::vector<int> begin = balanceRanges((int)steps.size(), grid);
        const int pieces = buildCoordPieces(steps, begin, items);
        auto put = [&](DBuf& d, const void* src, size_t bytes) {
            if (d.bytes < bytes) { d.alloc(bytes); destroyGraph(); }
            if (bytes) cudaCheck(cudaMemcpy(d.p, src, bytes, cudaMemcpyHostToDevice), "ranges");
        };
        put(stepsD, steps.data(), sizeof(CoordStep) * steps.size());
        put(itemsD, items.data(), sizeof(CoordItem) * items.size());
        if (cnPiece.bytes < sizeof(double) * std::max(1, pieces)) {
            cnPiece.alloc(sizeof(double) * std::max(1, pieces));
            destroyGraph();
        }
        // per-step gather tables (slot = user atom index in a walker's posq)
        const size_t n = std::max<size_t>(1, steps.size());
        const int ta = COORD_NW * tune.ra, ch = tune.ch;
        if (gBD.bytes < sizeof(int) * ch * n) { gBD.alloc(sizeof(int) * ch * n); destroyGraph(); }
        if (gAD.bytes < sizeof(int) * ta * n) { gAD.alloc(sizeof(int) * ta * n); destroyGraph(); }
        std::vector<const float4*> stepPosq(n, nullptr);
        for (size_t k = 0; k < steps.size(); k++) stepPosq[k] = walkersH[steps[k].sys].posq;
        put(stepPosqD, stepPosq.data(), sizeof(const float4*) * n);
        launchStepGathers(0, stepsD.as<CoordStep>(), (int)steps.size(), grid, atomsD.as<int>(), gBD.as<int>(),
                          gAD.as<int>(), ta, ch);
        // per-step pair constants (items and walker boxes are fixed for the batch)
        if (stepConstD.bytes < runConstBytes() * n) { stepConstD.alloc(runConstBytes() * n); destroyGraph(); }
        launchStepConsts(0, stepsD.as<CoordStep>(), (int)steps.size(), itemsD.as<CoordItem>(), boxesD.as<BoxDev>(),
                         static_cast<RunConst*>(stepConstD.p));
        cudaCheck(cudaGetLastError(), "gather tables");
        cudaCheck(cudaDeviceSynchronize(), "gather tables");
        dev.R.numSteps = (int)steps.size();
        dev.R.gB = gBD.as<int>();
        dev.R.gA = gAD.as<int>();
        dev.R.stepPosq = stepPosqD.as<const float4*>();
        dev.R.stepConst = static_cast<const RunConst*>(stepConstD.p);
        dev.R.steps = stepsD.as<CoordStep>();
        dev.R.items = itemsD.as<CoordItem>();
        dev.items = itemsD.as<CoordItem>();
        dev.R.cnPiece = cnPiece.as<double>();
    }

    // finalize CTAs whose rows fit: ceil(rows / (FT ROWS_PER_THREAD)), plus the
    // walker part when that is more than one
    int rowCTAs() const { return std::max(1, (rows + FT * ROWS_PER_THREAD - 1) / (FT * ROWS_PER_THREAD)); }
    int minParts() const { return rowCTAs() == 1 ? 1 : rowCTAs() + 1; }

    void plan() {
        // coordination steps over all walkers' items (walker-major)
        buildCoordSteps(items, tune.ra, tune.ch, steps, std::max(nC, 1));
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
        runKernelSetup((const void*)runs(), dynSmem());
        int perSM = 0;
        cudaCheck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, (const void*)runs(), RUNS_THREADS, dynSmem()),
                  "occupancy");
        if (perSM < 1) throw Error(GLUED_E_CUDA, "batched runs kernel cannot be resident");
        grid = sms * perSM;   // persistent: every CTA resident
        balance();
        parts = tune.parts > 0 ? std::max(minParts(), tune.parts) : minParts();
        hillPart.alloc(sizeof(double) * 3 * (size_t)W * grid);
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
        dev.R.acc = acc.as<unsigned long long>();
        dev.R.cnPiece = cnPiece.as<double>();
        dev.rowsPerWalker = rows;
        dev.parts = parts;
        dev.hill = hill;
        dev.hillPart = hillPart.as<double>();
        dev.hillParts = grid;
        dev.cvv = cvv.as<double>(); dev.energy = energy.as<double>(); dev.hillEnergy = hillEnergy.as<double>();
        // plan-time address tables: hill-CV atoms per walker and dimension, atom per row
        std::vector<const float4*> hcp((size_t)W * 8, nullptr);
        std::vector<int> hct((size_t)W * 2, 0);
        for (int w = 0; w < W && hill.present; w++)
            for (int d = 0; d < hill.D; d++)
                for (int k = 0; k < nS; k++) {
                    const BSimple& si = simpleH[(size_t)w * nS + k];
                    if (si.cv != hill.cv[d]) continue;
                    const int na = si.type == 1 ? 2 : si.type == 2 ? 3 : 4;
                    hct[w * 2 + d] = si.type;
                    for (int a = 0; a < na; a++) hcp[(size_t)w * 8 + d * 4 + a] = walkersH[w].posq + si.atoms[a];
                }
        hillCvPosD.upload(hcp);
        hillCvTypeD.upload(hct);
        std::vector<int> ra((size_t)std::max(1, W * rows), 0);
        for (int w = 0; w < W; w++) {
            int r = 0;
            for (int c = 0; c < nC; c++) {
                const CoordItem& it = items[(size_t)w * nC + c];
                for (int i = 0; i < it.nA; i++) ra[(size_t)w * rows + r++] = coordAtoms[it.a0 + i];
                for (int i = 0; i < it.nB; i++) ra[(size_t)w * rows + r++] = coordAtoms[it.b0 + i];
            }
        }
        rowAtomD.upload(ra);
        dev.hillCvPos = hillCvPosD.as<const float4*>();
        dev.hillCvType = hillCvTypeD.as<int>();
        dev.rowAtom = rowAtomD.as<int>();
        dev.status = status.as<int>();
        destroyGraph();
    }

    // dynamic shared memory of the runs kernel: coordination buffers, then the
    // hill staging area
    size_t dynSmem() const { return runsSmemOffset(tune.ra, tune.ch) + (hill.present ? sizeof(HillStage) : 0); }

    void launchRuns(cudaStream_t s) {
        void* args[] = {&dev};
        cudaCheck(cudaLaunchKernel((const void*)runs(), dim3(grid), dim3(RUNS_THREADS), args, dynSmem(), s), "runs");
    }
    // Programmatic dependent launch: the finalize CTAs may start as runs CTAs
    // retire, load what does not depend on the runs, then wait in hardware
    // (griddepcontrol.wait) for the runs grid to complete.
    void launchFinalize(cudaStream_t s) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(W * parts);
        cfg.blockDim = dim3(FT);
        cfg.dynamicSmemBytes = 0;
        cfg.stream = s;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = tune.plain ? 0 : 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        cudaCheck(cudaLaunchKernelEx(&cfg, k_batch_finalize, dev), "finalize");
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
        const double LOG2E = 1.4426950408889634;
        h.cut = (float)(8.0 * LOG2E);
        for (int d = 0; d < 2; d++) {
            h.cv[d] = d < D ? bs.cvs[d] : 0;
            const double sg = d < D ? bs.params[1 + d] : 1.0;
            if (d < D && !(sg > 0.0)) throw Error(GLUED_E_INVALID, "batch: METAD_HILLS sigma must be > 0");
            const double u = d < D ? std::sqrt(LOG2E / (2.0 * sg * sg)) : 0.0;
            h.u[d] = (float)u;
            h.gsc[d] = d < D ? (float)(-1.0 / (sg * sg * u)) : 0.0f;
            const int per = d < D ? bs.iparams[2 + d] : 0;
            const double L = d < D ? bs.params[3 + 2 * D + d] - bs.params[3 + D + d] : 0.0;
            h.pS[d] = per ? (float)(L * u) : 0.0f;
            h.ipS[d] = per ? (float)(1.0 / (L * u)) : 0.0f;
        }
        if (h.maxH < 1) throw Error(GLUED_E_INVALID, "batch: METAD_HILLS maxHills must be >= 1");
        h.cap = (h.maxH + 3) / 4 * 4;
        I.hMirror.alloc(sizeof(float) * 3 * (size_t)h.cap);
        I.hCenters.alloc(sizeof(double) * (size_t)h.maxH * D);
        I.hHeights.alloc(sizeof(double) * (size_t)h.maxH);
        I.hCount.alloc(sizeof(int) * 4);
        h.mirror = I.hMirror.as<float>(); h.centers = I.hCenters.as<double>();
        h.heights = I.hHeights.as<double>(); h.count = I.hCount.as<int>();
    }
    I.walkersD.upload(I.walkersH);
    I.simpleD.upload(simple);
    I.simpleH = simple;
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
    if ((t.ra != 4 && t.ra != 8) || (t.ch != 128 && t.ch != 256))
        throw Error(GLUED_E_INVALID, "batch tuning: ra must be 4 or 8 and the B chunk 128 or 256");
    if (!shapeAvailable(impl_->boxKind, impl_->kind, impl_->sumMode == SUM_FP32C, t.ra, t.ch))
        throw Error(GLUED_E_INVALID, "batch tuning: tile shapes other than ra 8 / chunk 128 need the n = 6, m = 12 "
                                     "switch, a rectangular or no box and plain FP32 sums");
    if (t.parts < 0 || t.parts > 4096) throw Error(GLUED_E_INVALID, "batch tuning: finalize parts must be 0..4096");
    if (t.plain != 0 && t.plain != 1) throw Error(GLUED_E_INVALID, "batch tuning: finalize launch mode must be 0 or 1");
    cudaCheck(cudaStreamSynchronize(impl_->stream), "sync");
    impl_->tune = t;
    impl_->plan();
}

// The tuning in effect: finalize parts as launched (requested, or the fewest).
BatchTuning Batch::tuning() const {
    BatchTuning t = impl_->tune;
    t.parts = impl_->parts;
    return t;
}
bool Batch::lastTuneCached() const { return impl_->cachedTune; }

void Batch::setSumPrecision(int mode) {
    if (mode != SUM_FP32 && mode != SUM_FP32C)
        throw Error(GLUED_E_INVALID, "batch sum precision: mode must be 1 (FP32) or 2 (FP32 two-sum)");
    cudaCheck(cudaStreamSynchronize(impl_->stream), "sync");
    if (mode != impl_->sumMode) {
        impl_->sumMode = mode;
        impl_->destroyGraph();
        BatchTuning& t = impl_->tune;
        if (!shapeAvailable(impl_->boxKind, impl_->kind, mode == SUM_FP32C, t.ra, t.ch)) {
            // compensated sums exist in the default tile shape only
            t.ra = 8;
            t.ch = 128;
            impl_->plan();
        }
        // the other instantiation of the runs kernel: its shared-memory limit
        runKernelSetup((const void*)impl_->runs(), impl_->dynSmem());
    }
}

int Batch::sumPrecision() const { return impl_->sumMode; }

void Batch::execute() {
    Impl& I = *impl_;
    if (!I.graph) {
        cudaGraph_t g = nullptr;
        cudaCheck(cudaStreamBeginCapture(I.cap, cudaStreamCaptureModeThreadLocal), "capture begin");
        bool launched = true;
        try {
            I.launch(I.cap);
        } catch (const Error&) {
            launched = false;
        }
        cudaError_t ce = cudaStreamEndCapture(I.cap, &g);
        cudaError_t ie = cudaErrorUnknown;
        if (launched && ce == cudaSuccess && g) ie = cudaGraphInstantiate(&I.graph, g, 0);
        if (g) cudaGraphDestroy(g);
        if (!launched || ce != cudaSuccess || ie != cudaSuccess) {
            cudaGetLastError();
            I.graph = nullptr;
            throw Error(GLUED_E_CUDA, "batch: step graph capture failed");
        }
    }
    cudaCheck(cudaGraphLaunch(I.graph, I.stream), "graph launch");
    I.launches += I.launchesPerStep();
    I.ready = true;
}

// Autotuner: the finalize CTAs per walker and its launch mode are timed on the
// live walkers with CUDA events (forces go to a scratch buffer) and the fastest
// combination is kept. Every timed step starts with L2 flushed (a 192 MB memset
// between steps), as in an MD loop where the engine's own kernels run between
// force evaluations; the flush buffer is freed before returning.
// Choices of the autotuner, per batch signature (signature()), for the process.
static std::map<std::string, BatchTuning>& tuneCache() {
    static std::map<std::string, BatchTuning> m;
    return m;
}
static std::mutex& tuneCacheMutex() {
    static std::mutex m;
    return m;
}

BatchTuning Batch::autotune(bool useCache) {
    Impl& I = *impl_;
    cudaCheck(cudaStreamSynchronize(I.stream), "sync");
    if (useCache) {
        BatchTuning hit;
        bool found = false;
        {
            std::lock_guard<std::mutex> lock(tuneCacheMutex());
            auto it = tuneCache().find(I.signature());
            if (it != tuneCache().end()) { hit = it->second; found = true; }
        }
        if (found) {
            I.tune = hit;
            I.plan();
            I.cachedTune = true;
            return hit;
        }
    }
    I.cachedTune = false;
    size_t maxPad = 0;
    for (auto& w : I.walkersH) maxPad = std::max(maxPad, (size_t)w.padded);
    I.scratchForce.alloc(sizeof(long long) * 3 * maxPad);
    std::vector<BWalker> tmp = I.walkersH;
    for (auto& w : tmp) w.force = I.scratchForce.as<unsigned long long>();
    cudaCheck(cudaMemcpy(I.walkersD.p, tmp.data(), sizeof(BWalker) * tmp.size(), cudaMemcpyHostToDevice), "tune");
    DBuf flush;
    flush.alloc((size_t)192 << 20);
    constexpr int reps = 8;
    cudaEvent_t ev[2 * reps];
    for (auto& e : ev) cudaCheck(cudaEventCreate(&e), "event");
    BatchTuning best = I.tune;
    float bestMs = 1e30f;
    // finalize parts: the fewest, then r row CTAs + the walker part for r = the
    // fewest row CTAs + 0, 1, 2 and x2, x4 (a grid over the SMs' resident CTAs
    // adds a second wave: 64 walkers x 7 parts of 256 threads at 80 registers
    // run 4 CTAs late and cost C4 ~2 us against 6 parts)
    const int rb = I.rowCTAs();
    std::vector<int> partsList = {I.minParts()};
    for (int r : {rb, rb + 1, rb + 2, 2 * rb, 4 * rb})
        if (std::find(partsList.begin(), partsList.end(), r + 1) == partsList.end()) partsList.push_back(r + 1);
    std::vector<BatchTuning> cands;
    for (int ra : {8, 4})
        for (int ch : {128, 256}) {
            if (!shapeAvailable(I.boxKind, I.kind, I.sumMode == SUM_FP32C, ra, ch)) continue;
            for (int plain : {0, 1})
                for (int parts : partsList) {
                    BatchTuning t;
                    t.ra = ra; t.ch = ch; t.plain = plain; t.parts = parts;
                    cands.push_back(t);
                }
        }
    for (const BatchTuning& t : cands) {
            I.tune = t;
            I.plan();
            for (int r = 0; r < 2; r++) I.launch(I.stream);
            for (int r = 0; r < reps; r++) {
                cudaCheck(cudaMemsetAsync(flush.p, r & 0xff, flush.bytes, I.stream), "flush");
                cudaCheck(cudaEventRecord(ev[2 * r], I.stream), "event");
                I.launch(I.stream);
                cudaCheck(cudaEventRecord(ev[2 * r + 1], I.stream), "event");
            }
            cudaCheck(cudaEventSynchronize(ev[2 * reps - 1]), "event");
            float ms = 0;
            for (int r = 0; r < reps; r++) {
                float x = 0;
                cudaCheck(cudaEventElapsedTime(&x, ev[2 * r], ev[2 * r + 1]), "event");
                ms += x;
            }
            ms /= reps;
            I.launches += (long long)(reps + 2) * I.launchesPerStep();
            if (ms < bestMs) { bestMs = ms; best = t; }
        }
    for (auto& e : ev) cudaEventDestroy(e);
    cudaCheck(cudaMemcpy(I.walkersD.p, I.walkersH.data(), sizeof(BWalker) * I.walkersH.size(), cudaMemcpyHostToDevice), "tune");
    I.tune = best;
    I.plan();
    I.lastMs = bestMs;
    {
        std::lock_guard<std::mutex> lock(tuneCacheMutex());
        tuneCache()[I.signature()] = best;
    }
    return best;
}

// Percentile p (0..100) of v (sorted in place).
static double pct(std::vector<double>& v, double p) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    size_t i = (size_t)std::min((double)v.size() - 1, std::floor(p / 100.0 * (double)(v.size() - 1) + 0.5));
    return v[i];
}

// One regular step launched without the graph, each launch between CUDA events
// and every CTA recording %globaltimer at its phase boundaries (runs: entry,
// staging issued, coordination done, hill slice done; finalize: six stamps);
// the layout of out[24] is given with glued_batch_phase_times.
void Batch::phaseTimes(double* out) {
    Impl& I = *impl_;
    constexpr int RS = 10, FS = 6;   // stamps per runs / finalize CTA
    const int fg = I.W * I.parts;
    DBuf st;
    st.alloc(sizeof(unsigned long long) * (RS * (size_t)I.grid + FS * (size_t)fg));
    cudaCheck(cudaMemsetAsync(st.p, 0, st.bytes, I.stream), "stamps");
    I.dev.stamps = st.as<unsigned long long>();
    I.dev.fstamps = st.as<unsigned long long>() + RS * (size_t)I.grid;
    // events around the whole step only: an event between the two launches
    // would hold the finalize back until the runs grid has drained (no
    // programmatic dependent launch), which the step graph does not do
    cudaEvent_t e[2];
    for (auto& x : e) cudaCheck(cudaEventCreate(&x), "event");
    cudaCheck(cudaEventRecord(e[0], I.stream), "event");
    I.launchRuns(I.stream);
    I.launchFinalize(I.stream);
    cudaCheck(cudaEventRecord(e[1], I.stream), "event");
    I.dev.stamps = nullptr;
    I.dev.fstamps = nullptr;
    cudaCheck(cudaEventSynchronize(e[1]), "event");
    float a = 0;
    cudaCheck(cudaEventElapsedTime(&a, e[0], e[1]), "event");
    // a second step with each launch between events: the kernels' own durations
    // (the finalize then starts after the runs grid has drained)
    cudaEvent_t k[3];
    for (auto& x : k) cudaCheck(cudaEventCreate(&x), "event");
    cudaCheck(cudaEventRecord(k[0], I.stream), "event");
    I.launchRuns(I.stream);
    cudaCheck(cudaEventRecord(k[1], I.stream), "event");
    I.launchFinalize(I.stream);
    cudaCheck(cudaEventRecord(k[2], I.stream), "event");
    cudaCheck(cudaEventSynchronize(k[2]), "event");
    float kr = 0, kf = 0;
    cudaCheck(cudaEventElapsedTime(&kr, k[0], k[1]), "event");
    cudaCheck(cudaEventElapsedTime(&kf, k[1], k[2]), "event");
    for (auto& x : k) cudaEventDestroy(x);
    I.launches += I.launchesPerStep();
    for (auto& x : e) cudaEventDestroy(x);
    I.launches += I.launchesPerStep();
    I.ready = true;
    std::vector<unsigned long long> h(st.bytes / sizeof(unsigned long long));
    cudaCheck(cudaMemcpy(h.data(), st.p, st.bytes, cudaMemcpyDeviceToHost), "stamps");
    // raw records: runs CTA {SM, steps, 6 times}, finalize CTA {6 times}
    {
        std::vector<int> begin = balanceRanges((int)I.steps.size(), I.grid);
        I.lastStamps.clear();
        for (int g = 0; g < I.grid; g++) {
            const unsigned long long* r = h.data() + RS * (size_t)g;
            I.lastStamps.push_back(r[6]);
            I.lastStamps.push_back((unsigned long long)(begin[g + 1] - begin[g]));
            for (int k = 0; k < 6; k++) I.lastStamps.push_back(r[k]);
            I.lastStamps.push_back(r[7]);
            I.lastStamps.push_back(r[8]);
            I.lastStamps.push_back(r[9]);
        }
        for (int g = 0; g < fg; g++)
            for (int k = 0; k < FS; k++) I.lastStamps.push_back(h[RS * (size_t)I.grid + FS * (size_t)g + k]);
    }
    unsigned long long t0 = ~0ull, f0 = ~0ull, f1 = 0;
    for (int g = 0; g < I.grid; g++) t0 = std::min(t0, h[RS * (size_t)g]);
    for (int g = 0; g < fg; g++) {
        f0 = std::min(f0, h[RS * (size_t)I.grid + FS * (size_t)g]);
        f1 = std::max(f1, h[RS * (size_t)I.grid + FS * (size_t)g + 5]);
    }
    std::vector<double> stage, coord, end, hw, he, hr, fdur, fph[5], ready, firstStep;
    for (int g = 0; g < I.grid; g++) {
        const unsigned long long* r = h.data() + RS * (size_t)g;
        if (r[7] && r[8]) {
            ready.push_back((r[7] - r[0]) * 1e-3);
            firstStep.push_back((r[8] - r[7]) * 1e-3);
        }
        stage.push_back((r[1] - r[0]) * 1e-3);
        coord.push_back((r[2] - t0) * 1e-3);
        hw.push_back((r[3] - r[2]) * 1e-3);
        he.push_back((r[4] - r[3]) * 1e-3);
        hr.push_back((r[5] - r[4]) * 1e-3);
        end.push_back((r[5] - t0) * 1e-3);
    }
    for (int g = 0; g < fg; g++) {
        const unsigned long long* r = h.data() + RS * (size_t)I.grid + FS * (size_t)g;
        fdur.push_back((r[5] - r[0]) * 1e-3);
        for (int k = 0; k < 5; k++) fph[k].push_back((r[k + 1] - r[k]) * 1e-3);
    }
    out[0] = a * 1e3; out[1] = (double)(f1 - t0) * 1e-3;
    out[2] = pct(stage, 50); out[3] = pct(stage, 100);
    out[4] = pct(coord, 0); out[5] = pct(coord, 50); out[6] = pct(coord, 100);
    out[7] = pct(end, 50); out[8] = pct(end, 100);
    out[9] = pct(fdur, 50); out[10] = pct(fdur, 100); out[11] = (double)(f0 - t0) * 1e-3;
    out[12] = (double)I.steps.size(); out[13] = (double)I.grid; out[14] = (double)I.parts; out[15] = (double)fg;
    for (int q = 0; q < 5; q++) out[16 + q] = pct(fph[q], 50);
    out[21] = pct(hw, 50); out[22] = pct(he, 50); out[23] = pct(hr, 50);
    out[24] = kr * 1e3; out[25] = kf * 1e3;
    out[26] = pct(ready, 50); out[27] = pct(firstStep, 50);
}

long long Batch::phaseStamps(unsigned long long* out, long long cap) {
    const std::vector<unsigned long long>& v = impl_->lastStamps;
    if (out) std::copy(v.begin(), v.begin() + std::min<long long>(cap, (long long)v.size()), out);
    return (long long)v.size();
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
    const int cap = I.hill.cap;
    std::vector<float> m((size_t)3 * cap, 0.0f);
    for (int k = 0; k < n; k++) {
        m[k] = (float)(centers[k * D] * I.hill.u[0]);
        m[cap + k] = D > 1 ? (float)(centers[k * D + 1] * I.hill.u[1]) : 0.0f;
        m[2 * (size_t)cap + k] = (float)heights[k];
    }
    if (n > 0) {
        cudaCheck(cudaMemcpy(I.hill.centers, centers, sizeof(double) * (size_t)n * D, cudaMemcpyHostToDevice), "hills");
        cudaCheck(cudaMemcpy(I.hill.heights, heights, sizeof(double) * n, cudaMemcpyHostToDevice), "hills");
        for (int c = 0; c < 3; c++)
            cudaCheck(cudaMemcpy(I.hill.mirror + (size_t)c * cap, m.data() + (size_t)c * cap, sizeof(float) * n,
                                 cudaMemcpyHostToDevice), "hills");
    }
    cudaCheck(cudaMemcpy(I.hill.count, &n, sizeof(int), cudaMemcpyHostToDevice), "hills");
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
