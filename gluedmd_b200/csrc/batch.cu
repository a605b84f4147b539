// Batched multi-walker step: every walker's CVs, biases and force scatter in one
// cooperative persistent launch per step (captured in a CUDA graph).
//
// The reference steps one OpenMM Context per walker and shares the bias through
// raw device pointers (tests/test_multiwalker.py:156-158,
// platforms/common/src/CommonGluedKernels.cpp:5234-5262). Here all walkers of a
// GPU are one launch:
//
// Phase A (work items pulled from an atomic counter, heavy items first):
//   - coordination tiles of every walker (coord_tile.cuh: partial gradients and
//     CN partials, deterministic),
//   - hill-table items: a chunk of 512 hills is staged into shared memory with a
//     TMA bulk copy (cp.async.bulk + mbarrier, local memory only) and evaluated
//     for up to 64 walkers (8 per warp); each item walks the chunks
//     hill_items apart, so the launch shape does not depend on the hill count.
//     Sums are FP32 per lane over <= ~16 terms, a fixed xor tree over the warp,
//     and FP64 across items: a blocked summation with O((16 + 5) eps) error
//     instead of O(N eps).
// Grid barrier (bounded spin; on time-out the status word is set and the kernel
//   returns).
// Phase B (walker, part) items: the walker's CN (sum of its CTA partials),
//   distance/angle/dihedral values and Jacobians, the shared hill bias
//   (sum of item partials), harmonic restraints -> dU/dCV; then the walker's
//   force rows are reduced from the partials and scattered straight into its
//   2^32 fixed-point force buffer. No Jacobian table is materialised.
//
// Deposition (updateState at pace): one hill per walker, in walker order, with
// the well-tempered height from that walker's last hill-bias energy.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <string>

#include "batch.hpp"
#include "context.hpp"
#include "coord_tile.cuh"

namespace glued {

namespace {
constexpr int HCH = 512;       // hills per staged chunk (float4: c0, c1, h, 0)
constexpr int WBLK = 64;       // walkers per hill item (8 per warp)
constexpr int MAXCV = 32;      // CV values per walker
constexpr int MAXSIMPLE = 16;  // distance/angle/dihedral CVs per walker
constexpr int MAXHARM = 32;    // harmonic terms per walker
constexpr int SMEM_BYTES = 16384;
}

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
    CoordDev C;             // items [W][nC]
    int coordBlocks;
    int hillItems;          // per walker block
    int nWB;                // walker blocks
    int parts;
    BHill hill;
    double* hillPart;       // [hillItems][W][3]
    double* cvv;            // [W][nCV]
    double* energy;         // [W]
    double* hillEnergy;     // [W]
    unsigned int* bar;      // {count, generation}
    int* work;
    int* status;
    unsigned long long spinLimit;
    unsigned long long* stamps;  // optional [grid][6] phase timestamps (nullptr = off)
};

// ------------------------------------------------------------- grid barrier
__device__ bool gridBarrier(unsigned int* bar, int* status, unsigned long long limit) {
    __shared__ int sOk;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned int* vgen = bar + 1;
        unsigned int gen = *vgen;
        __threadfence();
        unsigned int arrived = atomicAdd(bar, 1u);
        int ok = 1;
        if (arrived == gridDim.x - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            unsigned long long it = 0;
            while (*vgen == gen) {
                __nanosleep(100);
                if (++it > limit) { atomicOr(status, 1); ok = 0; break; }
            }
        }
        __threadfence();
        sOk = ok;
    }
    __syncthreads();
    return sOk != 0;
}

__device__ __forceinline__ unsigned long long globalTimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// ------------------------------------------------------------- TMA helpers
__device__ __forceinline__ unsigned smemAddr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool mbarWait(unsigned mbar, unsigned parity, unsigned long long limit) {
    unsigned long long it = 0;
    for (;;) {
        unsigned done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done) : "r"(mbar), "r"(parity) : "memory");
        if (done) return true;
        if (++it > limit) return false;
    }
}

// ------------------------------------------------------------- hill items
__device__ void hillItem(const BatchDev& B, int item, unsigned char* smem, unsigned long long* mbarPtr) {
    const int h = item % B.hillItems;
    const int wb = item / B.hillItems;
    const int w0 = wb * WBLK;
    const int nw = min(WBLK, B.W - w0);
    float4* sH = reinterpret_cast<float4*>(smem);                 // HCH hills
    float* sS = reinterpret_cast<float*>(smem + HCH * 16);         // [WBLK][2]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const BHill& hb = B.hill;
    // CV values of this block's walkers the hill bias acts on
    if (tid < nw) {
        const int w = w0 + tid;
        const BWalker& wk = B.walkers[w];
        for (int d = 0; d < 2; d++) {
            float v = 0.0f;
            if (d < hb.D) {
                for (int s = 0; s < B.nS; s++) {
                    const BSimple& si = B.simple[w * B.nS + s];
                    if (si.cv == hb.cv[d]) v = simpleCV(si.type, si.atoms, wk.posq, nullptr, wk.box, nullptr);
                }
            }
            sS[tid * 2 + d] = v;
        }
    }
    const unsigned mbar = smemAddr(mbarPtr);
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(1) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    float acc[8][3];
#pragma unroll
    for (int j = 0; j < 8; j++) acc[j][0] = acc[j][1] = acc[j][2] = 0.0f;
    const int count = *hb.count;
    unsigned parity = 0;
    bool ok = true;
    for (int c = h; c * HCH < count; c += B.hillItems) {
        const int n = min(HCH, count - c * HCH);
        if (tid == 0) {
            unsigned bytes = (unsigned)n * 16u;
            // shared memory may have been written through the generic proxy by an
            // earlier item of this CTA
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                    smemAddr(sH)),
                "l"(hb.mirror + (size_t)c * HCH), "r"(bytes), "r"(mbar)
                : "memory");
        }
        // one thread waits (bounded) and the result is broadcast, so every
        // thread takes the same path through the block barriers below
        if (tid == 0) {
            int got = mbarWait(mbar, parity, B.spinLimit) ? 1 : 0;
            if (!got) atomicOr(B.status, 2);
            *reinterpret_cast<volatile int*>(sS + 2 * WBLK) = got;
        }
        __syncthreads();
        if (!*reinterpret_cast<volatile int*>(sS + 2 * WBLK)) { ok = false; break; }
        parity ^= 1u;
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const int wl = warp + 8 * j;
            if (wl < nw) {
                const float s0 = sS[wl * 2], s1 = sS[wl * 2 + 1];
                float V = 0.0f, g0 = 0.0f, g1 = 0.0f;
                for (int k = lane; k < n; k += 32) {
                    const float4 hk = sH[k];
                    float dx = s0 - hk.x, dy = s1 - hk.y;
                    if (hb.period[0] > 0.0f) dx -= hb.period[0] * rintf(dx * hb.iperiod[0]);
                    if (hb.period[1] > 0.0f) dy -= hb.period[1] * rintf(dy * hb.iperiod[1]);
                    const float ex = dx * dx * hb.a[0] + dy * dy * hb.a[1];
                    const float g = ex <= 8.0f ? hk.z * __expf(-ex) : 0.0f;
                    V += g; g0 += g * dx; g1 += g * dy;
                }
                acc[j][0] += V; acc[j][1] += g0; acc[j][2] += g1;
            }
        }
        __syncthreads();  // chunk fully read before it is overwritten
    }
    if (tid == 0) asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(mbar) : "memory");
    if (!ok) return;
#pragma unroll
    for (int j = 0; j < 8; j++) {
        const int wl = warp + 8 * j;
        float V = warpSumF(acc[j][0]), g0 = warpSumF(acc[j][1]), g1 = warpSumF(acc[j][2]);
        if (lane == 0 && wl < nw) {
            double* out = B.hillPart + 3 * ((size_t)h * B.W + w0 + wl);
            out[0] = V;
            out[1] = -(double)g0 * hb.isig2[0];
            out[2] = -(double)g1 * hb.isig2[1];
        }
    }
    __syncthreads();
}

// ------------------------------------------------------------- finalize
__device__ void finalizeWalker(const BatchDev& B, int w, int part, unsigned char* smem) {
    double* sCV = reinterpret_cast<double*>(smem);           // [MAXCV]
    double* sdU = sCV + MAXCV;                               // [MAXCV]
    double* sScal = sdU + MAXCV;                             // [4]
    F3* sJac = reinterpret_cast<F3*>(sScal + 4);             // [MAXSIMPLE][4]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const BWalker& wk = B.walkers[w];
    if (tid < MAXCV) { sCV[tid] = 0.0; sdU[tid] = 0.0; }
    __syncthreads();
    if (tid < B.nS) {
        const BSimple& si = B.simple[w * B.nS + tid];
        F3 jac[4];
        float v = simpleCV(si.type, si.atoms, wk.posq, nullptr, wk.box, jac);
        for (int k = 0; k < 4; k++) sJac[tid * 4 + k] = jac[k];
        sCV[si.cv] = (double)v;
    }
    if (warp == 1) {
        for (int c = 0; c < B.nC; c++) {
            const CoordItem& it = B.C.items[w * B.nC + c];
            int nb = it.tilesA * it.splitsB;
            double s = 0;
            for (int k = lane; k < nb; k += 32) s += B.C.cnPart[it.cn0 + k];
            s = warpSum(s);
            if (lane == 0) sCV[it.cv] = s;
        }
    }
    if (warp == 2 && B.hill.present) {
        double v[3] = {0, 0, 0};
        for (int h = lane; h < B.hillItems; h += 32) {
            const double* p = B.hillPart + 3 * ((size_t)h * B.W + w);
            v[0] += p[0]; v[1] += p[1]; v[2] += p[2];
        }
        for (int k = 0; k < 3; k++) v[k] = warpSum(v[k]);
        if (lane == 0) { sScal[0] = v[0]; sScal[1] = v[1]; sScal[2] = v[2]; }
    }
    __syncthreads();
    if (tid == 0) {
        const double TWO_PI = 6.283185307179586;
        double E = 0.0;
        for (int k = 0; k < B.nH; k++) {
            const BHarm& hm = B.harm[w * B.nH + k];
            double ds = sCV[hm.cv] - (double)hm.at;
            if (hm.periodic) ds -= TWO_PI * round(ds / TWO_PI);
            E += 0.5 * (double)hm.k * ds * ds;
            sdU[hm.cv] += (double)hm.k * ds;
        }
        if (B.hill.present) {
            E += sScal[0];
            sdU[B.hill.cv[0]] += sScal[1];
            if (B.hill.D > 1) sdU[B.hill.cv[1]] += sScal[2];
        }
        if (part == 0) {
            for (int k = 0; k < B.nCV; k++) B.cvv[(size_t)w * B.nCV + k] = sCV[k];
            B.energy[w] = E;
            B.hillEnergy[w] = B.hill.present ? sScal[0] : 0.0;
        }
    }
    __syncthreads();
    const double S = 4294967296.0;
    unsigned long long* F = wk.force;
    const int P = wk.padded;
    if (part == 0 && tid < B.nS * 4) {
        const BSimple& si = B.simple[w * B.nS + tid / 4];
        const int k = tid % 4;
        const int na = si.type == 1 ? 2 : si.type == 2 ? 3 : 4;
        const double g = sdU[si.cv];
        if (k < na && g != 0.0) {
            F3 j = sJac[tid];
            int a = si.atoms[k];
            atomicAdd(F + a, (unsigned long long)(long long)(-(g * (double)j.x) * S));
            atomicAdd(F + a + P, (unsigned long long)(long long)(-(g * (double)j.y) * S));
            atomicAdd(F + a + 2 * P, (unsigned long long)(long long)(-(g * (double)j.z) * S));
        }
    }
    for (int c = 0; c < B.nC; c++) {
        const CoordItem& it = B.C.items[w * B.nC + c];
        const double g = sdU[it.cv];
        if (g == 0.0) continue;
        const int R = it.nA + it.nB;
        const int r0 = (int)((long long)R * part / B.parts), r1 = (int)((long long)R * (part + 1) / B.parts);
        for (int i = r0 + tid; i < r1; i += blockDim.x) {
            double x = 0, y = 0, z = 0;
            int atom;
            if (i < it.nA) {
                const float* p = B.C.partA + 3 * ((size_t)it.partA + i);
                for (int sb = 0; sb < it.splitsB; sb++) {
                    const float* q = p + 3 * (size_t)sb * it.nA;
                    x += q[0]; y += q[1]; z += q[2];
                }
                atom = B.C.atoms[it.a0 + i];
            } else {
                const int b = i - it.nA;
                const float* p = B.C.partB + 3 * ((size_t)it.partB + b);
                for (int ta = 0; ta < it.tilesA; ta++) {
                    const float* q = p + 3 * (size_t)ta * it.nB;
                    x += q[0]; y += q[1]; z += q[2];
                }
                atom = B.C.atoms[it.b0 + b];
            }
            // Same rounding as the per-context path: the gradient is stored as float.
            const float gx = (float)x, gy = (float)y, gz = (float)z;
            atomicAdd(F + atom, (unsigned long long)(long long)(-(g * (double)gx) * S));
            atomicAdd(F + atom + P, (unsigned long long)(long long)(-(g * (double)gy) * S));
            atomicAdd(F + atom + 2 * P, (unsigned long long)(long long)(-(g * (double)gz) * S));
        }
    }
    __syncthreads();
}

// ------------------------------------------------------------- the step
template <int RA, int BOX, int NH>
__global__ void __launch_bounds__(256, 2) k_batch_step(BatchDev B) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ int sItem;
    __shared__ double red[32];
    __shared__ __align__(8) unsigned long long mbar;
    const int tid = threadIdx.x;
    const int numA = B.coordBlocks + B.hillItems * B.nWB;
    unsigned long long* stamp = B.stamps ? B.stamps + 6 * (size_t)blockIdx.x : nullptr;
    int nCoord = 0, nHill = 0;
    if (stamp && tid == 0) stamp[0] = globalTimer();
    for (;;) {
        if (tid == 0) sItem = atomicAdd(B.work, 1);
        __syncthreads();
        const int item = sItem;
        __syncthreads();
        if (item >= numA) break;
        if (item < B.coordBlocks) {
            const int ci = B.C.blockItem[item];
            const CoordItem it = B.C.items[ci];
            const BWalker& wk = B.walkers[ci / B.nC];
            const BoxDev box = wk.box;
            const int local = item - it.block0;
            const int ta = local / it.splitsB, sb = local % it.splitsB;
            float (*sB)[TB * 3] = reinterpret_cast<float (*)[TB * 3]>(smem);
            coordTile<RA, BOX, NH>(wk.posq, nullptr, B.C, it, ta, sb, box, sB, red);
            __syncthreads();
            nCoord++;
        } else {
            hillItem(B, item - B.coordBlocks, smem, &mbar);
            nHill++;
        }
    }
    if (stamp && tid == 0) { stamp[1] = globalTimer(); stamp[4] = nCoord; stamp[5] = nHill; }
    if (!gridBarrier(B.bar, B.status, B.spinLimit)) return;
    if (stamp && tid == 0) stamp[2] = globalTimer();
    if (blockIdx.x == 0 && tid == 0) *B.work = 0;
    for (int p = blockIdx.x; p < B.W * B.parts; p += gridDim.x) finalizeWalker(B, p / B.parts, p % B.parts, smem);
    if (stamp && tid == 0) stamp[3] = globalTimer();
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

typedef void (*StepFn)(BatchDev);

template <int RA, int NH>
StepFn stepKernelB(int box) {
    return box == 0 ? k_batch_step<RA, 0, NH> : box == 1 ? k_batch_step<RA, 1, NH> : k_batch_step<RA, 2, NH>;
}

template <int RA>
StepFn stepKernelK(int box, int kind) {
    return kind == 3 ? stepKernelB<RA, 3>(box) : kind == -1 ? stepKernelB<RA, -1>(box) : stepKernelB<RA, 0>(box);
}

StepFn stepKernel(int ra, int box, int kind) {
    return ra == 4 ? stepKernelK<4>(box, kind) : stepKernelK<8>(box, kind);
}

// ================================================================== host
struct Batch::Impl {
    int W = 0, nCV = 0, nS = 0, nC = 0, nH = 0, boxKind = 1, kind = 3;
    std::vector<BWalker> walkersH;
    std::vector<CoordItem> items;
    std::vector<int> coordAtoms;
    DBuf walkersD, simpleD, harmD, itemsD, atomsD, blockItemD, partA, partB, cnPart, hillPart;
    DBuf cvv, energy, hillEnergy, bar, work, status, scratchForce;
    DBuf hMirror, hCenters, hHeights, hCount;
    BHill hill{};
    BatchTuning tune;
    BatchDev dev{};
    int grid = 0;
    cudaStream_t stream = 0;
    cudaStream_t cap = nullptr;
    cudaGraphExec_t graph = nullptr;
    long long launches = 0;
    int lastUpdateStep = -1;
    bool ready = false;
    bool useGraph = true;
    float lastMs = 0;

    void destroyGraph() {
        if (graph) { cudaGraphExecDestroy(graph); graph = nullptr; }
    }

    void plan() {
        const int TA = 8 * tune.ra;
        int blocks = 0, pa = 0, pb = 0, cn = 0;
        std::vector<int> blockItem;
        for (size_t i = 0; i < items.size(); i++) {
            CoordItem& it = items[i];
            it.tilesA = std::max(1, (it.nA + TA - 1) / TA);
            it.splitsB = std::max(1, (it.nB + tune.bSplit - 1) / tune.bSplit);
            it.block0 = blocks;
            it.partA = pa; it.partB = pb; it.cn0 = cn;
            const int nb = it.tilesA * it.splitsB;
            blocks += nb; cn += nb;
            pa += it.splitsB * it.nA; pb += it.tilesA * it.nB;
        }
        // heavy items first: order the coordination blocks walker-interleaved
        blockItem.resize(blocks);
        for (size_t i = 0; i < items.size(); i++)
            for (int k = 0; k < items[i].tilesA * items[i].splitsB; k++) blockItem[items[i].block0 + k] = (int)i;
        itemsD.upload(items);
        blockItemD.upload(blockItem);
        if (partA.bytes < sizeof(float) * 3 * (size_t)std::max(pa, 1)) partA.alloc(sizeof(float) * 3 * std::max(pa, 1));
        if (partB.bytes < sizeof(float) * 3 * (size_t)std::max(pb, 1)) partB.alloc(sizeof(float) * 3 * std::max(pb, 1));
        if (cnPart.bytes < sizeof(double) * (size_t)std::max(cn, 1)) cnPart.alloc(sizeof(double) * std::max(cn, 1));
        const int nWB = (W + WBLK - 1) / WBLK;
        size_t hp = sizeof(double) * 3 * (size_t)tune.hillItems * W;
        if (hillPart.bytes < hp) hillPart.alloc(hp);
        dev.walkers = walkersD.as<BWalker>();
        dev.W = W; dev.nCV = nCV; dev.nS = nS; dev.nC = nC; dev.nH = nH;
        dev.simple = simpleD.as<BSimple>();
        dev.harm = harmD.as<BHarm>();
        dev.C.items = itemsD.as<CoordItem>();
        dev.C.numItems = (int)items.size();
        dev.C.atoms = atomsD.as<int>();
        dev.C.blockItem = blockItemD.as<int>();
        dev.C.partA = partA.as<float>(); dev.C.partB = partB.as<float>(); dev.C.cnPart = cnPart.as<double>();
        dev.C.bSplit = tune.bSplit;
        dev.coordBlocks = blocks;
        dev.hillItems = hill.present ? tune.hillItems : 0;
        dev.nWB = hill.present ? nWB : 0;
        dev.parts = tune.parts;
        dev.hill = hill;
        dev.hillPart = hillPart.as<double>();
        dev.cvv = cvv.as<double>(); dev.energy = energy.as<double>(); dev.hillEnergy = hillEnergy.as<double>();
        dev.bar = bar.as<unsigned int>(); dev.work = work.as<int>(); dev.status = status.as<int>();
        dev.spinLimit = 1ull << 24;
        cudaCheck(cudaMemset(bar.p, 0, bar.bytes), "reset");
        cudaCheck(cudaMemset(work.p, 0, work.bytes), "reset");
        cudaCheck(cudaMemset(status.p, 0, status.bytes), "reset");
        StepFn fn = stepKernel(tune.ra, boxKind, kind);
        int dev_ = 0, sms = 0, perSM = 0;
        cudaCheck(cudaGetDevice(&dev_), "device");
        cudaCheck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev_), "attr");
        cudaCheck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, (const void*)fn, 256, SMEM_BYTES), "occupancy");
        if (perSM < 1) throw Error(GLUED_E_CUDA, "batched step kernel cannot be resident");
        grid = sms * perSM;
        destroyGraph();
    }

    void launch(cudaStream_t s) {
        StepFn fn = stepKernel(tune.ra, boxKind, kind);
        void* args[] = {&dev};
        cudaCheck(cudaLaunchCooperativeKernel((const void*)fn, dim3(grid), dim3(256), args, SMEM_BYTES, s),
                  "cooperative launch");
    }
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
    I.bar.alloc(sizeof(unsigned int) * 4);
    I.work.alloc(sizeof(int) * 4);
    I.status.alloc(sizeof(int) * 4);
    cudaCheck(cudaStreamCreateWithFlags(&I.cap, cudaStreamNonBlocking), "stream");
    for (int r : {4, 8}) {
        StepFn fn = stepKernel(r, I.boxKind, I.kind);
        cudaCheck(cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES), "attr");
    }
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
    if (t.ra != 4 && t.ra != 8) throw Error(GLUED_E_INVALID, "batch tuning: ra must be 4 or 8");
    if (t.bSplit < 128 || t.bSplit % 128) throw Error(GLUED_E_INVALID, "batch tuning: bSplit must be a multiple of 128");
    if (t.hillItems < 1 || t.parts < 1) throw Error(GLUED_E_INVALID, "batch tuning: hillItems and parts must be >= 1");
    cudaCheck(cudaStreamSynchronize(impl_->stream), "sync");
    impl_->tune = t;
    impl_->plan();
}

BatchTuning Batch::tuning() const { return impl_->tune; }

void Batch::execute() {
    Impl& I = *impl_;
    if (!I.graph && I.useGraph) {
        cudaGraph_t g = nullptr;
        bool ok = cudaStreamBeginCapture(I.cap, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
        if (ok) {
            StepFn fn = stepKernel(I.tune.ra, I.boxKind, I.kind);
            void* args[] = {&I.dev};
            cudaError_t le = cudaLaunchCooperativeKernel((const void*)fn, dim3(I.grid), dim3(256), args, SMEM_BYTES, I.cap);
            cudaError_t ce = cudaStreamEndCapture(I.cap, &g);
            ok = le == cudaSuccess && ce == cudaSuccess && g &&
                 cudaGraphInstantiate(&I.graph, g, 0) == cudaSuccess;
            if (g) cudaGraphDestroy(g);
        }
        if (!ok) {
            // cooperative launches are not capturable here: launch directly
            cudaGetLastError();
            I.graph = nullptr;
            I.useGraph = false;
        }
    }
    if (I.graph) cudaCheck(cudaGraphLaunch(I.graph, I.stream), "graph launch");
    else I.launch(I.stream);
    I.launches++;
    I.ready = true;
}

// Autotuner: tile shape, B split, hill items and finalize parts are timed on
// the live walkers with CUDA events (forces go to a scratch buffer) and the
// fastest combination is kept.
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
    for (int ra : {4, 8})
        for (int bs : {128, 256, 512})
            for (int hi : {32, 64, 128, 256})
                for (int parts : {2, 4, 8}) {
                    BatchTuning t;
                    t.ra = ra; t.bSplit = bs; t.hillItems = hi; t.parts = parts;
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
                    I.launches += reps + 2;
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
void Batch::phaseTimes(double* out) {
    Impl& I = *impl_;
    DBuf st;
    st.alloc(sizeof(unsigned long long) * 6 * (size_t)I.grid);
    cudaCheck(cudaMemsetAsync(st.p, 0, st.bytes, I.stream), "stamps");
    I.dev.stamps = st.as<unsigned long long>();
    I.launch(I.stream);
    I.dev.stamps = nullptr;
    I.launches++;
    I.ready = true;
    std::vector<unsigned long long> h(6 * (size_t)I.grid);
    cudaCheck(cudaStreamSynchronize(I.stream), "sync");
    cudaCheck(cudaMemcpy(h.data(), st.p, st.bytes, cudaMemcpyDeviceToHost), "stamps");
    unsigned long long t0 = ~0ull, aMin = ~0ull, aMax = 0, bMax = 0, eMax = 0;
    long long nc = 0, nh = 0, most = 0, fewest = 1ll << 40;
    for (int g = 0; g < I.grid; g++) {
        const unsigned long long* r = h.data() + 6 * (size_t)g;
        t0 = std::min(t0, r[0]);
        aMin = std::min(aMin, r[1]); aMax = std::max(aMax, r[1]);
        bMax = std::max(bMax, r[2]); eMax = std::max(eMax, r[3]);
        nc += (long long)r[4]; nh += (long long)r[5];
        most = std::max(most, (long long)(r[4] + r[5]));
        fewest = std::min(fewest, (long long)(r[4] + r[5]));
    }
    out[0] = (aMin - t0) * 1e-3; out[1] = (aMax - t0) * 1e-3;
    out[2] = (bMax - t0) * 1e-3; out[3] = (eMax - t0) * 1e-3;
    out[4] = (double)nc; out[5] = (double)nh; out[6] = (double)most; out[7] = (double)fewest;
    int s = status();
    if (s) throw Error(GLUED_E_TIMEOUT, "batch: bounded wait gave up (status " + std::to_string(s) + ")");
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
    std::vector<float4> m(n);
    for (int k = 0; k < n; k++)
        m[k] = make_float4((float)centers[k * D], D > 1 ? (float)centers[k * D + 1] : 0.0f, (float)heights[k], 0.0f);
    if (n > 0) {
        cudaCheck(cudaMemcpy(I.hill.centers, centers, sizeof(double) * (size_t)n * D, cudaMemcpyHostToDevice), "hills");
        cudaCheck(cudaMemcpy(I.hill.heights, heights, sizeof(double) * n, cudaMemcpyHostToDevice), "hills");
        cudaCheck(cudaMemcpy(I.hill.mirror, m.data(), sizeof(float4) * n, cudaMemcpyHostToDevice), "hills");
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
