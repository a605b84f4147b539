// Coordination pairs as static per-CTA runs of (item, A tile, B chunk) steps.
//
// Work decomposition. Every coordination item (one CV of one system) is cut into
// A tiles of TA = NW*RA atoms (NW = 16 warps, RA A atoms per warp: 8 by default,
// 128 atoms) and B chunks of CH = 32*RB atoms (RB B atoms per lane: 4 by
// default, 128 atoms); one step is one (tile, chunk) block of TA x CH pairs. The
// batched path instantiates other (RA, RB) shapes for its autotuner. The host
// lists the steps tile-major (CoordStep) and gives every CTA of a persistent grid
// of one 512-thread CTA per SM one contiguous range of them with the same number
// of steps. One CTA per SM, its warps meeting at a barrier every step, keeps
// every warp of the SM at the same pace (with two CTAs per SM the scheduler let
// one run ahead and the other finish alone). A CTA walks its range once: A atoms
// stay in registers while consecutive steps belong to the same tile.
//
// Data movement. Positions are gathered with 16-byte cp.async copies into
// shared memory two steps ahead (double buffer), so a step computes while the
// next one lands; gather indices for step s+2 are loaded into registers before
// step s computes and the copies are issued after its barrier. Step descriptors
// of a window of up to WIN steps sit in shared memory.
//
// Arithmetic. Coordinates are scaled by 1/r0 (A once per tile, B once per step,
// both rounded the same way, never contracted), so the pair's squared distance is
// x^2 directly and an atom present in both groups gives exactly zero. For the
// n = 6, m = 12 switch, f = 1/(1 + x^6) and the gradient factor h = x^4 f^2 need
// one reciprocal and no square root; full steps of that switch use packed FP32
// (f32x2) instructions, two pairs per instruction. The reference's lower bound
// r^2 >= 1e-20 (CommonGluedKernels.cpp:983-987) is compared on every pair; the
// upper bound x <= 1000 (and the optional cutoff) only where the box admits such
// distances (template flag HI).
//
// Accumulation. Per-pair gradients h*d (scaled units) are summed in FP32 over a
// step: per lane over its A atoms for B, per warp over lanes for A (one butterfly
// for all A atoms of the warp). The A sums run in registers over the whole tile
// run (its steps = the B group in chunks of CH) and are reduced once at its end;
// with BLK (blocked sums) they are reduced and flushed every BLK_STEPS steps
// instead, so that no FP32 partial holds more than 4 * BLK_STEPS pairs per lane
// (a register-resident two-sum would need 48 more registers per thread, and the
// kernel is at the 128 of one 512-thread CTA per SM). Those sums are converted to 64-bit fixed point
// (value * 2^32) and added with integer atomics into acc[row][3] (integer
// addition is exact and order-independent, so the sums are bitwise reproducible
// and do not depend on the grid); the reader multiplies by the item's scale
// (-n/r0 for the n = 6, m = 12 switch, 1/r0 otherwise), converts to FP64 and
// clears the rows. The CN partial of each run piece (a maximal sub-run of one
// tile on one CTA; FP64 block sum) goes to the slot the host assigned to the
// piece (CoordStep::pieceSlot of its last step); an item's slots are contiguous
// and in step order, the reader sums them in that order, and nothing needs
// clearing.
#pragma once

#include "devfn.cuh"

namespace glued {

namespace crun {
constexpr int NW = COORD_NW;   // warps per CTA
constexpr int WIN = 64;        // step descriptors per shared-memory window
constexpr int BLK_STEPS = 8;   // steps per A partial with blocked sums
constexpr float FX = 4294967296.0f;   // 2^32
constexpr double FXD = 4294967296.0;
constexpr double IFXD = 1.0 / 4294967296.0;
constexpr int F_FIRST = COORD_F_FIRST, F_LAST = COORD_F_LAST;
}  // namespace crun

// Pair constants of one item in scaled units (coordinates divided by r0).
struct alignas(16) RunConst {
    float lo, hi;       // valid pairs: lo <= x^2 < hi
    float n, m;         // general exponents (kind 0)
    int ni, mi;         // integer exponents (kind -1)
    float ir0;
    BoxDev box;         // scaled: a, b, c divided by r0; inv multiplied by r0
};

// Shared memory of a run with A tiles of NW * RA atoms and B chunks of 32 * RB.
template <int RA, int RB>
struct CoordRunSmem {
    float4 pos[2][32 * RB];
    float4 apos[2][crun::NW * RA];
    float g[2][crun::NW][32 * RB * 3];
    CoordStep st[crun::WIN];
    alignas(16) RunConst kst[crun::WIN];   // constants of the window's steps (those that start a tile run)
    double red[2][crun::NW];
};

__device__ __forceinline__ unsigned smemU32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

// 16-byte global -> shared copy; valid == false writes zeros (nothing is read).
__device__ __forceinline__ void cpAsync16(void* dst, const void* src, bool valid) {
    unsigned n = valid ? 16u : 0u;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smemU32(dst)), "l"(src), "r"(n) : "memory");
}
// 16-byte global -> shared copy of which the first `bytes` (0..16, multiple of
// 4) are read and the rest written as zeros.
__device__ __forceinline__ void cpAsyncBytes(void* dst, const void* src, int bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smemU32(dst)), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cpAsyncCommit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cpAsyncWaitAll() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

__device__ __forceinline__ void redAddI64(unsigned long long* p, long long v) {
    redAddGlobal(p, (unsigned long long)v);
}

__device__ __forceinline__ RunConst runConst(const CoordItem& it, const BoxDev& b) {
    RunConst k;
    k.ir0 = 1.0f / it.r0;
    const float ir0sq = k.ir0 * k.ir0;
    k.lo = 1e-20f * ir0sq;
    const float hiX = 1e6f * 1.0000002f;
    k.hi = it.rc2 > 0.0f ? fminf(it.rc2 * ir0sq, hiX) : hiX;
    k.n = it.n; k.m = it.m;
    k.ni = (int)it.n; k.mi = (int)it.m;
    k.box = b;
    for (int i = 0; i < 3; i++) {
        k.box.a[i] = b.a[i] * k.ir0; k.box.b[i] = b.b[i] * k.ir0; k.box.c[i] = b.c[i] * k.ir0;
        k.box.inv[i] = b.inv[i] * it.r0;
    }
    return k;
}

// Minimum image of a scaled difference (same rounding as imageT in coord_tile.cuh).
template <int BOX>
__device__ __forceinline__ void imageS(float& dx, float& dy, float& dz, const BoxDev& b) {
    constexpr float R = 12582912.0f;
    if (BOX == 1) {
        dx = fmaf(-(fmaf(dx, b.inv[0], R) - R), b.a[0], dx);
        dy = fmaf(-(fmaf(dy, b.inv[1], R) - R), b.b[1], dy);
        dz = fmaf(-(fmaf(dz, b.inv[2], R) - R), b.c[2], dz);
    } else if (BOX == 2) {
        float s3 = fmaf(dz, b.inv[2], R) - R;
        dx = fmaf(-s3, b.c[0], dx); dy = fmaf(-s3, b.c[1], dy); dz = fmaf(-s3, b.c[2], dz);
        float s2 = fmaf(dy, b.inv[1], R) - R;
        dx = fmaf(-s2, b.b[0], dx); dy = fmaf(-s2, b.b[1], dy);
        float s1 = fmaf(dx, b.inv[0], R) - R;
        dx = fmaf(-s1, b.a[0], dx);
    }
}

// f and h = (df/dx)/x of one pair from x^2 (scaled). For NH > 0 (m = 2n, n = 2NH)
// the bounds are applied by the caller; for the other kinds `valid` gates the
// pair and must already include the bounds.
template <int NH>
__device__ __forceinline__ void switchX2(float x2, bool valid, const RunConst& k, float& f, float& h) {
    if (NH > 0) {
        float p = 1.0f;
#pragma unroll
        for (int e = 1; e < NH; e++) p = e == 1 ? x2 : p * x2;
        float y = valid ? fmaf(p, x2, 1.0f) : __int_as_float(0x7f800000);
        float ff;
        asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(ff) : "f"(y));
        f = ff;
        h = (p * ff) * ff;
    } else if (NH < 0) {
        float x = sqrtf(x2);
        float ff, dfdx;
        ratioSwitch(x, k.ni, k.mi, ff, dfdx);
        f = valid ? ff : 0.0f;
        h = valid ? dfdx / x : 0.0f;
    } else {
        // Non-integer exponents: the reference formula (Taylor branch within
        // 1e-4 of x = 1, CommonGluedKernels.cpp:983-1003) evaluated in FP64; in
        // FP32 the quotient (1 - x^n)/(1 - x^m) loses up to ~1e-2 relative force
        // accuracy through cancellation just outside the Taylor window.
        const double x = sqrt((double)x2);
        const double n = k.n, m = k.m;
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
        h = valid ? (float)(dfdx / x) : 0.0f;
    }
}

// Scale that turns an acc sum into dCN/dx (nm^-1) for the item's switch kind.
__device__ __host__ __forceinline__ double coordAccScale(const CoordItem& it) {
    return it.kind > 0 ? -(double)it.n / (double)it.r0 : 1.0 / (double)it.r0;
}

// Packed FP32 (f32x2, sm_100): one instruction operates on two floats held in
// a 64-bit register pair. These halve the issue slots of the pair arithmetic;
// the FP32 pipe throughput per element is unchanged.
namespace f2 {
__device__ __forceinline__ unsigned long long pk(float a, float b) {
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ void upk(unsigned long long v, float& a, float& b) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
}
__device__ __forceinline__ unsigned long long fma(unsigned long long a, unsigned long long b, unsigned long long c) {
    unsigned long long d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ unsigned long long add(unsigned long long a, unsigned long long b) {
    unsigned long long d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ unsigned long long sub(unsigned long long a, unsigned long long b) {
    unsigned long long d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ unsigned long long mul(unsigned long long a, unsigned long long b) {
    unsigned long long d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
}  // namespace f2

// Image constants of a step in packed form (both halves equal).
struct PackedConst {
    unsigned long long ivx, ivy, ivz, nLx, nLy, nLz;
};
__device__ __forceinline__ PackedConst packedConst(const RunConst& K) {
    PackedConst c;
    c.ivx = f2::pk(K.box.inv[0], K.box.inv[0]); c.ivy = f2::pk(K.box.inv[1], K.box.inv[1]);
    c.ivz = f2::pk(K.box.inv[2], K.box.inv[2]);
    c.nLx = f2::pk(-K.box.a[0], -K.box.a[0]); c.nLy = f2::pk(-K.box.b[1], -K.box.b[1]);
    c.nLz = f2::pk(-K.box.c[2], -K.box.c[2]);
    return c;
}

// The pairs of one full step (TA x CH, switch m = 2n = 4 NH) with packed
// arithmetic: A atoms (2i, 2i+1) of the warp are one packed operand (apx[i], ...,
// kept packed across steps), each B atom is broadcast (negated) into both
// halves, and the B atoms of the lane are taken two at a time so that their
// packed gradient partials fit in registers. Same per-pair operations and
// bounds as the scalar loop; B-gradient and CN sums are kept as two partials
// (even / odd A atoms) and added at the end of the step. Writes the warp's B
// partials to gw (negated sums) and adds the step's CN to cnc.
template <int RA, int RB, int BOX, int NH, bool HI>
__device__ __forceinline__ void pairsPacked(const unsigned long long (&apx)[RA / 2],
                                            const unsigned long long (&apy)[RA / 2],
                                            const unsigned long long (&apz)[RA / 2], unsigned long long (&gpx)[RA / 2],
                                            unsigned long long (&gpy)[RA / 2], unsigned long long (&gpz)[RA / 2],
                                            const float4* pos, const RunConst& K, float* gw, float& cnc) {
    static_assert(RA % 2 == 0 && NH > 0 && BOX != 2, "packed pair block");
    constexpr float R = 12582912.0f;   // 1.5 * 2^23: adding and removing it rounds to an integer
    const int lane = threadIdx.x & 31;
    const unsigned long long R2 = f2::pk(R, R), ONE2 = f2::pk(1.0f, 1.0f);
    const PackedConst C = packedConst(K);
    const float INF = __int_as_float(0x7f800000);
    unsigned long long cn2 = 0ull;
#pragma unroll
    for (int half = 0; half < RB / 2; half++) {
        unsigned long long nbx[2], nby[2], nbz[2], gbx[2], gby[2], gbz[2];
#pragma unroll
        for (int jj = 0; jj < 2; jj++) {
            const float4 p = pos[lane + 32 * (2 * half + jj)];
            const float x = -__fmul_rn(p.x, K.ir0), y = -__fmul_rn(p.y, K.ir0), z = -__fmul_rn(p.z, K.ir0);
            nbx[jj] = f2::pk(x, x); nby[jj] = f2::pk(y, y); nbz[jj] = f2::pk(z, z);
            gbx[jj] = gby[jj] = gbz[jj] = 0ull;
        }
#pragma unroll
        for (int i = 0; i < RA / 2; i++) {
#pragma unroll
            for (int jj = 0; jj < 2; jj++) {
                unsigned long long dx = f2::add(apx[i], nbx[jj]), dy = f2::add(apy[i], nby[jj]),
                                   dz = f2::add(apz[i], nbz[jj]);
                if (BOX == 1) {
                    dx = f2::fma(f2::sub(f2::fma(dx, C.ivx, R2), R2), C.nLx, dx);
                    dy = f2::fma(f2::sub(f2::fma(dy, C.ivy, R2), R2), C.nLy, dy);
                    dz = f2::fma(f2::sub(f2::fma(dz, C.ivz, R2), R2), C.nLz, dz);
                }
                const unsigned long long x2 = f2::fma(dz, dz, f2::fma(dy, dy, f2::mul(dx, dx)));
                unsigned long long pw = NH == 1 ? ONE2 : x2;
#pragma unroll
                for (int e = 2; e < NH; e++) pw = f2::mul(pw, x2);
                const unsigned long long yy = f2::fma(pw, x2, ONE2);
                float xa, xb, ya, yb;
                f2::upk(x2, xa, xb);
                f2::upk(yy, ya, yb);
                ya = (HI ? (xa >= K.lo && xa < K.hi) : (xa >= K.lo)) ? ya : INF;
                yb = (HI ? (xb >= K.lo && xb < K.hi) : (xb >= K.lo)) ? yb : INF;
                float fa, fb;
                asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(fa) : "f"(ya));
                asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(fb) : "f"(yb));
                const unsigned long long ff = f2::pk(fa, fb);
                const unsigned long long h = f2::mul(f2::mul(pw, ff), ff);
                cn2 = f2::add(cn2, ff);
                gpx[i] = f2::fma(h, dx, gpx[i]); gpy[i] = f2::fma(h, dy, gpy[i]); gpz[i] = f2::fma(h, dz, gpz[i]);
                gbx[jj] = f2::fma(h, dx, gbx[jj]); gby[jj] = f2::fma(h, dy, gby[jj]); gbz[jj] = f2::fma(h, dz, gbz[jj]);
            }
        }
#pragma unroll
        for (int jj = 0; jj < 2; jj++) {
            const int o = (lane + 32 * (2 * half + jj)) * 3;
            float a, c;
            f2::upk(gbx[jj], a, c); gw[o] = -(a + c);
            f2::upk(gby[jj], a, c); gw[o + 1] = -(a + c);
            f2::upk(gbz[jj], a, c); gw[o + 2] = -(a + c);
        }
    }
    float c0, c1;
    f2::upk(cn2, c0, c1);
    cnc += c0 + c1;
}

struct NoPieceHook {
    __device__ void operator()(int, int) const {}
};
struct NoStartHook {
    __device__ void operator()() const {}
};

// Runs steps [s0, s1) of R on this CTA. Hook(item, steps) is called by all
// threads after a piece (maximal sub-run of one tile) has been fully
// accumulated; a hook that publishes completion must fence first. Start() is
// called once by all threads when the copies issued before the call and those
// of the first two steps have landed (after a barrier), before the first step
// computes: cp.async copies it issues land while that step computes and are
// complete after its end-of-step wait. AfterFirst() is called once by all
// threads right after the first step's end-of-step barrier (everything Start()
// issued has landed and is visible).
template <int RA, int RB, int BOX, int NH, bool HI, bool BLK, class Hook, class Start = NoStartHook,
          class AfterFirst = NoStartHook>
__device__ void coordRun(const CoordRunDev& R, int s0, int s1, CoordRunSmem<RA, RB>& sm, const Hook& hook,
                         const Start& start = Start(), const AfterFirst& afterFirst = AfterFirst()) {
    using namespace crun;
    static_assert(RA % 2 == 0 && 3 * RA <= 32, "A atoms per warp");
    static_assert(RB % 2 == 0 && RB >= 2, "B atoms per lane");
    constexpr int TA = NW * RA;
    constexpr int CH = 32 * RB;
    static_assert(TA <= COORD_TA_MAX && CH <= COORD_CH_MAX, "step packing");
    constexpr int RH = RA / 2;
    const int tid = threadIdx.x, lane = tid & 31, ty = tid >> 5;
    // A atoms 2i, 2i+1 of the warp (scaled) and their gradient sums, packed
    unsigned long long apx[RH], apy[RH], apz[RH], gpx[RH], gpy[RH], gpz[RH];
    RunConst K;
    double cn = 0.0;
    int pieceSteps = 0;
    for (int w0 = s0; w0 < s1; w0 += WIN) {
        const int w1 = min(s1, w0 + WIN);
        const int nw = w1 - w0;
        __syncthreads();  // previous window fully consumed
        // gather indices of step w0 + ls from the per-step tables (no other load
        // first): B (threads < CH) and A (threads < TA; -1: no A gather)
        auto loadIdx = [&](int ls, int& ib, int& ia, const float4*& pq) {
            const size_t s = (size_t)(w0 + ls);
            ib = tid < CH ? __ldg(R.gB + s * CH + tid) : -1;
            ia = tid < TA ? __ldg(R.gA + s * TA + tid) : -1;
            pq = R.stepPosq[s];
        };
        auto issue = [&](int ls, int ib, int ia, const float4* pq) {
            const int b = (w0 + ls - s0) & 1;
            if (tid < CH) cpAsync16(&sm.pos[b][tid], pq + (ib >= 0 ? ib : 0), ib >= 0);
            if (tid < TA && ia != -1) cpAsync16(&sm.apos[b][tid], pq + (ia >= 0 ? ia : 0), ia >= 0);
            cpAsyncCommit();
        };
        if (R.stepConst) {
            // constants precomputed per step: the step records and constants of the
            // window are copied along with the first two steps' gathers (nothing
            // to wait for before issuing them), one round trip after the indices
            const int4* src = reinterpret_cast<const int4*>(R.steps + w0);
            for (int i = tid; i < nw * 2; i += blockDim.x) cpAsync16(reinterpret_cast<int4*>(sm.st) + i, src + i, true);
            constexpr int W16 = (int)(sizeof(RunConst) / 16);
            const int4* cs = reinterpret_cast<const int4*>(R.stepConst + w0);
            for (int i = tid; i < nw * W16; i += blockDim.x)
                cpAsync16(reinterpret_cast<int4*>(sm.kst) + i, cs + i, true);
            int ib0, ia0, ib1 = -1, ia1 = -1;
            const float4 *pq0, *pq1 = nullptr;
            loadIdx(0, ib0, ia0, pq0);
            if (nw > 1) loadIdx(1, ib1, ia1, pq1);
            issue(0, ib0, ia0, pq0);
            if (nw > 1) issue(1, ib1, ia1, pq1);
        } else {
            // the window's first two steps: gathers first, then the step records
            // (both independent), then the constants of the steps that start a
            // tile run, while the gathers land
            {
                int ib0, ia0, ib1 = -1, ia1 = -1;
                const float4 *pq0, *pq1 = nullptr;
                loadIdx(0, ib0, ia0, pq0);
                if (nw > 1) loadIdx(1, ib1, ia1, pq1);
                issue(0, ib0, ia0, pq0);
                if (nw > 1) issue(1, ib1, ia1, pq1);
            }
            {
                const int4* src = reinterpret_cast<const int4*>(R.steps + w0);
                int4* dst = reinterpret_cast<int4*>(sm.st);
                for (int i = tid; i < nw * 2; i += blockDim.x) dst[i] = __ldg(src + i);
            }
            __syncthreads();
            for (int i = tid; i < nw; i += blockDim.x) {
                const CoordStep& d = sm.st[i];
                if (w0 + i == s0 || i == 0 || (stepFlags(d.packed) & F_FIRST))
                    sm.kst[i] = runConst(R.items[d.item], R.sysBox[d.sys]);
            }
        }
        cpAsyncWaitAll();
        __syncthreads();
        if (w0 == s0) start();
        for (int ls = 0; ls < nw; ls++) {
            const int s = w0 + ls;
            const int b = (s - s0) & 1;
            const CoordStep d = sm.st[ls];
            const int nAv = stepNA(d.packed), nBv = stepNB(d.packed), fl = stepFlags(d.packed);
            const bool first = (s == s0) || (fl & F_FIRST);
            const bool last = (s == s1 - 1) || (fl & F_LAST);
            int ib2 = -1, ia2 = -1;
            const float4* pq2 = nullptr;
            if (ls + 2 < nw) loadIdx(ls + 2, ib2, ia2, pq2);
            if (first) {
                K = sm.kst[ls];
#pragma unroll
                for (int i = 0; i < RH; i++) {
                    const float4 p = sm.apos[b][ty + NW * (2 * i)], q = sm.apos[b][ty + NW * (2 * i + 1)];
                    apx[i] = f2::pk(__fmul_rn(p.x, K.ir0), __fmul_rn(q.x, K.ir0));
                    apy[i] = f2::pk(__fmul_rn(p.y, K.ir0), __fmul_rn(q.y, K.ir0));
                    apz[i] = f2::pk(__fmul_rn(p.z, K.ir0), __fmul_rn(q.z, K.ir0));
                    gpx[i] = gpy[i] = gpz[i] = 0ull;
                }
                cn = 0.0;
                pieceSteps = 0;
            }
            pieceSteps++;
            float cnc = 0.0f;
            const bool full = nAv == TA && nBv == CH;
            float* gw = sm.g[b][ty];
            bool packed = false;
            if constexpr (NH > 0 && BOX != 2) {
                if (full) {
                    pairsPacked<RA, RB, BOX, NH, HI>(apx, apy, apz, gpx, gpy, gpz, sm.pos[b], K, gw, cnc);
                    packed = true;
                }
            }
            if (!packed) {
                // Scalar pairs (ragged steps, triclinic boxes, other switch
                // kinds). B is scaled exactly as A, so that an atom present in
                // both groups gives a difference of exactly zero (excluded by the
                // lower bound); the products are rounded, never contracted.
                // B atoms in blocks of (at most) 4 per lane
                constexpr int QB = RB < 4 ? RB : 4;
#pragma unroll
                for (int jb = 0; jb < RB; jb += QB) {
                    float bx[QB], by[QB], bz[QB], gbx[QB], gby[QB], gbz[QB];
#pragma unroll
                    for (int j = 0; j < QB; j++) {
                        const float4 p = sm.pos[b][lane + 32 * (jb + j)];
                        bx[j] = __fmul_rn(p.x, K.ir0); by[j] = __fmul_rn(p.y, K.ir0); bz[j] = __fmul_rn(p.z, K.ir0);
                        gbx[j] = gby[j] = gbz[j] = 0.0f;
                    }
#pragma unroll
                    for (int i = 0; i < RH; i++) {
                        float ax[2], ay[2], az[2], gx[2], gy[2], gz[2];
                        f2::upk(apx[i], ax[0], ax[1]); f2::upk(apy[i], ay[0], ay[1]); f2::upk(apz[i], az[0], az[1]);
                        f2::upk(gpx[i], gx[0], gx[1]); f2::upk(gpy[i], gy[0], gy[1]); f2::upk(gpz[i], gz[0], gz[1]);
#pragma unroll
                        for (int e = 0; e < 2; e++) {
                            const bool av = (ty + NW * (2 * i + e)) < nAv;
#pragma unroll
                            for (int j = 0; j < QB; j++) {
                                const bool bv = (lane + 32 * (jb + j)) < nBv;
                                float dx = ax[e] - bx[j], dy = ay[e] - by[j], dz = az[e] - bz[j];
                                imageS<BOX>(dx, dy, dz, K.box);
                                const float x2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
                                float f, h;
                                switchX2<NH>(x2, av && bv && x2 >= K.lo && x2 < K.hi, K, f, h);
                                cnc += f;
                                gx[e] = fmaf(h, dx, gx[e]); gy[e] = fmaf(h, dy, gy[e]); gz[e] = fmaf(h, dz, gz[e]);
                                gbx[j] = fmaf(-h, dx, gbx[j]); gby[j] = fmaf(-h, dy, gby[j]);
                                gbz[j] = fmaf(-h, dz, gbz[j]);
                            }
                        }
                        gpx[i] = f2::pk(gx[0], gx[1]); gpy[i] = f2::pk(gy[0], gy[1]); gpz[i] = f2::pk(gz[0], gz[1]);
                    }
#pragma unroll
                    for (int j = 0; j < QB; j++) {
                        const int o = (lane + 32 * (jb + j)) * 3;
                        gw[o] = gbx[j]; gw[o + 1] = gby[j]; gw[o + 2] = gbz[j];
                    }
                }
            }
            cn += (double)cnc;
            if (last || (BLK && pieceSteps % BLK_STEPS == 0)) {
                // A sums over lanes: slot 3k + c = component c of A atom k, one
                // butterfly for all slots; lane 3k + c adds its slot
                float v[32];
#pragma unroll
                for (int i = 0; i < RH; i++) {
                    f2::upk(gpx[i], v[6 * i], v[6 * i + 3]);
                    f2::upk(gpy[i], v[6 * i + 1], v[6 * i + 4]);
                    f2::upk(gpz[i], v[6 * i + 2], v[6 * i + 5]);
                }
#pragma unroll
                for (int k = 3 * RA; k < 32; k++) v[k] = 0.0f;
                const float t = warpTransposeSum32(v);
                const int k = lane / 3, c = lane - 3 * k;
                const int i = ty + NW * k;
                if (lane < 3 * RA && i < nAv) redAddI64(R.acc + 3 * (size_t)(d.rowA + i) + c, __float2ll_rn(t * FX));
                if (BLK && !last) {
#pragma unroll
                    for (int q = 0; q < RH; q++) gpx[q] = gpy[q] = gpz[q] = 0ull;
                }
            }
            if (last) {
                const double cs = warpSum(cn);
                if (lane == 0) sm.red[b][ty] = cs;
            }
            cpAsyncWaitAll();
            __syncthreads();
            if (s == s0) afterFirst();
            if (ls + 2 < nw) issue(ls + 2, ib2, ia2, pq2);
            // B sums over warps in fixed order
            for (int v = tid; v < CH * 3; v += blockDim.x) {
                if (v / 3 < nBv) {
                    float t = 0.0f;
#pragma unroll
                    for (int y = 0; y < NW; y++) t += sm.g[b][y][v];
                    redAddI64(R.acc + 3 * (size_t)d.rowB + v, __float2ll_rn(t * FX));
                }
            }
            if (last) {
                if (tid == 0) {
                    double t = 0.0;
#pragma unroll
                    for (int y = 0; y < NW; y++) t += sm.red[b][y];
                    R.cnPiece[d.pieceSlot] = t;
                }
                hook(d.item, pieceSteps);
            }
        }
    }
}

}  // namespace glued
