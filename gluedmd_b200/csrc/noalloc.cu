// Coordination number of one CV without any device allocation by the call.
//
// Who needs this: callers that cannot call cudaMalloc while they evaluate
// forces — an MD engine that reserves all device memory at start-up and forbids
// allocation inside its step loop, code that owns the device heap through its
// own allocator, or a host loop that must not take the allocator's locks. The
// regular path (glued_context_*) allocates its tile partials when the context
// is created; this entry point instead keeps them in a fixed array that is part
// of this library's device image. The array is created when the library's
// device code is loaded on a GPU and stays resident on every GPU that loads it
// until the process exits. The caller passes only inputs and outputs.
//
// The kernels are the partial-sum coordination tile (coord_tile.cuh: one CTA
// per 64-atom A tile and B split, float partials) and a fixed-order reduction of
// its partials. They are not the context path's kernels (fixed-point step runs,
// coord_run.cuh), but they evaluate the same switch in the same precision per
// kind (S_n/S_m for integer exponents in FP32, the reference formula in FP64
// for non-integer ones), so the two agree to the rounding of FP32 partial sums.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <string>

#include "../../include/glued_b200.h"
#include "context.hpp"
#include "coord_tile.cuh"

namespace glued {

namespace {
constexpr size_t kScratchBytes = (size_t)GLUED_NOALLOC_SCRATCH_BYTES;
constexpr int kRA = 8;  // A atoms per thread, TA = 64
constexpr int kTA = 8 * kRA;

// File-scope scratch for tile partials. In host code this name is only a
// handle for cudaGetSymbolAddress; kernels receive the device address.
static __device__ __align__(256) unsigned char g_noallocScratch[kScratchBytes];

// Device address of the scratch array in the current device's context, looked
// up on every call: the lookup allocates nothing and costs little once the
// module is loaded (the first call on a device may load it), and a cached
// address would go stale when the context is torn down and recreated
// (cudaDeviceReset) between calls.
void* scratchOnCurrentDevice() {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noallocScratch);
    if (e != cudaSuccess || p == nullptr)
        throw Error(GLUED_E_CUDA, std::string("cudaGetSymbolAddress of the scratch array failed: ") +
                                      cudaGetErrorString(e));
    return p;
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }
}  // namespace

template <int BOX, int NH>
__global__ void __launch_bounds__(256, 2) k_noalloc_pairs(const float4* __restrict__ posq, CoordDev C, CoordItem it,
                                                         BoxDev box) {
    __shared__ float sB[NY][TB * 3];
    __shared__ double red[32];
    const int ta = blockIdx.x / it.splitsB, sb = blockIdx.x % it.splitsB;
    coordTile<kRA, BOX, NH>(posq, nullptr, C, it, ta, sb, box, sB, red);
}

// Rows A then B; one thread per (row, component); partials summed in fixed order.
__global__ void k_noalloc_finalize(CoordDev C, CoordItem it, double* __restrict__ cnOut, float* __restrict__ gradOut) {
    const int R = it.nA + it.nB;
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid < 3 * R) {
        const int comp = gid % 3, row = gid / 3;
        const float* p;
        int n;
        size_t stride;
        if (row < it.nA) {
            p = C.partA + 3 * (size_t)row + comp;
            n = it.splitsB;
            stride = 3 * (size_t)it.nA;
        } else {
            p = C.partB + 3 * (size_t)(row - it.nA) + comp;
            n = it.tilesA;
            stride = 3 * (size_t)it.nB;
        }
        double acc = 0.0;
        for (int k = 0; k < n; k++) acc += __ldg(p + (size_t)k * stride);
        gradOut[(size_t)comp * R + row] = (float)acc;
    }
    if (blockIdx.x == 0 && threadIdx.x < 32) {
        const int nb = it.tilesA * it.splitsB;
        double s = 0;
        for (int k = threadIdx.x; k < nb; k += 32) s += C.cnPart[k];
        s = warpSum(s);
        if (threadIdx.x == 0) *cnOut = s;
    }
}

template <int BOX>
void launchPairs(cudaStream_t s, int blocks, int kind, const float4* posq, const CoordDev& C, const CoordItem& it,
                 const BoxDev& box) {
    if (kind == 3) k_noalloc_pairs<BOX, 3><<<blocks, 256, 0, s>>>(posq, C, it, box);
    else if (kind == -1) k_noalloc_pairs<BOX, -1><<<blocks, 256, 0, s>>>(posq, C, it, box);
    else k_noalloc_pairs<BOX, 0><<<blocks, 256, 0, s>>>(posq, C, it, box);
}

void coordinationNoAlloc(cudaStream_t stream, const void* posq, const int* groupA, int nA, const int* groupB, int nB,
                         double r0, double n, double m, int periodic, const double* box9, double* cnOut,
                         float* gradOut) {
    if (!posq || !groupA || !groupB || !cnOut || !gradOut)
        throw Error(GLUED_E_INVALID, "coordination (no-alloc): null argument");
    if (nA < 1 || nB < 1) throw Error(GLUED_E_INVALID, "coordination (no-alloc): both groups need at least one atom");
    if (!(std::isfinite(r0) && r0 > 0.0)) throw Error(GLUED_E_INVALID, "coordination (no-alloc): r0 must be finite and > 0");
    // n == m is allowed: the switch is then 1 for every pair (the reference
    // formula's quotient and its Taylor branch at x = 1 both give n/m = 1)
    if (!(std::isfinite(n) && std::isfinite(m) && n > 0.0 && m > 0.0))
        throw Error(GLUED_E_INVALID, "coordination (no-alloc): n and m must be finite and > 0");
    if (periodic && !box9) throw Error(GLUED_E_INVALID, "coordination (no-alloc): periodic needs box vectors");
    // Same tiling rule as the context path (Context::buildPlan).
    const long long pairs = (long long)nA * nB;
    const long long perCta = std::max<long long>(1, pairs / (148LL * 8));
    const int bSplit =
        (int)std::min<long long>(1 << 20, std::max<long long>(128, ((perCta / kTA + 127) / 128) * 128));
    CoordItem it{};
    it.cv = 0; it.jac0 = 0;
    it.nA = nA; it.nB = nB; it.a0 = 0; it.b0 = nA;
    it.r0 = (float)r0; it.n = (float)n; it.m = (float)m; it.rc2 = 0.0f;
    it.kind = coordKind(it.n, it.m);
    it.tilesA = (nA + kTA - 1) / kTA;
    it.splitsB = (nB + bSplit - 1) / bSplit;
    it.block0 = 0; it.partA = 0; it.partB = 0; it.cn0 = 0;
    // scratch layout: atoms | partials of A | partials of B | CN per CTA
    const size_t oAtoms = 0;
    const size_t oPartA = align256(oAtoms + sizeof(int) * ((size_t)nA + nB));
    const size_t oPartB = align256(oPartA + sizeof(float) * 3 * (size_t)it.splitsB * nA);
    const size_t oCn = align256(oPartB + sizeof(float) * 3 * (size_t)it.tilesA * nB);
    const size_t need = oCn + sizeof(double) * (size_t)it.tilesA * it.splitsB;
    if (need > kScratchBytes)
        throw Error(GLUED_E_INVALID, "coordination (no-alloc): groups of " + std::to_string(nA) + " x " +
                                         std::to_string(nB) + " atoms need " + std::to_string(need) +
                                         " bytes of scratch; the fixed array holds " + std::to_string(kScratchBytes) +
                                         " bytes (GLUED_NOALLOC_SCRATCH_BYTES)");
    unsigned char* base = static_cast<unsigned char*>(scratchOnCurrentDevice());
    int* atoms = reinterpret_cast<int*>(base + oAtoms);
    // Every partial slot is written by exactly one CTA before it is read, so the
    // contents left by an earlier call need no clearing.
    cudaCheck(cudaMemcpyAsync(atoms, groupA, sizeof(int) * nA, cudaMemcpyDeviceToDevice, stream), "copy group A");
    cudaCheck(cudaMemcpyAsync(atoms + nA, groupB, sizeof(int) * nB, cudaMemcpyDeviceToDevice, stream), "copy group B");
    CoordDev C{};
    C.items = nullptr; C.numItems = 1;
    C.atoms = atoms;
    C.blockItem = nullptr;
    C.partA = reinterpret_cast<float*>(base + oPartA);
    C.partB = reinterpret_cast<float*>(base + oPartB);
    C.cnPart = reinterpret_cast<double*>(base + oCn);
    C.bSplit = bSplit;
    BoxDev box{};
    box.kind = 0;
    if (periodic) {
        for (int i = 0; i < 3; i++) { box.a[i] = (float)box9[i]; box.b[i] = (float)box9[3 + i]; box.c[i] = (float)box9[6 + i]; }
        box.inv[0] = (float)(1.0 / box9[0]); box.inv[1] = (float)(1.0 / box9[4]); box.inv[2] = (float)(1.0 / box9[8]);
        bool rect = box9[1] == 0 && box9[2] == 0 && box9[3] == 0 && box9[5] == 0 && box9[6] == 0 && box9[7] == 0;
        box.kind = rect ? 1 : 2;
    }
    const int blocks = it.tilesA * it.splitsB;
    const float4* p = static_cast<const float4*>(posq);
    if (box.kind == 0) launchPairs<0>(stream, blocks, it.kind, p, C, it, box);
    else if (box.kind == 1) launchPairs<1>(stream, blocks, it.kind, p, C, it, box);
    else launchPairs<2>(stream, blocks, it.kind, p, C, it, box);
    cudaCheck(cudaGetLastError(), "coordination (no-alloc) pairs");
    const int rows3 = 3 * (nA + nB);
    k_noalloc_finalize<<<(rows3 + 255) / 256, 256, 0, stream>>>(C, it, cnOut, gradOut);
    cudaCheck(cudaGetLastError(), "coordination (no-alloc) finalize");
}

}  // namespace glued
