// Differentiable bias: contact map + path CV + hill bias on (CMAP, s), with a
// hand-written backward that gives dE/d(positions), dE/d(r0), dE/d(frames) and
// dE/d(heights). No reference counterpart as a whole (GLUED has no autograd);
// the CV definitions are the reference's contact map (CommonGluedKernels.cpp:
// 1236-1323) and path CV (:641-794).
//
//   CMAP = sum_p w_p s_p,  s_p = (1 - x^n)/(1 - x^m), x = d_p / r0_p
//          (integer n, m: evaluated as S_n(x)/S_m(x), the cancellation-free form)
//   w_f  = exp(-lambda MSD_f), MSD_f = sum_j |x_j - ref_fj|^2 / M
//   s    = sum_f (f+1) w_f / S, z = -ln(S)/lambda, S = sum_f w_f
//   E    = sum_k h_k exp(-(CMAP - c_k0)^2/(2 sig0^2) - (s - c_k1)^2/(2 sig1^2))
//
// The backward recomputes every per-pair switching value instead of storing it.
// Position gradients are summed as 2^40 fixed point with 64-bit integer atomics
// (order independent, so bitwise repeatable) and converted once.
#include <cuda_runtime.h>

#include <algorithm>

#include "pdl.cuh"
#include "../../include/glued_b200.h"
#include "context.hpp"
#include "devfn.cuh"
#include "kernels.hpp"

namespace glued {

// The spec crosses the C ABI as glued_ad_spec (include/glued_b200.h).
typedef glued_ad_spec AdSpec;

namespace {
constexpr double kFix = 1099511627776.0;  // 2^40

template <class R>
__device__ __forceinline__ void ratioSwitchT(R x, int n, int m, R& f, R& dfdx) {
    R sn = 0, dsn = 0, sm = 0, dsm = 0;
    for (int j = n - 1; j >= 0; j--) { dsn = dsn * x + sn; sn = sn * x + (R)1; }
    for (int j = m - 1; j >= 0; j--) { dsm = dsm * x + sm; sm = sm * x + (R)1; }
    R ism = (R)1 / sm;
    f = sn * ism;
    dfdx = (dsn * sm - sn * dsm) * ism * ism;
}

template <class R>
__device__ __forceinline__ void pairGeom(const AdSpec& S, int p, R& d, R dr[3]) {
    const R* pos = static_cast<const R*>(S.pos);
    int a = S.pairs[2 * p], b = S.pairs[2 * p + 1];
    for (int c = 0; c < 3; c++) {
        R x = pos[3 * b + c] - pos[3 * a + c];
        if (S.periodic) x -= (R)S.box[c] * floor(x / (R)S.box[c] + (R)0.5);
        dr[c] = x;
    }
    d = sqrt(dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2]);
}
}  // namespace

// out: [0] E, [1] CMAP, [2] s, [3] z, [4] S, [5..5+F) w_f; part: per-CTA CMAP partials
template <class R>
// CTAs [0, nPart): contact-map partial sums over the pairs; CTAs nPart + f: the
// mean-square deviation sum of path frame f (path atoms gathered, frame
// coordinates streamed coalesced), written to out[5 + f], where
// k_ad_path_hills turns it into the frame weight. Spreading the frames over
// CTAs keeps enough loads in flight to stream the frames from DRAM.
__global__ void k_ad_cmap(AdSpec S, double* part, int nPart, double* out) {
    pdlEnter();
    __shared__ double red[32];
    double acc = 0.0;
    if (blockIdx.x < nPart) {
        const R* r0 = static_cast<const R*>(S.r0);
        for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < S.nPairs; p += nPart * blockDim.x) {
            R d, dr[3];
            pairGeom<R>(S, p, d, dr);
            R x = d / r0[p], f, dfdx;
            ratioSwitchT<R>(x, (int)S.nmw[3 * p], (int)S.nmw[3 * p + 1], f, dfdx);
            acc += (double)((R)S.nmw[3 * p + 2] * f);
        }
        double v[1] = {acc};
        blockSum<1>(v, red);
        if (threadIdx.x == 0) part[blockIdx.x] = v[0];
    } else {
        const int f = blockIdx.x - nPart;
        const R* pos = static_cast<const R*>(S.pos);
        const R* fr = static_cast<const R*>(S.frames) + (size_t)f * S.M * 3;
#pragma unroll 4
        for (int i = threadIdx.x; i < 3 * S.M; i += blockDim.x) {
            const int a = S.pathAtoms[i / 3];
            const R dx = pos[3 * a + i % 3] - fr[i];
            acc += (double)(dx * dx);
        }
        double v[1] = {acc};
        blockSum<1>(v, red);
        if (threadIdx.x == 0) out[5 + f] = v[0];
    }
}

// Positions, frames and the hill table are the caller's inputs, complete before
// the first kernel of the step passed its wait; the kernels after it load their
// share of them before their own wait and read only the previous kernel's
// output after it.
constexpr int AD_HP = 4;   // hills per thread loaded before the wait

template <class R>
__global__ void __launch_bounds__(512) k_ad_path_hills(AdSpec S, const double* part, int nPart, double* out) {
    const R* h = static_cast<const R*>(S.heights);
    double pc0[AD_HP], pc1[AD_HP], ph[AD_HP];
#pragma unroll
    for (int u = 0; u < AD_HP; u++) {
        const int k = threadIdx.x + u * blockDim.x;
        pc0[u] = k < S.K ? S.hillC[2 * k] : 0.0;
        pc1[u] = k < S.K ? S.hillC[2 * k + 1] : 0.0;
        ph[u] = k < S.K ? (double)h[k] : 0.0;
    }
    pdlEnter();
    __shared__ double red[32 * 3];
    __shared__ double sw[128];
    __shared__ double bc[4];
    const int tid = threadIdx.x;
    // frame weights from the frame MSD sums of k_ad_cmap
    for (int f = tid; f < S.F; f += blockDim.x) sw[f] = exp(-S.lambda * out[5 + f] / S.M);
    __syncthreads();
    if (tid == 0) {
        double cm = 0;
        for (int k = 0; k < nPart; k++) cm += part[k];
        double Ssum = 0, sn = 0;
        for (int f = 0; f < S.F; f++) { Ssum += sw[f]; sn += (f + 1) * sw[f]; }
        bc[0] = cm;
        bc[1] = sn / Ssum;
        bc[2] = -log(Ssum) / S.lambda;
        bc[3] = Ssum;
    }
    __syncthreads();
    const double cm = bc[0], s = bc[1];
    double v[3] = {0, 0, 0};
    auto hill = [&](double c0, double c1, double hk) {
        double d0 = cm - c0, d1 = s - c1;
        double g = hk * exp(-d0 * d0 / (2 * S.sig[0] * S.sig[0]) - d1 * d1 / (2 * S.sig[1] * S.sig[1]));
        v[0] += g;
        v[1] += -g * d0 / (S.sig[0] * S.sig[0]);
        v[2] += -g * d1 / (S.sig[1] * S.sig[1]);
    };
#pragma unroll
    for (int u = 0; u < AD_HP; u++)
        if (tid + u * (int)blockDim.x < S.K) hill(pc0[u], pc1[u], ph[u]);
    for (int k = tid + AD_HP * blockDim.x; k < S.K; k += blockDim.x)
        hill(S.hillC[2 * k], S.hillC[2 * k + 1], (double)h[k]);
    blockSum<3>(v, red);
    if (tid == 0) {
        out[0] = v[0]; out[1] = cm; out[2] = s; out[3] = bc[2]; out[4] = bc[3];
        out[5 + S.F] = v[1];      // dE/dCMAP
        out[6 + S.F] = v[2];      // dE/ds
    }
    for (int f = tid; f < S.F; f += blockDim.x) out[5 + f] = sw[f];
}

// gE: device scalar dL/dE. Position gradient accumulates into fixed-point acc.
template <class R>
__global__ void k_ad_back_pairs(AdSpec S, const double* out, const double* gE, long long* acc, R* gR0) {
    pdlEnter();
    const R* r0 = static_cast<const R*>(S.r0);
    const double gC = gE[0] * out[5 + S.F];
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < S.nPairs; p += gridDim.x * blockDim.x) {
        R d, dr[3];
        pairGeom<R>(S, p, d, dr);
        R x = d / r0[p], f, dfdx;
        ratioSwitchT<R>(x, (int)S.nmw[3 * p], (int)S.nmw[3 * p + 1], f, dfdx);
        const double w = S.nmw[3 * p + 2];
        // dCMAP/dd = w dfdx / r0; dd/dr_b = dr/d
        const double coef = gC * w * (double)dfdx / (double)r0[p] / (double)d;
        int a = S.pairs[2 * p], b = S.pairs[2 * p + 1];
        for (int c = 0; c < 3; c++) {
            long long q = __double2ll_rn(coef * (double)dr[c] * kFix);
            atomicAdd(reinterpret_cast<unsigned long long*>(acc + 3 * b + c), (unsigned long long)q);
            atomicAdd(reinterpret_cast<unsigned long long*>(acc + 3 * a + c), (unsigned long long)(-q));
        }
        // dCMAP/dr0 = w dfdx * (-x / r0)
        gR0[p] = (R)(gC * w * (double)dfdx * (-(double)x / (double)r0[p]));
    }
}

template <class R>
__global__ void k_ad_back_path(AdSpec S, const double* out, const double* gE, long long* acc, R* gFrames) {
    const R* pos = static_cast<const R*>(S.pos);
    const R* fr = static_cast<const R*>(S.frames);
    const int t0 = blockIdx.x * blockDim.x + threadIdx.x;
    double dx0[3] = {0, 0, 0};
    int a0 = 0;
    if (t0 < S.M * S.F) {
        const int f = t0 / S.M, j = t0 % S.M;
        a0 = S.pathAtoms[j];
        for (int c = 0; c < 3; c++)
            dx0[c] = (double)pos[3 * a0 + c] - (double)fr[((size_t)f * S.M + j) * 3 + c];
    }
    pdlEnter();
    const double gS = gE[0] * out[6 + S.F];
    const double s = out[2], Ssum = out[4];
    const double* w = out + 5;
    const double sc = 2.0 * S.lambda / (S.M * Ssum);
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < S.M * S.F; t += gridDim.x * blockDim.x) {
        // thread per (frame, atom): d s / d ref_fj = sc (f+1-s) w_f (x_j - ref_fj)
        int f = t / S.M, j = t % S.M;
        const bool first = t == t0;
        int a = first ? a0 : S.pathAtoms[j];
        double k = gS * sc * ((f + 1) - s) * w[f];
        for (int c = 0; c < 3; c++) {
            double dx = first ? dx0[c] : (double)pos[3 * a + c] - (double)fr[((size_t)f * S.M + j) * 3 + c];
            gFrames[((size_t)f * S.M + j) * 3 + c] = (R)(k * dx);
            // d s / d x_j = -(that), summed over frames into the atom's gradient
            long long q = __double2ll_rn(-k * dx * kFix);
            atomicAdd(reinterpret_cast<unsigned long long*>(acc + 3 * a + c), (unsigned long long)q);
        }
    }
}

template <class R>
__global__ void k_ad_back_hills_and_convert(AdSpec S, const double* out, const double* gE, const long long* acc,
                                            R* gPos, R* gH) {
    const int k0 = blockIdx.x * blockDim.x + threadIdx.x;
    const double c00 = k0 < S.K ? S.hillC[2 * k0] : 0.0, c01 = k0 < S.K ? S.hillC[2 * k0 + 1] : 0.0;
    pdlEnter();
    const double cm = out[1], s = out[2];
    for (int k = k0; k < S.K; k += gridDim.x * blockDim.x) {
        const bool first = k == k0;
        double d0 = cm - (first ? c00 : S.hillC[2 * k]), d1 = s - (first ? c01 : S.hillC[2 * k + 1]);
        gH[k] = (R)(gE[0] * exp(-d0 * d0 / (2 * S.sig[0] * S.sig[0]) - d1 * d1 / (2 * S.sig[1] * S.sig[1])));
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 3 * S.nAtoms; i += gridDim.x * blockDim.x)
        gPos[i] = (R)((double)acc[i] / kFix);
}

template <class R>
void adForwardT(cudaStream_t st, const AdSpec& S, double* out, double* part, int nPart) {
    launchPdl(k_ad_cmap<R>, dim3(nPart + S.F), dim3(256), 0, st, S, part, nPart, out);
    launchPdl(k_ad_path_hills<R>, dim3(1), dim3(512), 0, st, S, static_cast<const double*>(part), nPart, out);
}

template <class R>
void adBackwardT(cudaStream_t st, const AdSpec& S, const double* out, const double* gE, long long* acc, void* gPos,
                 void* gR0, void* gFrames, void* gH) {
    cudaCheck(cudaMemsetAsync(acc, 0, sizeof(long long) * 3 * (size_t)S.nAtoms, st), "memset");
    int bp = (S.nPairs + 255) / 256;
    if (bp > 0) launchPdl(k_ad_back_pairs<R>, dim3(bp), dim3(256), 0, st, S, out, gE, acc, static_cast<R*>(gR0));
    int bf = (S.M * S.F + 255) / 256;
    if (bf > 0) launchPdl(k_ad_back_path<R>, dim3(bf), dim3(256), 0, st, S, out, gE, acc, static_cast<R*>(gFrames));
    int bc = (std::max(S.K, 3 * S.nAtoms) + 255) / 256;
    launchPdl(k_ad_back_hills_and_convert<R>, dim3(bc), dim3(256), 0, st, S, out, gE, static_cast<const long long*>(acc),
              static_cast<R*>(gPos), static_cast<R*>(gH));
}

void adForward(int dtype, cudaStream_t st, const AdSpec& S, double* out, double* part, int nPart) {
    if (S.F > 128) throw Error(GLUED_E_INVALID, "path frame count exceeds 128");
    if (dtype == 1) adForwardT<double>(st, S, out, part, nPart);
    else adForwardT<float>(st, S, out, part, nPart);
    cudaCheck(cudaGetLastError(), "autograd forward");
}

void adBackward(int dtype, cudaStream_t st, const AdSpec& S, const double* out, const double* gE, long long* acc,
                void* gPos, void* gR0, void* gFrames, void* gH) {
    if (dtype == 1) adBackwardT<double>(st, S, out, gE, acc, gPos, gR0, gFrames, gH);
    else adBackwardT<float>(st, S, out, gE, acc, gPos, gR0, gFrames, gH);
    cudaCheck(cudaGetLastError(), "autograd backward");
}

}  // namespace glued
