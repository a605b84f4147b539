// OPES deposit (CommonGluedKernels.cpp:2752-3003), compiled with -fmad=false.
//
// The merge decision is an integer outcome of FP64 arithmetic. This translation
// unit contracts no multiply-add and takes exp/log/pow from glued_dmath.h, so
// every value the decision depends on (Silverman bandwidth, heights, merged
// centres/sigmas/log-weights) has the same bits as the CPU oracle's.
//
// k_opes_deposit (one warp):
//   - neff, Silverman sigma, height correction (lane 0),
//   - nearest kernel by Mahalanobis distance with that kernel's sigma: each lane
//     scans a strided subset with the reference's early exit, then a warp
//     arg-min with ties to the lowest index reproduces the sequential scan
//     (strict '<', first minimum wins, :2868-2882),
//   - merge (GMM moments) or append into slot numAllocated (:2885-2933),
//   - for an append, the O(N) sum_uprob increment (:2955-2981).
// After a merge the reference recomputes sum_uprob over all N^2 kernel pairs
// (:2982-3002); k_opes_uprob_pairs spreads that over the GPU and
// k_opes_uprob_finish adds the per-CTA partials in a fixed order.
#include "dev.hpp"
#include "glued_dmath.h"
#include "kernels.hpp"

namespace glued {

using namespace glued_dmath;

__device__ __forceinline__ double wsum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__global__ void k_opes_deposit(const BiasDev* __restrict__ bp, const double* __restrict__ cvv,
                               const double* __restrict__ energies, int* __restrict__ mergeFlag) {
    const BiasDev& b = *bp;
    const int lane = threadIdx.x;
    const int D = b.D;
    __shared__ double sc[16], ssg[16], sh[4];
    __shared__ int sflag[4];
    if (lane == 0) {
        sflag[0] = 0;
        if (b.adaptiveStride > 0 && b.nSamples[0] < b.adaptiveStride) {
            sflag[0] = 1;
            *b.lastDecision = -2;
        } else {
            if (b.variant != 1 && b.adaptiveStride == 0) b.nSamples[0]++;
            int n = b.nSamples[0];
            for (int d = 0; d < D; d++) sc[d] = cvv[b.cvIdx[d]];
            double VkT = energies[b.slot] * (1.0 / b.kT);
            double lwRaw, hRaw;
            if (b.variant == 2) { lwRaw = 0.0; hRaw = 1.0; } else { lwRaw = VkT; hRaw = gd_exp(VkT); }
            b.sumW[0] += hRaw;
            b.sumW[1] += hRaw * hRaw;
            b.stepCount[0]++;
            double sw = b.sumW[0], sw2 = b.sumW[1];
            double neff = (1.0 + sw) * (1.0 + sw) / (1.0 + sw2);
            double size = b.variant == 2 ? (double)b.stepCount[0] : neff;
            for (int d = 0; d < D; d++) {
                double s;
                if (b.variant == 1) s = b.sigma0[d];
                else if (b.adaptiveStride > 0) {
                    double factor = b.variant == 2 ? 1.0 : b.gamma;
                    double var = n > 1 ? b.runM2[d] / factor / (double)(n - 1) : 0.0;
                    s = var > 0.0 ? sqrt(var) : 1.0;
                    if (s < b.sigmaMin) s = b.sigmaMin;
                } else {
                    double resc = gd_pow(size * (D + 2) / 4.0, -1.0 / (D + 4.0));
                    s = b.sigma0[d] * resc;
                    if (s < b.sigmaMin) s = b.sigmaMin;
                }
                ssg[d] = s;
            }
            double lwNew = lwRaw;
            if (b.variant != 1 && b.adaptiveStride == 0)
                for (int d = 0; d < D; d++) lwNew += gd_log(b.sigma0[d] / ssg[d]);
            sh[0] = lwNew;
            sh[1] = gd_exp(lwNew);
            sh[2] = hRaw;
            *b.sumWeights += hRaw;  // KDNorm (:2945)
        }
    }
    __syncwarp();
    if (sflag[0]) return;
    const int nB = *b.numKernels;
    // nearest kernel, strided scan + warp arg-min
    double best = 1.0;
    int bestK = -1;
    for (int kp = lane; kp < nB; kp += 32) {
        double n2 = 0;
        bool over = false;
        for (int d = 0; d < D; d++) {
            double x = (sc[d] - b.centers[kp * D + d]) / b.sigmas[kp * D + d];
            n2 += x * x;
            if (n2 >= best) { over = true; break; }
        }
        if (!over) { best = n2; bestK = kp; }
    }
    for (int o = 16; o > 0; o >>= 1) {
        double ob = __shfl_xor_sync(0xffffffffu, best, o);
        int ok = __shfl_xor_sync(0xffffffffu, bestK, o);
        if (ok >= 0 && (bestK < 0 || ob < best || (ob == best && ok < bestK))) { best = ob; bestK = ok; }
    }
    const double lwNew = sh[0], hNew = sh[1];
    const double eps = gd_exp(-0.5 * b.cutoff2);
    if (bestK >= 0) {
        if (lane == 0) {
            int mk = bestK;
            double lwo = b.logW[mk], ho = gd_exp(lwo), ht = ho + hNew;
            double lmax = lwo > lwNew ? lwo : lwNew, lmin = lwo < lwNew ? lwo : lwNew;
            double lwm = lmax + gd_log1p(gd_exp(lmin - lmax));
            double f1 = ho / ht, f2 = hNew / ht;
            for (int d = 0; d < D; d++) {
                double c1 = b.centers[mk * D + d], s1 = b.sigmas[mk * D + d], c2 = sc[d], s2 = ssg[d];
                double cm = f1 * c1 + f2 * c2;
                double ss = f1 * (s1 * s1 + c1 * c1) + f2 * (s2 * s2 + c2 * c2) - cm * cm;
                if (ss < 0.0) ss = 0.0;
                double sm = sqrt(ss);
                if (sm < b.sigmaMin) sm = b.sigmaMin;
                b.centers[mk * D + d] = cm;
                b.sigmas[mk * D + d] = sm;
            }
            b.logW[mk] = lwm;
            *b.lastDecision = mk;
            *mergeFlag = 1;
        }
        return;
    }
    int k = 0;
    if (lane == 0) k = atomicAdd(b.numAllocated, 1);
    k = __shfl_sync(0xffffffffu, k, 0);
    if (k >= b.maxKernels) {
        // table full: roll back the claim; the reference then recomputes
        // sum_uprob over the unchanged table (:2982-3002)
        if (lane == 0) { atomicAdd(b.numAllocated, -1); *b.lastDecision = -3; *mergeFlag = 1; }
        return;
    }
    // O(N) increment of sum_uprob before the new row becomes visible
    double delta = 0.0;
    for (int j = lane; j < nB; j += 32) {
        double n2 = 0;
        bool skip = false;
        for (int d = 0; d < D; d++) {
            double dc = b.centers[j * D + d] - sc[d];
            n2 += dc * dc / (ssg[d] * ssg[d]);
            if (n2 >= b.cutoff2) { skip = true; break; }
        }
        if (!skip) delta += hNew * (gd_exp(-0.5 * n2) - eps);
    }
    for (int kp = lane; kp < nB; kp += 32) {
        double n2 = 0;
        bool skip = false;
        for (int d = 0; d < D; d++) {
            double dc = sc[d] - b.centers[kp * D + d], s = b.sigmas[kp * D + d];
            n2 += dc * dc / (s * s);
            if (n2 >= b.cutoff2) { skip = true; break; }
        }
        if (!skip) delta += gd_exp(b.logW[kp]) * (gd_exp(-0.5 * n2) - eps);
    }
    delta = wsum(delta);
    if (lane == 0) {
        for (int d = 0; d < D; d++) { b.centers[k * D + d] = sc[d]; b.sigmas[k * D + d] = ssg[d]; }
        b.logW[k] = lwNew;
        __threadfence();
        atomicAdd(b.numKernels, 1);
        *b.sumUprob += hNew * (1.0 - eps) + delta;
        *b.lastDecision = -1;
    }
}

// Full sum_uprob after a merge: sum over j, kp of h_kp (G(c_j; c_kp, s_kp) - eps).
__global__ void __launch_bounds__(256) k_opes_uprob_pairs(const BiasDev* __restrict__ bp,
                                                          const int* __restrict__ mergeFlag,
                                                          double* __restrict__ partial) {
    if (*mergeFlag == 0) return;
    const BiasDev& b = *bp;
    const int D = b.D, N = *b.numKernels;
    const double eps = gd_exp(-0.5 * b.cutoff2);
    double acc = 0.0;
    long long total = (long long)N * N;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        int j = (int)(t / N), kp = (int)(t % N);
        double n2 = 0;
        bool skip = false;
        for (int d = 0; d < D; d++) {
            double dc = b.centers[j * D + d] - b.centers[kp * D + d], s = b.sigmas[kp * D + d];
            n2 += dc * dc / (s * s);
            if (n2 >= b.cutoff2) { skip = true; break; }
        }
        if (!skip) acc += gd_exp(b.logW[kp]) * (gd_exp(-0.5 * n2) - eps);
    }
    __shared__ double red[8];
    acc = wsum(acc);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += red[w];
        partial[blockIdx.x] = s;
    }
}

__global__ void k_opes_uprob_finish(const BiasDev* __restrict__ bp, int* __restrict__ mergeFlag,
                                    const double* __restrict__ partial, int nPartial) {
    if (*mergeFlag == 0) return;
    double s = 0;
    for (int i = threadIdx.x; i < nPartial; i += 32) s += partial[i];
    s = wsum(s);
    if (threadIdx.x == 0) {
        *bp->sumUprob = s;
        *mergeFlag = 0;
    }
}

void launchOpesDeposit(cudaStream_t s, const BiasDev* b, const double* cvv, const double* energies,
                       int* mergeFlag, double* partial, int nPartial) {
    k_opes_deposit<<<1, 32, 0, s>>>(b, cvv, energies, mergeFlag);
    k_opes_uprob_pairs<<<nPartial, 256, 0, s>>>(b, mergeFlag, partial);
    k_opes_uprob_finish<<<1, 32, 0, s>>>(b, mergeFlag, partial, nPartial);
}

}  // namespace glued
