// Bias evaluation, chain-rule scatter and MetaD deposition.
//
// k_biases : every bias of the context inside one CTA, added into dU/dCV in
//            the reference's evaluation order (harmonic, OPES, MetaD grid,
//            PBMETAD, EXTERNAL, then this library's hill-sum MetaD;
//            CommonGluedKernels.cpp:4955-5026). The bias records are copied to
//            shared memory before the wait for the previous kernel (the host
//            writes them only between steps). The single-thread biases
//            (harmonic, MetaD, PBMETAD, EXTERNAL) are evaluated concurrently,
//            one warp each, into per-bias contributions that thread 0 then adds
//            in evaluation order, so dU/dCV is summed in the same order as a
//            sequential pass. dU/dCV is accumulated in shared memory and written
//            once, so no separate clearing pass is needed (the reference relies
//            on OpenMM's autoclear, :4244). Kernel/hill sums are split over all
//            threads and reduced by a fixed tree in FP64.
// k_scatter: F[atom] -= dU/dCV * dCV/dx as 2^32 fixed point with three 64-bit
//            integer atomics per Jacobian row (CommonGluedKernels.cpp:2430-2456);
//            integer addition keeps the result order-independent.
// k_metad_deposit: WT Gaussian added only inside the +-4 sigma window that can
//            pass the reference's exponent <= 8 test (CommonGluedKernels.cpp:
//            3645-3680 scans the whole grid); each grid point is written by one
//            thread, so the deposit is deterministic.
#include <algorithm>

#include "devfn.cuh"
#include "kernels.hpp"
#include "pdl.cuh"
#include "force.hpp"

namespace glued {

// MetaD / EXTERNAL grid (CommonGluedKernels.cpp:3574-3636), one thread, D <= 3
// (checked at setup): multilinear interpolation over the 2^D cell corners with
// periodic wrap or clamping. All corner values are loaded before the arithmetic.
// Writes the energy and dE/ds_d into out[d].
__device__ __noinline__ void evalMetadGrid(const BiasDev& b, const double* cvv, double* energies, double* out) {
    int lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    double al[3] = {0, 0, 0};
    const int D = b.D;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        if (d >= D) break;
        double fr = (cvv[b.cvIdx[d]] - b.origin[d]) * b.invSp[d];
        int N = b.npts[d];
        if (N <= 1) { lo[d] = hi[d] = 0; al[d] = 0; }
        else if (b.per[d]) {
            fr = fr - floor(fr / (double)N) * (double)N;
            if (fr < 0.0) fr += N;
            lo[d] = (int)fr;
            if (lo[d] >= N) lo[d] = N - 1;
            al[d] = fr - lo[d];
            hi[d] = (lo[d] + 1) % N;
        } else {
            if (fr < 0.0) fr = 0.0;
            if (fr > (double)(N - 1)) fr = (double)(N - 1);
            lo[d] = (int)fr;
            if (lo[d] >= N - 1) lo[d] = N - 2;
            al[d] = fr - lo[d];
            hi[d] = lo[d] + 1;
        }
    }
    const int nc = 1 << D;
    double val[8];
#pragma unroll
    for (int c = 0; c < 8; c++) {
        if (c < nc) {
            int flat = 0;
#pragma unroll
            for (int d = 0; d < 3; d++)
                if (d < D) flat += (((c >> d) & 1) ? hi[d] : lo[d]) * b.strides[d];
            val[c] = b.grid[flat];
        }
    }
    double V = 0, dV[3] = {0, 0, 0};
#pragma unroll
    for (int c = 0; c < 8; c++) {
        if (c >= nc) break;
        double w = 1;
#pragma unroll
        for (int d = 0; d < 3; d++)
            if (d < D) w *= ((c >> d) & 1) ? al[d] : (1.0 - al[d]);
        V += w * val[c];
#pragma unroll
        for (int d = 0; d < 3; d++) {
            if (d >= D) break;
            double sg = ((c >> d) & 1) ? 1.0 : -1.0, wo = 1;
#pragma unroll
            for (int e = 0; e < 3; e++)
                if (e < D && e != d) wo *= ((c >> e) & 1) ? al[e] : (1.0 - al[e]);
            dV[d] += sg * wo * val[c];
        }
    }
    energies[b.slot] = V;
#pragma unroll
    for (int d = 0; d < 3; d++)
        if (d < D) out[d] = dV[d] * b.invSp[d];
}

// PBMETAD (CommonGluedKernels.cpp:3694-3760), one thread: sub-grid d is a 1-D
// grid over CV cvIdx[d], linearly interpolated (periodic wrap or clamp, as the
// MetaD grid); the sub-grid energies V_d combine as
// E = -kT (ln sum_d exp((Vmin - V_d)/kT) - ln N) + Vmin, and dE/ds_d = w_d dV_d/ds_d
// with the softmax weights w_d = exp((Vmin - V_d)/kT) / sum, written to out[d].
// V_d and w_d are kept in pbState for the deposit.
__device__ __noinline__ void evalPbmetad(const BiasDev& b, const double* cvv, double* energies, double* out) {
    const int N = b.D;
    // vlo / vhi hold the cell values, then V_d / dV_d/ds_d
    double vlo[8], vhi[8], al[8];
    double* const V = vlo;
    double* const G = vhi;
    // all sub-grid cells first, so their loads are in flight together
#pragma unroll
    for (int d = 0; d < 8; d++) {
        if (d >= N) break;
        const double* g = b.grid + b.goff[d];
        const int n = b.npts[d];
        double fr = (cvv[b.cvIdx[d]] - b.origin[d]) * b.invSp[d];
        int lo, hi;
        if (b.per[d]) {
            fr = fr - floor(fr / (double)n) * (double)n;
            if (fr < 0.0) fr += n;
            lo = (int)fr;
            if (lo >= n) lo = n - 1;
            hi = (lo + 1) % n;
        } else {
            if (fr < 0.0) fr = 0.0;
            if (fr > (double)(n - 1)) fr = (double)(n - 1);
            lo = (int)fr;
            if (lo >= n - 1) lo = n - 2;
            hi = lo + 1;
        }
        al[d] = fr - lo;
        vlo[d] = g[lo];
        vhi[d] = g[hi];
    }
#pragma unroll
    for (int d = 0; d < 8; d++) {
        if (d >= N) break;
        const double v = vlo[d] * (1.0 - al[d]) + vhi[d] * al[d];
        G[d] = (vhi[d] - vlo[d]) * b.invSp[d];
        V[d] = v;
    }
    double vmin = V[0];
#pragma unroll
    for (int d = 1; d < 8; d++)
        if (d < N) vmin = V[d] < vmin ? V[d] : vmin;
    double ene = 0.0;
#pragma unroll 1
    for (int d = 0; d < N; d++) ene += exp((vmin - V[d]) / b.kT);
    energies[b.slot] = -b.kT * (log(ene) - log((double)N)) + vmin;
#pragma unroll 1
    for (int d = 0; d < N; d++) {
        const double w = exp((vmin - V[d]) / b.kT) / ene;
        b.pbState[d] = V[d];
        b.pbState[N + d] = w;
        out[d] = w * G[d];
    }
}

// Kernel sums of the OPES and hill-sum MetaD biases (CommonGluedKernels.cpp:2642-2700
// for OPES), spread over KSUM_CTAS CTAs per bias: each CTA sums a contiguous
// range of kernels into 9 FP64 partials {dV/ds_0..7 terms, value}; k_biases sums
// the partials in CTA order.
//
// MODE (the context's sum precision): SUM_FP64 evaluates and sums every kernel
// in FP64 (per thread, then a fixed block tree). SUM_FP32 / SUM_FP32C evaluate
// the Gaussians and accumulate in FP32, plain or with a two-sum compensation
// term per accumulator (also through the warp tree); the exponent that decides
// whether a hill counts (> 8 truncated, a jump of h e^-8) is still formed in
// FP64, so that decision is the FP64 path's. OPES heights exp(logW) are taken
// relative to the largest logW of the warp, M_w: FP32 holds exp(logW - M_w) <= 1,
// and the warp's sums are scaled by exp(M_w) in FP64 when they become partials
// (the log-sum-exp normalisation in FP64). Kernels whose FP64 height would not
// be finite (logW >= log 1e308) are skipped in every mode.
//
// The kernel tables (count, centres, sigmas, log-weights; hill centres and
// heights) are written only by the deposit kernels of updateState, which have
// completed before this launch can start (the kernel it depends on has passed
// its own wait, or is a plain launch); so the record, the count and each
// thread's first OPES kernel are loaded before the wait, and only the CV values
// of the kernel before are read after it.
__device__ __forceinline__ void twoSumAcc(float& s, float& c, float b) {
    const float t = __fadd_rn(s, b);
    const float bb = __fsub_rn(t, s);
    c = __fadd_rn(c, __fadd_rn(__fsub_rn(s, __fsub_rn(t, bb)), __fsub_rn(b, bb)));
    s = t;
}

template <int MODE>
__device__ __forceinline__ void accF(float& s, float& c, float b) {
    if (MODE == SUM_FP32C) twoSumAcc(s, c, b);
    else s = __fadd_rn(s, b);
}

template <int MODE>
__global__ void __launch_bounds__(256) k_kernel_sums(const BiasDev* __restrict__ biases,
                                                      const double* __restrict__ cvv, double* __restrict__ part) {
    __shared__ double red[32 * 9];
    const BiasDev& b = biases[blockIdx.y];
    const int type = b.type;
    if (type != BIAS_OPES && type != BIAS_METAD_HILLS) {
        pdlEnter();
        return;  // uniform over the CTA
    }
    const int tid = threadIdx.x, nt = blockDim.x;
    const int D = b.D;
    const int K = type == BIAS_OPES ? *b.numKernels : *b.hCount;
    const int k0 = (int)((long long)K * blockIdx.x / gridDim.x);
    const int k1 = (int)((long long)K * (blockIdx.x + 1) / gridDim.x);
    constexpr double LW_MAX = 709.1962086421661;   // log(1e308)
    double pc[8], ps[8], plw = 0.0;
    const int kf = k0 + tid;
    if (type == BIAS_OPES && kf < k1) {
        for (int d = 0; d < D; d++) { pc[d] = b.centers[kf * D + d]; ps[d] = b.sigmas[kf * D + d]; }
        plw = b.logW[kf];
    }
    pdlEnter();
    double s[8];
    for (int d = 0; d < D; d++) s[d] = cvv[b.cvIdx[d]];
    if constexpr (MODE == SUM_FP64) {
        double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        if (type == BIAS_OPES) {
            const double kfloor = exp(-0.5 * b.cutoff2);
            for (int k = kf; k < k1; k += nt) {
                const bool first = k == kf;
                double n2 = 0, dc[8], is2[8];
                for (int d = 0; d < D; d++) {
                    dc[d] = s[d] - (first ? pc[d] : b.centers[k * D + d]);
                    double sg = first ? ps[d] : b.sigmas[k * D + d];
                    is2[d] = 1.0 / (sg * sg);
                    n2 += dc[d] * dc[d] * is2[d];
                }
                if (!(n2 < b.cutoff2)) continue;
                double G = exp(-0.5 * n2), kern = G - kfloor;
                if (kern <= 0.0) continue;
                double h = exp(first ? plw : b.logW[k]);
                if (!(h > 0.0 && h < 1e308)) continue;
                acc[8] += h * kern;
                for (int d = 0; d < D; d++) acc[d] += h * G * (-dc[d] * is2[d]);
            }
        } else {
            // direct hill sum, exponent > 8 truncated like the grid deposit
            for (int k = k0 + tid; k < k1; k += nt) {
                double ex = 0, dc[8];
                for (int d = 0; d < D; d++) {
                    double x = s[d] - b.hCenters[k * D + d];
                    if (b.period[d] > 0) x -= round(x / b.period[d]) * b.period[d];
                    dc[d] = x;
                    ex += x * x / (2.0 * b.sigma[d] * b.sigma[d]);
                }
                if (ex > 8.0) continue;
                double g = b.hHeights[k] * exp(-ex);
                acc[8] += g;
                for (int d = 0; d < D; d++) acc[d] += -g * dc[d] / (b.sigma[d] * b.sigma[d]);
            }
        }
        blockSum<9>(acc, red);
        if (tid < 9) part[((size_t)blockIdx.y * gridDim.x + blockIdx.x) * 9 + tid] = acc[tid];
    } else {
        float acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, cmp[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        const int lane = tid & 31, warp = tid >> 5;
        double M = 0.0;   // OPES: the warp's largest logW (-inf: no kernel in the warp)
        if (type == BIAS_OPES) {
            double m = -INFINITY;
            for (int k = kf; k < k1; k += nt) {
                const double lw = k == kf ? plw : b.logW[k];
                if (lw < LW_MAX && lw > m) m = lw;
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
            M = m;
            const float kfloor = __expf(-0.5f * (float)b.cutoff2);
            const float cut2 = (float)b.cutoff2;
            for (int k = kf; k < k1; k += nt) {
                const bool first = k == kf;
                const double lw = first ? plw : b.logW[k];
                if (!(lw < LW_MAX)) continue;
                float n2 = 0.0f, dc[8], is2[8];
                for (int d = 0; d < D; d++) {
                    dc[d] = (float)(s[d] - (first ? pc[d] : b.centers[k * D + d]));
                    const float isg = __frcp_rn((float)(first ? ps[d] : b.sigmas[k * D + d]));
                    const float u = dc[d] * isg;
                    is2[d] = isg * isg;
                    n2 = fmaf(u, u, n2);
                }
                if (!(n2 < cut2)) continue;
                const float G = __expf(-0.5f * n2), kern = G - kfloor;
                if (kern <= 0.0f) continue;
                const float h = __expf((float)(lw - M));
                accF<MODE>(acc[8], cmp[8], h * kern);
                const float hG = h * G;
                for (int d = 0; d < D; d++) accF<MODE>(acc[d], cmp[d], hG * (-dc[d] * is2[d]));
            }
        } else {
            for (int k = k0 + tid; k < k1; k += nt) {
                double ex = 0;
                float dc[8];
                for (int d = 0; d < D; d++) {
                    double x = s[d] - b.hCenters[k * D + d];
                    if (b.period[d] > 0) x -= round(x / b.period[d]) * b.period[d];
                    dc[d] = (float)x;
                    ex += x * x / (2.0 * b.sigma[d] * b.sigma[d]);
                }
                if (ex > 8.0) continue;
                const float g = (float)b.hHeights[k] * __expf(-(float)ex);
                accF<MODE>(acc[8], cmp[8], g);
                for (int d = 0; d < D; d++) accF<MODE>(acc[d], cmp[d], -g * dc[d] * b.isg2f[d]);
            }
        }
        // warp tree (the compensation terms travel with their sums), then the
        // warps' partials in FP64, scaled by exp(M_w), summed in warp order
#pragma unroll
        for (int i = 0; i < 9; i++) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const float hs = __shfl_xor_sync(0xffffffffu, acc[i], o);
                if (MODE == SUM_FP32C) {
                    const float hc = __shfl_xor_sync(0xffffffffu, cmp[i], o);
                    cmp[i] = __fadd_rn(cmp[i], hc);
                    twoSumAcc(acc[i], cmp[i], hs);
                } else {
                    acc[i] = __fadd_rn(acc[i], hs);
                }
            }
        }
        if (lane == 0) {
            const double scale = type == BIAS_OPES ? (M > -INFINITY ? exp(M) : 0.0) : 1.0;
#pragma unroll
            for (int i = 0; i < 9; i++)
                red[warp * 9 + i] = ((double)acc[i] + (MODE == SUM_FP32C ? (double)cmp[i] : 0.0)) * scale;
        }
        __syncthreads();
        if (tid < 9) {
            double t = 0.0;
            for (int w = 0; w < (nt >> 5); w++) t += red[w * 9 + tid];
            part[((size_t)blockIdx.y * gridDim.x + blockIdx.x) * 9 + tid] = t;
        }
    }
}

__device__ __forceinline__ bool singleLaneBias(int t) {
    return t == BIAS_HARMONIC || t == BIAS_METAD || t == BIAS_PBMETAD || t == BIAS_EXTERNAL;
}

// Shared memory: sG[numCVs] | contrib[nb][8] | (stage) records[nb]. SINGLE: the
// context has single-lane biases (the instantiation without them carries none of
// their code, which matters when every step starts with cold caches).
template <bool SINGLE>
__global__ void __launch_bounds__(512) k_biases(const BiasDev* __restrict__ gbiases, int nb, int stage,
                                                 const double* __restrict__ cvv, int numCVs,
                                                 const double* __restrict__ testGrad, double* __restrict__ dUdCV,
                                                 double* __restrict__ energies, const double* __restrict__ sumPart) {
    extern __shared__ __align__(16) double sm[];
    __shared__ double red[32 * 9];
    const int tid = threadIdx.x, nt = blockDim.x, warp = tid >> 5, lane = tid & 31;
    double* sG = sm;
    double* contrib = sm + ((numCVs + 1) & ~1);
    const BiasDev* biases = gbiases;
    if (stage) {
        // records are written by the host between steps only: copy them while the
        // previous kernel finishes
        BiasDev* rec = reinterpret_cast<BiasDev*>(contrib + 8 * nb);
        const unsigned long long* src = reinterpret_cast<const unsigned long long*>(gbiases);
        unsigned long long* dst = reinterpret_cast<unsigned long long*>(rec);
        const int words = nb * (int)(sizeof(BiasDev) / 8);
        for (int i = tid; i < words; i += nt) dst[i] = src[i];
        biases = rec;
    }
    // OPES kernel counts and sum_uprob are written by the deposits only (see
    // k_kernel_sums): read them before the wait, one thread per bias
    __shared__ int sK[16];
    __shared__ double sSu[16];
    if (tid < nb && tid < 16 && gbiases[tid].type == BIAS_OPES) {
        sK[tid] = *gbiases[tid].numKernels;
        sSu[tid] = *gbiases[tid].sumUprob;
    }
    pdlEnter();
    for (int i = tid; i < numCVs; i += nt) sG[i] = testGrad ? testGrad[i] : 0.0;
    __syncthreads();
    if (!testGrad) {
        // single-lane biases, one warp each (CommonGluedKernels.cpp:2513-2540,
        // :3574-3636, :3698-3763; EXTERNAL through the MetaD grid,
        // CommonBiasKernels.cpp:425-488)
        if constexpr (SINGLE) {
            for (int bi = warp; bi < nb; bi += nt >> 5) {
                const BiasDev& b = biases[bi];
                if (lane != 0 || !singleLaneBias(b.type)) continue;
                double* out = contrib + 8 * bi;
                if (b.type == BIAS_HARMONIC) {
                    // k and s0 stored as float
                    const double TWO_PI = 6.283185307179586;
                    double V = 0;
                    for (int d = 0; d < b.D; d++) {
                        double ds = cvv[b.cvIdx[d]] - (double)b.hs0[d];
                        if (b.periodicFlag) ds -= TWO_PI * round(ds / TWO_PI);
                        V += 0.5 * (double)b.hk[d] * ds * ds;
                        out[d] = (double)b.hk[d] * ds;
                    }
                    energies[b.slot] = V;
                } else if (b.type == BIAS_PBMETAD) {
                    evalPbmetad(b, cvv, energies, out);
                } else {
                    evalMetadGrid(b, cvv, energies, out);
                }
            }
            __syncthreads();
        }
        for (int bi = 0; bi < nb; bi++) {
            const BiasDev& b = biases[bi];
            const int D = b.D;
            if (SINGLE && singleLaneBias(b.type)) {
                if (tid == 0)
                    for (int d = 0; d < D; d++) sG[b.cvIdx[d]] += contrib[8 * bi + d];
            } else if (b.type == BIAS_OPES) {
                // CommonGluedKernels.cpp:2642-2723.
                if (tid == 0 && b.adaptiveStride > 0) {
                    // every-execute Welford update (CommonGluedKernels.cpp:3009-3027, :4976-4981).
                    // Each operation rounded on its own (no FMA contraction): the
                    // statistics set the adaptive bandwidth, which enters the
                    // merge decisions that must match the oracle bit for bit.
                    int n = ++b.nSamples[0];
                    for (int d = 0; d < D; d++) {
                        double x = cvv[b.cvIdx[d]], dl = __dsub_rn(x, b.runMean[d]);
                        double mean = __dadd_rn(b.runMean[d], __ddiv_rn(dl, (double)n));
                        b.runMean[d] = mean;
                        b.runM2[d] = __dadd_rn(b.runM2[d], __dmul_rn(dl, __dsub_rn(x, mean)));
                    }
                }
                const int K = bi < 16 ? sK[bi] : *b.numKernels;
                if (K == 0) {
                    if (tid == 0) energies[b.slot] = -b.barrier;
                } else {
                    // kernel sum: partials of k_kernel_sums, summed in CTA order
                    double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
                    if (tid < KSUM_CTAS)
                        for (int i = 0; i < 9; i++) acc[i] = sumPart[((size_t)bi * KSUM_CTAS + tid) * 9 + i];
                    blockSum<9>(acc, red);
                    if (tid == 0) {
                        double prob = acc[8];
                        double su = bi < 16 ? sSu[bi] : *b.sumUprob;
                        double pz = su > 0.0 ? prob * (double)K / su : 0.0;
                        if (!(pz >= 0.0)) pz = 0.0;
                        double arg = pz + b.eps;
                        energies[b.slot] = b.invGF * b.kT * log(arg > 1e-30 ? arg : 1e-30);
                        if (prob > 0.0) {
                            double f = b.invGF * b.kT * (pz / (pz + b.eps)) / prob;
                            for (int d = 0; d < D; d++) sG[b.cvIdx[d]] += f * acc[d];
                        }
                    }
                }
                __syncthreads();
            }
        }
        for (int bi = 0; bi < nb; bi++) {
            const BiasDev& b = biases[bi];
            if (b.type != BIAS_METAD_HILLS) continue;
            // Direct hill sum, exponent > 8 truncated like the grid deposit.
            const int D = b.D;
            double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            if (tid < KSUM_CTAS)
                for (int i = 0; i < 9; i++) acc[i] = sumPart[((size_t)bi * KSUM_CTAS + tid) * 9 + i];
            blockSum<9>(acc, red);
            if (tid == 0) {
                energies[b.slot] = acc[8];
                for (int d = 0; d < D; d++) sG[b.cvIdx[d]] += acc[d];
            }
            __syncthreads();
        }
    }
    __syncthreads();
    for (int i = tid; i < numCVs; i += nt) dUdCV[i] = sG[i];
}

// The atom and CV columns of the Jacobian rows are written once when the plan is
// built and the user -> slot map at bind / reorder, long before this launch: the
// first row of every thread resolves its slot before the wait; the gradients and
// dU/dCV of this step are read after it.
__global__ void k_scatter(JacDev J, const int* __restrict__ u2g, const double* __restrict__ dUdCV,
                          unsigned long long* __restrict__ force, int padded) {
    const int rf = blockIdx.x * blockDim.x + threadIdx.x;
    int cvf = 0, af = 0;
    if (rf < J.rows) {
        cvf = J.cv[rf];
        af = u2g[J.atom[rf]];
    }
    pdlEnter();
    const double S = 4294967296.0;
    for (int r = rf; r < J.rows; r += gridDim.x * blockDim.x) {
        const bool first = r == rf;
        double g = dUdCV[first ? cvf : J.cv[r]];
        if (g == 0.0) continue;  // adds zero in the reference
        int a = first ? af : u2g[J.atom[r]];
        long long fx = (long long)(-(g * (double)J.gx[r]) * S);
        long long fy = (long long)(-(g * (double)J.gy[r]) * S);
        long long fz = (long long)(-(g * (double)J.gz[r]) * S);
        redAddGlobal(force + a, (unsigned long long)fx);
        redAddGlobal(force + a + padded, (unsigned long long)fy);
        redAddGlobal(force + a + 2 * padded, (unsigned long long)fz);
    }
}

// WT MetaD Gaussian deposit restricted to the exponent <= 8 window.
__global__ void k_metad_deposit(const BiasDev* __restrict__ bp, const double* __restrict__ cvv,
                                const double* __restrict__ energies) {
    const BiasDev& b = *bp;
    const int D = b.D;
    double V = energies[b.slot];
    double h = b.hif > 0.0 ? b.h0 * exp(-V * b.hif) : b.h0;
    double c[8];
    int lo[8], cnt[8];
    long long total = 1;
    for (int d = 0; d < D; d++) {
        c[d] = cvv[b.cvIdx[d]];
        double w = 4.0 * b.sigma[d];
        int l = (int)floor((c[d] - w - b.origin[d]) * b.invSp[d]) - 1;
        int u = (int)ceil((c[d] + w - b.origin[d]) * b.invSp[d]) + 1;
        if (b.per[d]) {
            int n = u - l + 1;
            cnt[d] = n < b.npts[d] ? n : b.npts[d];
            lo[d] = l;
        } else {
            if (l < 0) l = 0;
            if (u > b.npts[d] - 1) u = b.npts[d] - 1;
            lo[d] = l;
            cnt[d] = u >= l ? u - l + 1 : 0;
        }
        total *= cnt[d];
    }
    for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < total;
         w += (long long)gridDim.x * blockDim.x) {
        long long rem = w;
        int flat = 0;
        double ex = 0;
        for (int d = 0; d < D; d++) {
            int o = (int)(rem % cnt[d]);
            rem /= cnt[d];
            int bi = lo[d] + o;
            if (b.per[d]) { bi %= b.npts[d]; if (bi < 0) bi += b.npts[d]; }
            flat += bi * b.strides[d];
            double pos = b.origin[d] + (double)bi / b.invSp[d];
            double dc = pos - c[d];
            if (b.per[d]) {
                double L = (double)b.npts[d] / b.invSp[d];
                dc -= round(dc / L) * L;
            }
            ex += dc * dc / (2.0 * b.sigma[d] * b.sigma[d]);
        }
        if (ex <= 8.0) atomicAdd(b.grid + flat, h * exp(-ex));  // atomic: walkers may share the grid
    }
}

// Hill-sum MetaD: append one hill at the current CVs with the WT height.
__global__ void k_hills_deposit(const BiasDev* __restrict__ bp, const double* __restrict__ cvv,
                                const double* __restrict__ energies) {
    const BiasDev& b = *bp;
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int n = *b.hCount;
    if (n >= b.maxHills) return;
    double V = energies[b.slot];
    double h = b.hif > 0.0 ? b.h0 * exp(-V * b.hif) : b.h0;
    for (int d = 0; d < b.D; d++) b.hCenters[n * b.D + d] = cvv[b.cvIdx[d]];
    b.hHeights[n] = h;
    *b.hCount = n + 1;
}

void launchBiases(cudaStream_t s, const BiasDev* biases, int nb, const double* cvv, int numCVs,
                  const double* testGrad, double* dUdCV, double* energies, double* sumPart, bool kernelSums,
                  bool singleLane, int sumMode) {
    if (kernelSums && !testGrad && nb > 0) {
        if (sumMode == SUM_FP32)
            launchPdl(k_kernel_sums<SUM_FP32>, dim3(KSUM_CTAS, nb), dim3(256), 0, s, biases, cvv, sumPart);
        else if (sumMode == SUM_FP32C)
            launchPdl(k_kernel_sums<SUM_FP32C>, dim3(KSUM_CTAS, nb), dim3(256), 0, s, biases, cvv, sumPart);
        else
            launchPdl(k_kernel_sums<SUM_FP64>, dim3(KSUM_CTAS, nb), dim3(256), 0, s, biases, cvv, sumPart);
    }
    // sG (rounded to an even count, so what follows is 16-byte aligned), the
    // per-bias contributions, then the staged records when they fit in 48 KB
    static_assert(sizeof(BiasDev) % 8 == 0, "bias records are copied as 8-byte words");
    size_t smem = sizeof(double) * ((size_t)((numCVs + 1) & ~1) + 8 * (size_t)nb);
    if (smem == 0) smem = 16;
    int stage = smem + sizeof(BiasDev) * (size_t)nb <= 48 * 1024 ? 1 : 0;
    if (stage) smem += sizeof(BiasDev) * (size_t)nb;
    if (singleLane)
        launchPdl(k_biases<true>, dim3(1), dim3(512), smem, s, biases, nb, stage, cvv, numCVs, testGrad, dUdCV,
                  energies, sumPart);
    else
        launchPdl(k_biases<false>, dim3(1), dim3(512), smem, s, biases, nb, stage, cvv, numCVs, testGrad, dUdCV,
                  energies, sumPart);
}

void launchScatter(cudaStream_t s, const JacDev& J, const int* u2g, const double* dUdCV, long long* force,
                   int padded) {
    if (J.rows <= 0) return;
    int blocks = (J.rows + 255) / 256;
    if (blocks > 1184) blocks = 1184;
    launchPdl(k_scatter, dim3(blocks), dim3(256), 0, s, J, u2g, dUdCV, reinterpret_cast<unsigned long long*>(force), padded);
}

// PBMETAD deposit (CommonGluedKernels.cpp:3765-3797): sub-grid d receives a
// Gaussian at the current value of its CV with height w_d h0 exp(-V_d hif)
// (w_d h0 without well-tempering), V_d and w_d from the last evaluation,
// wherever the exponent is <= 8.
__global__ void k_pbmetad_deposit(const BiasDev* __restrict__ bp, const double* __restrict__ cvv) {
    const BiasDev& b = *bp;
    for (int d = 0; d < b.D; d++) {
        const double Vi = b.pbState[d], wi = b.pbState[b.D + d];
        const double height = b.hif > 0.0 ? wi * b.h0 * exp(-Vi * b.hif) : wi * b.h0;
        const double center = cvv[b.cvIdx[d]];
        double* g = b.grid + b.goff[d];
        const double s2 = 2.0 * b.sigma[d] * b.sigma[d];
        for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < b.npts[d]; idx += gridDim.x * blockDim.x) {
            const double pos = b.origin[d] + (double)idx / b.invSp[d];
            double dc = pos - center;
            if (b.per[d]) {
                const double period = (double)b.npts[d] / b.invSp[d];
                dc -= round(dc / period) * period;
            }
            const double ex = dc * dc / s2;
            if (ex <= 8.0) g[idx] += height * exp(-ex);
        }
    }
}

void launchPbmetadDeposit(cudaStream_t s, const BiasDev* b, const double* cvv, int maxPoints) {
    const int blocks = std::max(1, std::min(148, (maxPoints + 255) / 256));
    k_pbmetad_deposit<<<blocks, 256, 0, s>>>(b, cvv);
}

void launchMetadDeposit(cudaStream_t s, const BiasDev* b, const double* cvv, const double* energies) {
    k_metad_deposit<<<148, 256, 0, s>>>(b, cvv, energies);
}

void launchHillsDeposit(cudaStream_t s, const BiasDev* b, const double* cvv, const double* energies) {
    k_hills_deposit<<<1, 32, 0, s>>>(b, cvv, energies);
}

}  // namespace glued
