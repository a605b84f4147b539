// Bias evaluation, chain-rule scatter and MetaD deposition.
//
// k_biases : every bias of the context in the reference's evaluation order
//            (harmonic, OPES, MetaD grid, then this library's hill-sum MetaD;
//            CommonGluedKernels.cpp:4955-5026) inside one CTA. dU/dCV is
//            accumulated in shared memory and written once, so no separate
//            clearing pass is needed (the reference relies on OpenMM's autoclear,
//            :4244). Kernel/hill sums are split over all threads and reduced by a
//            fixed tree in FP64.
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

__device__ void evalMetadGrid(const BiasDev& b, const double* cvv, double* sG, double* energies) {
    // CommonGluedKernels.cpp:3574-3636, one thread.
    int lo[8], hi[8];
    double al[8];
    const int D = b.D;
    for (int d = 0; d < D; d++) {
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
    double V = 0, dV[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int c = 0; c < (1 << D); c++) {
        int flat = 0;
        for (int d = 0; d < D; d++) flat += (((c >> d) & 1) ? hi[d] : lo[d]) * b.strides[d];
        double val = b.grid[flat], w = 1;
        for (int d = 0; d < D; d++) w *= ((c >> d) & 1) ? al[d] : (1.0 - al[d]);
        V += w * val;
        for (int d = 0; d < D; d++) {
            double sg = ((c >> d) & 1) ? 1.0 : -1.0, wo = 1;
            for (int e = 0; e < D; e++) if (e != d) wo *= ((c >> e) & 1) ? al[e] : (1.0 - al[e]);
            dV[d] += sg * wo * val;
        }
    }
    energies[b.slot] = V;
    for (int d = 0; d < D; d++) sG[b.cvIdx[d]] += dV[d] * b.invSp[d];
}

// PBMETAD (CommonGluedKernels.cpp:3694-3760), one thread: sub-grid d is a 1-D
// grid over CV cvIdx[d], linearly interpolated (periodic wrap or clamp, as the
// MetaD grid); the sub-grid energies V_d combine as
// E = -kT (ln sum_d exp((Vmin - V_d)/kT) - ln N) + Vmin, and dE/ds_d = w_d dV_d/ds_d
// with the softmax weights w_d = exp((Vmin - V_d)/kT) / sum. V_d and w_d are kept
// in pbState for the deposit.
__device__ void evalPbmetad(const BiasDev& b, const double* cvv, double* sG, double* energies) {
    const int N = b.D;
    double V[8], G[8];
    for (int d = 0; d < N; d++) {
        const double* g = b.grid + b.goff[d];
        const int n = b.npts[d];
        double fr = (cvv[b.cvIdx[d]] - b.origin[d]) * b.invSp[d];
        int lo, hi;
        double al;
        if (b.per[d]) {
            fr = fr - floor(fr / (double)n) * (double)n;
            if (fr < 0.0) fr += n;
            lo = (int)fr;
            if (lo >= n) lo = n - 1;
            al = fr - lo;
            hi = (lo + 1) % n;
        } else {
            if (fr < 0.0) fr = 0.0;
            if (fr > (double)(n - 1)) fr = (double)(n - 1);
            lo = (int)fr;
            if (lo >= n - 1) lo = n - 2;
            al = fr - lo;
            hi = lo + 1;
        }
        V[d] = g[lo] * (1.0 - al) + g[hi] * al;
        G[d] = (g[hi] - g[lo]) * b.invSp[d];
    }
    double vmin = V[0];
    for (int d = 1; d < N; d++) vmin = V[d] < vmin ? V[d] : vmin;
    double ene = 0.0;
    for (int d = 0; d < N; d++) ene += exp((vmin - V[d]) / b.kT);
    energies[b.slot] = -b.kT * (log(ene) - log((double)N)) + vmin;
    for (int d = 0; d < N; d++) {
        const double w = exp((vmin - V[d]) / b.kT) / ene;
        b.pbState[d] = V[d];
        b.pbState[N + d] = w;
        sG[b.cvIdx[d]] += w * G[d];
    }
}

// Kernel sums of the OPES and hill-sum MetaD biases (CommonGluedKernels.cpp:2642-2700
// for OPES), spread over KSUM_CTAS CTAs per bias: each CTA sums a contiguous
// range of kernels (per thread, then a fixed block tree) into 9 FP64 partials
// {dV/ds_0..7 terms, value}; k_biases sums the partials in CTA order.
__global__ void __launch_bounds__(256) k_kernel_sums(const BiasDev* __restrict__ biases,
                                                      const double* __restrict__ cvv, double* __restrict__ part) {
    pdlEnter();
    __shared__ double red[32 * 9];
    const BiasDev& b = biases[blockIdx.y];
    if (b.type != BIAS_OPES && b.type != BIAS_METAD_HILLS) return;  // uniform over the CTA
    const int tid = threadIdx.x, nt = blockDim.x;
    const int D = b.D;
    const int K = b.type == BIAS_OPES ? *b.numKernels : *b.hCount;
    const int k0 = (int)((long long)K * blockIdx.x / gridDim.x);
    const int k1 = (int)((long long)K * (blockIdx.x + 1) / gridDim.x);
    double s[8];
    for (int d = 0; d < D; d++) s[d] = cvv[b.cvIdx[d]];
    double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (b.type == BIAS_OPES) {
        const double kfloor = exp(-0.5 * b.cutoff2);
        for (int k = k0 + tid; k < k1; k += nt) {
            double n2 = 0, dc[8], is2[8];
            for (int d = 0; d < D; d++) {
                dc[d] = s[d] - b.centers[k * D + d];
                double sg = b.sigmas[k * D + d];
                is2[d] = 1.0 / (sg * sg);
                n2 += dc[d] * dc[d] * is2[d];
            }
            if (!(n2 < b.cutoff2)) continue;
            double G = exp(-0.5 * n2), kern = G - kfloor;
            if (kern <= 0.0) continue;
            double h = exp(b.logW[k]);
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
}

__global__ void __launch_bounds__(512) k_biases(const BiasDev* __restrict__ biases, int nb,
                                                 const double* __restrict__ cvv, int numCVs,
                                                 const double* __restrict__ testGrad, double* __restrict__ dUdCV,
                                                 double* __restrict__ energies, const double* __restrict__ sumPart) {
    pdlEnter();
    extern __shared__ double sG[];
    __shared__ double red[32 * 9];
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int i = tid; i < numCVs; i += nt) sG[i] = testGrad ? testGrad[i] : 0.0;
    __syncthreads();
    if (!testGrad) {
        for (int bi = 0; bi < nb; bi++) {
            const BiasDev& b = biases[bi];
            const int D = b.D;
            if (b.type == BIAS_HARMONIC) {
                // CommonGluedKernels.cpp:2513-2540; k and s0 stored as float.
                if (tid == 0) {
                    const double TWO_PI = 6.283185307179586;
                    double V = 0;
                    for (int d = 0; d < D; d++) {
                        double ds = cvv[b.cvIdx[d]] - (double)b.hs0[d];
                        if (b.periodicFlag) ds -= TWO_PI * round(ds / TWO_PI);
                        V += 0.5 * (double)b.hk[d] * ds * ds;
                        sG[b.cvIdx[d]] += (double)b.hk[d] * ds;
                    }
                    energies[b.slot] = V;
                }
            } else if (b.type == BIAS_METAD) {
                if (tid == 0) evalMetadGrid(b, cvv, sG, energies);
            } else if (b.type == BIAS_PBMETAD) {
                if (tid == 0) evalPbmetad(b, cvv, sG, energies);
            } else if (b.type == BIAS_EXTERNAL) {
                // user grid, evaluated as the MetaD grid (CommonBiasKernels.cpp:425-488)
                if (tid == 0) evalMetadGrid(b, cvv, sG, energies);
            } else if (b.type == BIAS_OPES) {
                // CommonGluedKernels.cpp:2642-2723.
                if (tid == 0 && b.adaptiveStride > 0) {
                    // every-execute Welford update (CommonGluedKernels.cpp:3009-3027, :4976-4981)
                    int n = ++b.nSamples[0];
                    for (int d = 0; d < D; d++) {
                        double x = cvv[b.cvIdx[d]], dl = x - b.runMean[d];
                        b.runMean[d] += dl / n;
                        b.runM2[d] += dl * (x - b.runMean[d]);
                    }
                }
                const int K = *b.numKernels;
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
                        double su = *b.sumUprob;
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
            }
            __syncthreads();
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
    for (int i = tid; i < numCVs; i += nt) dUdCV[i] = sG[i];
}

__global__ void k_scatter(JacDev J, const int* __restrict__ u2g, const double* __restrict__ dUdCV,
                          unsigned long long* __restrict__ force, int padded) {
    pdlEnter();
    const double S = 4294967296.0;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < J.rows; r += gridDim.x * blockDim.x) {
        double g = dUdCV[J.cv[r]];
        if (g == 0.0) continue;  // adds zero in the reference
        int a = u2g[J.atom[r]];
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
                  const double* testGrad, double* dUdCV, double* energies, double* sumPart, bool kernelSums) {
    if (kernelSums && !testGrad && nb > 0) launchPdl(k_kernel_sums, dim3(KSUM_CTAS, nb), dim3(256), 0, s, biases, cvv, sumPart);
    size_t smem = sizeof(double) * (size_t)(numCVs > 0 ? numCVs : 1);
    launchPdl(k_biases, dim3(1), dim3(512), smem, s, biases, nb, cvv, numCVs, testGrad, dUdCV, energies, sumPart);
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
