// CV kernels of the plain per-context path.
//   k_simple_cvs : distance / angle / dihedral, one thread per CV
//                  (CommonGluedKernels.cpp:177-444)
//   k_group_cvs  : one CTA per CV for the group CVs (COM distance, gyration, RMSD,
//                  PCA, path, contact map, Kabsch RMSD) with deterministic block
//                  reductions instead of the reference's one-thread loops
//                  (CommonGluedKernels.cpp:456-881, :1236-1323, :1633-1681)
//   k_group_cvs_cluster: COM distance, gyration, RMSD and PCA over a cluster of
//                  GROUP_CLUSTER CTAs per CV when the groups are large: each CTA
//                  gathers and processes a contiguous slice of the atoms, and the
//                  per-CTA sums are added through distributed shared memory in
//                  rank order, so every CTA holds the same totals
//   k_test_force : setTestForce modes 1-3 (CommonGluedKernels.cpp:114-164)
//   k_invert_index: user -> GPU slot map from OpenMM's atomIndexArray
// Values go to cvValues (double); Jacobian gradients to the float SoA table whose
// atom / CV columns are written once when the plan is built.
#include <algorithm>

#include <cooperative_groups.h>

#include "context.hpp"
#include "devfn.cuh"
#include "kernels.hpp"
#include "pdl.cuh"
#include "force.hpp"

namespace glued {

__global__ void k_invert_index(const int* __restrict__ atomIndex, int* __restrict__ u2g, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        int u = atomIndex ? atomIndex[i] : i;
        if (u >= 0 && u < n) u2g[u] = i;
    }
}

// slot[k] = u2g[atoms[k]] for the distance / angle / dihedral items: the posq
// row of each atom, rebuilt whenever OpenMM reorders atoms, so the CV kernel
// reads positions without the map.
__global__ void k_compose_simple_slots(SimpleItem* __restrict__ items, const int* __restrict__ u2g, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int na = items[i].type == CV_DISTANCE ? 2 : items[i].type == CV_ANGLE ? 3 : 4;
    for (int k = 0; k < na; k++) items[i].slot[k] = u2g[items[i].atoms[k]];
}

__device__ __forceinline__ void simpleCvItem(const float4* __restrict__ posq, const int* __restrict__ u2g,
                                             const SimpleItem* __restrict__ items, int i,
                                             const BoxDev* __restrict__ boxp, double* __restrict__ cvv, JacDev& J) {
    const BoxDev box = *boxp;
    SimpleItem it = items[i];
    int r = it.jac0;
    if (it.type == CV_DISTANCE) {
        F3 d = minImage(sub3(loadPos(posq, nullptr, it.slot[1]), loadPos(posq, nullptr, it.slot[0])), box);
        float dist = sqrtf(dot3(d, d));
        float inv = dist > 1e-10f ? 1.0f / dist : 0.0f;
        cvv[it.cv] = (double)dist;
        J.gx[r] = -d.x * inv; J.gy[r] = -d.y * inv; J.gz[r] = -d.z * inv;
        J.gx[r + 1] = d.x * inv; J.gy[r + 1] = d.y * inv; J.gz[r + 1] = d.z * inv;
    } else if (it.type == CV_ANGLE) {
        F3 pb = loadPos(posq, nullptr, it.slot[1]);
        F3 d1 = minImage(sub3(loadPos(posq, nullptr, it.slot[0]), pb), box);
        F3 d2 = minImage(sub3(loadPos(posq, nullptr, it.slot[2]), pb), box);
        float r1 = sqrtf(dot3(d1, d1)), r2 = sqrtf(dot3(d2, d2));
        float i1 = r1 > 1e-10f ? 1.0f / r1 : 0.0f, i2 = r2 > 1e-10f ? 1.0f / r2 : 0.0f;
        F3 n1 = f3(d1.x * i1, d1.y * i1, d1.z * i1), n2 = f3(d2.x * i2, d2.y * i2, d2.z * i2);
        float ct = fmaxf(-1.0f, fminf(1.0f, dot3(n1, n2)));
        float th = acosf(ct);
        float st = sqrtf(1.0f - ct * ct);
        float is = st > 1e-6f ? 1.0f / st : 0.0f;
        cvv[it.cv] = (double)th;
        float s1 = i1 * is, s2 = i2 * is;
        F3 jA = f3(-(n2.x - ct * n1.x) * s1, -(n2.y - ct * n1.y) * s1, -(n2.z - ct * n1.z) * s1);
        F3 jC = f3(-(n1.x - ct * n2.x) * s2, -(n1.y - ct * n2.y) * s2, -(n1.z - ct * n2.z) * s2);
        J.gx[r] = jA.x; J.gy[r] = jA.y; J.gz[r] = jA.z;
        J.gx[r + 1] = -(jA.x + jC.x); J.gy[r + 1] = -(jA.y + jC.y); J.gz[r + 1] = -(jA.z + jC.z);
        J.gx[r + 2] = jC.x; J.gy[r + 2] = jC.y; J.gz[r + 2] = jC.z;
    } else {  // dihedral, Blondel-Karplus
        F3 pa = loadPos(posq, nullptr, it.slot[0]), pb = loadPos(posq, nullptr, it.slot[1]);
        F3 pc = loadPos(posq, nullptr, it.slot[2]), pd = loadPos(posq, nullptr, it.slot[3]);
        F3 b1 = minImage(sub3(pb, pa), box), b2 = minImage(sub3(pc, pb), box), b3 = minImage(sub3(pd, pc), box);
        F3 t = cross3(b1, b2), u = cross3(b2, b3);
        float d = sqrtf(dot3(b2, b2));
        float t2 = dot3(t, t), u2 = dot3(u, u);
        float phi = atan2f(d * dot3(b1, u), dot3(t, u));
        cvv[it.cv] = (double)phi;
        float it2 = t2 > 1e-10f ? 1.0f / t2 : 0.0f;
        float iu2 = u2 > 1e-10f ? 1.0f / u2 : 0.0f;
        float id = d > 1e-10f ? 1.0f / d : 0.0f;
        float c1 = dot3(b1, b2) * id, c2 = dot3(b3, b2) * id;
        float aT = d * it2, aU = d * iu2, bTB = (d + c1) * it2, bUB = c2 * iu2;
        F3 jA = f3(-aT * t.x, -aT * t.y, -aT * t.z);
        F3 jD = f3(aU * u.x, aU * u.y, aU * u.z);
        F3 jB = f3(bTB * t.x + bUB * u.x, bTB * t.y + bUB * u.y, bTB * t.z + bUB * u.z);
        J.gx[r] = jA.x; J.gy[r] = jA.y; J.gz[r] = jA.z;
        J.gx[r + 1] = jB.x; J.gy[r + 1] = jB.y; J.gz[r + 1] = jB.z;
        J.gx[r + 2] = -(jA.x + jB.x + jD.x); J.gy[r + 2] = -(jA.y + jB.y + jD.y); J.gz[r + 2] = -(jA.z + jB.z + jD.z);
        J.gx[r + 3] = jD.x; J.gy[r + 3] = jD.y; J.gz[r + 3] = jD.z;
    }
}

// LATE: launched beside the plain-launched coordination grid, as for the group
// CVs (k_group_cvs): computes first, waits for the grid only at its end.
template <bool LATE>
__global__ void k_simple_cvs(const float4* __restrict__ posq, const int* __restrict__ u2g,
                             const SimpleItem* __restrict__ items, int n, const BoxDev* __restrict__ boxp,
                             double* __restrict__ cvv, JacDev J) {
    if constexpr (LATE)
        asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    else
        pdlEnter();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) simpleCvItem(posq, u2g, items, i, boxp, cvv, J);
    if constexpr (LATE) asm volatile("griddepcontrol.wait;" ::: "memory");
}

// ---------------------------------------------------------------- group CVs

// Jacobi eigen-decomposition of a symmetric 4x4 in FP64 (quaternion RMSD).
// Largest eigenvalue and a unit eigenvector of a symmetric, traceless 4x4 F
// (the quaternion key matrix of optimal superposition), in FP64 on one thread:
//   - lambda by Newton on the characteristic polynomial
//     P(l) = l^4 - (tr F^2 / 2) l^2 - (tr F^3 / 3) l + det F, started at an upper
//     bound `upper` of the spectrum, from which it descends monotonically to the
//     largest root;
//   - the eigenvector by two steps of inverse iteration with (F - mu I), mu
//     just above lambda (Gaussian elimination with partial pivoting), which
//     also serves a nearly double largest eigenvalue;
//   - lambda again as the Rayleigh quotient of that vector.
// A handful of divisions in all, against about 200 divisions and square roots
// of a cyclic Jacobi solve, whose serial latency was ~10 us per Kabsch CV.
__device__ __forceinline__ void maxEigen4(const double (&F)[4][4], double upper, double& lam, double (&v)[4]) {
    double p2 = 0.0, p3 = 0.0;
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) {
            double f2 = 0.0;
#pragma unroll
            for (int k = 0; k < 4; k++) f2 += F[i][k] * F[k][j];
            p2 += F[i][j] * F[j][i];
            p3 += F[i][j] * f2;   // (F F^2)_ii summed: tr F^3 (F symmetric)
        }
    // det F by elimination with partial pivoting on a copy
    double M[4][4];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) M[i][j] = F[i][j];
    double det = 1.0;
#pragma unroll
    for (int c = 0; c < 4; c++) {
        int piv = c;
#pragma unroll
        for (int r = c + 1; r < 4; r++)
            if (fabs(M[r][c]) > fabs(M[piv][c])) piv = r;
        if (piv != c) {
            det = -det;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                // swap rows c and piv with compile-time row indices only
                double a = M[c][j], b = 0.0;
#pragma unroll
                for (int r = c + 1; r < 4; r++) b = (r == piv) ? M[r][j] : b;
                M[c][j] = b;
#pragma unroll
                for (int r = c + 1; r < 4; r++)
                    if (r == piv) M[r][j] = a;
            }
        }
        const double d = M[c][c];
        det *= d;
        if (d != 0.0) {
            const double id = 1.0 / d;
#pragma unroll
            for (int r = c + 1; r < 4; r++) {
                const double f = M[r][c] * id;
#pragma unroll
                for (int j = c; j < 4; j++) M[r][j] -= f * M[c][j];
            }
        }
    }
    const double c2 = -0.5 * p2, c1 = -p3 / 3.0, c0 = det;
    double l = upper;
    for (int it = 0; it < 100; it++) {
        const double P = ((l * l + c2) * l + c1) * l + c0;
        const double dP = (4.0 * l * l + 2.0 * c2) * l + c1;
        if (!(dP > 0.0)) break;
        const double step = P / dP;
        l -= step;
        if (fabs(step) <= 1e-15 * fabs(l) + 1e-300) break;
    }
    // inverse iteration with mu slightly above lambda
    const double mu = l + 1e-12 * (fabs(l) + fabs(upper)) + 1e-300;
    double x[4] = {1.0, 1.0, 1.0, 1.0};
    for (int rep = 0; rep < 2; rep++) {
        double A[4][5];
#pragma unroll
        for (int i = 0; i < 4; i++) {
#pragma unroll
            for (int j = 0; j < 4; j++) A[i][j] = F[i][j] - (i == j ? mu : 0.0);
            A[i][4] = x[i];
        }
#pragma unroll
        for (int c = 0; c < 4; c++) {
            int piv = c;
#pragma unroll
            for (int r = c + 1; r < 4; r++)
                if (fabs(A[r][c]) > fabs(A[piv][c])) piv = r;
#pragma unroll
            for (int j = 0; j < 5; j++) {
                double a = A[c][j], b = a;
#pragma unroll
                for (int r = c + 1; r < 4; r++) b = (r == piv) ? A[r][j] : b;
                A[c][j] = b;
#pragma unroll
                for (int r = c + 1; r < 4; r++)
                    if (r == piv) A[r][j] = a;
            }
            const double d = A[c][c] != 0.0 ? A[c][c] : 1e-300;
            const double id = 1.0 / d;
#pragma unroll
            for (int r = c + 1; r < 4; r++) {
                const double f = A[r][c] * id;
#pragma unroll
                for (int j = c; j < 5; j++) A[r][j] -= f * A[c][j];
            }
        }
        double y[4];
#pragma unroll
        for (int c = 3; c >= 0; c--) {
            double t = A[c][4];
#pragma unroll
            for (int j = c + 1; j < 4; j++) t -= A[c][j] * y[j];
            y[c] = t / (A[c][c] != 0.0 ? A[c][c] : 1e-300);
        }
        const double n = sqrt(y[0] * y[0] + y[1] * y[1] + y[2] * y[2] + y[3] * y[3]);
        const double in = n > 0.0 ? 1.0 / n : 0.0;
#pragma unroll
        for (int i = 0; i < 4; i++) x[i] = y[i] * in;
    }
    double rq = 0.0;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        double fx = 0.0;
#pragma unroll
        for (int j = 0; j < 4; j++) fx += F[i][j] * x[j];
        rq += x[i] * fx;
        v[i] = x[i];
    }
    lam = rq;
}

// Positions of the group atoms [a0, a1) are gathered once into shared memory
// (through the precomposed posq rows, GATHER_U loads in flight per thread) when
// the group fits GROUP_CACHE atoms; every pass of the CV then reads them there.
constexpr int GROUP_CACHE = 8192;
constexpr int GROUP_THREADS = 512;
constexpr int GATHER_U = 16;

// LATE: launched as the programmatic dependent of the plain-launched coordination
// grid, on the SMs that grid leaves free; everything it reads was complete before
// that grid started and it writes nothing the grid reads, so it computes first and
// waits for the grid only at its end (which keeps the chain's completion order).
template <bool LATE>
__global__ void __launch_bounds__(GROUP_THREADS) k_group_cvs(const float4* __restrict__ posq,
                                                             const int* __restrict__ u2g, GroupDev G,
                                                             const BoxDev* __restrict__ boxp,
                                                             double* __restrict__ cvv, JacDev J) {
    if constexpr (LATE)
        asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    else
        pdlEnter();
    extern __shared__ float4 sPos[];
    __shared__ double red[32 * 16];
    __shared__ float wbuf[128];
    __shared__ double bc[16];
    const GroupItem it = (int)blockIdx.x < G.nInl ? G.inl[blockIdx.x] : G.items[blockIdx.x];
    const BoxDev box = *boxp;
    const int tid = threadIdx.x, nt = blockDim.x;
    // atoms read through pos(j): cached when the group fits
    int a0 = it.s0, a1 = it.s1;
    if (it.type == CV_COM_DISTANCE) a1 = it.s2;
    const bool cached = it.type != CV_CONTACTMAP && a1 - a0 <= GROUP_CACHE;
    if (cached) {
        const int n = a1 - a0;
        // masses (COM distance, gyration) ride in the .w lane of the cache
        const bool withMass = it.type == CV_COM_DISTANCE || it.type == CV_GYRATION;
        for (int base = tid; base < n; base += nt * GATHER_U) {
            int slot[GATHER_U];
            float m[GATHER_U];
#pragma unroll
            for (int u = 0; u < GATHER_U; u++) {
                const int j = base + nt * u;
                slot[u] = j < n ? __ldg(G.slots + a0 + j) : -1;
                m[u] = (withMass && j < n) ? __ldg(G.mass + a0 + j) : 0.0f;
            }
#pragma unroll
            for (int u = 0; u < GATHER_U; u++)
                if (slot[u] >= 0) {
                    float4 p = __ldg(posq + slot[u]);
                    p.w = m[u];
                    sPos[base + nt * u] = p;
                }
        }
        __syncthreads();
    }
    auto pos = [&](int j) -> F3 {
        if (cached) { const float4 p = sPos[j - a0]; return f3(p.x, p.y, p.z); }
        return loadPos(posq, nullptr, G.slots[j]);
    };
    auto massAt = [&](int j) -> float { return cached ? sPos[j - a0].w : G.mass[j]; };

    if (it.type == CV_COM_DISTANCE) {
        double v[6] = {0, 0, 0, 0, 0, 0};
        for (int j = it.s0 + tid; j < it.s2; j += nt) {
            F3 p = pos(j);
            double m = massAt(j);
            int o = j < it.s1 ? 0 : 3;
            v[o] += m * p.x; v[o + 1] += m * p.y; v[o + 2] += m * p.z;
        }
        blockSum<6>(v, red);
        float i1 = 1.0f / it.f0, i2 = 1.0f / it.f1;
        F3 c1 = f3((float)v[0] * i1, (float)v[1] * i1, (float)v[2] * i1);
        F3 c2 = f3((float)v[3] * i2, (float)v[4] * i2, (float)v[5] * i2);
        F3 d = minImage(sub3(c2, c1), box);
        float dist = sqrtf(dot3(d, d));
        float inv = dist > 1e-10f ? 1.0f / dist : 0.0f;
        if (tid == 0) cvv[it.cv] = (double)dist;
        for (int j = it.s0 + tid; j < it.s2; j += nt) {
            bool g1 = j < it.s1;
            float w = massAt(j) / (g1 ? it.f0 : it.f1);
            float s = g1 ? -inv * w : inv * w;
            int r = it.jac0 + j;
            J.gx[r] = d.x * s; J.gy[r] = d.y * s; J.gz[r] = d.z * s;
        }
    } else if (it.type == CV_GYRATION) {
        double v[3] = {0, 0, 0};
        for (int j = it.s0 + tid; j < it.s1; j += nt) {
            F3 p = pos(j);
            double m = massAt(j);
            v[0] += m * p.x; v[1] += m * p.y; v[2] += m * p.z;
        }
        blockSum<3>(v, red);
        float iM = 1.0f / it.f0;
        F3 com = f3((float)v[0] * iM, (float)v[1] * iM, (float)v[2] * iM);
        double q[1] = {0};
        for (int j = it.s0 + tid; j < it.s1; j += nt) {
            F3 d = minImage(sub3(pos(j), com), box);
            q[0] += (double)massAt(j) * (double)dot3(d, d);
        }
        blockSum<1>(q, red);
        float rg = (float)sqrt(q[0] / (double)it.f0);
        float irg = rg > 1e-10f ? 1.0f / rg : 0.0f;
        if (tid == 0) cvv[it.cv] = (double)rg;
        for (int j = it.s0 + tid; j < it.s1; j += nt) {
            F3 d = minImage(sub3(pos(j), com), box);
            float w = massAt(j) / it.f0;
            int r = it.jac0 + j;
            J.gx[r] = w * d.x * irg; J.gy[r] = w * d.y * irg; J.gz[r] = w * d.z * irg;
        }
    } else if (it.type == CV_RMSD) {
        double q[1] = {0};
#pragma unroll 4
        for (int j = it.s0 + tid; j < it.s1; j += nt) {
            F3 p = pos(j);
            F3 d = f3(p.x - G.ref[3 * j], p.y - G.ref[3 * j + 1], p.z - G.ref[3 * j + 2]);
            q[0] += (double)dot3(d, d);
        }
        blockSum<1>(q, red);
        int na = it.s1 - it.s0;
        float rmsd = (float)sqrt(q[0] / na);
        float sc = (rmsd > 1e-10f ? 1.0f / rmsd : 0.0f) / (float)na;
        if (tid == 0) cvv[it.cv] = (double)rmsd;
#pragma unroll 4
        for (int j = it.s0 + tid; j < it.s1; j += nt) {
            F3 p = pos(j);
            int r = it.jac0 + j;
            J.gx[r] = (p.x - G.ref[3 * j]) * sc; J.gy[r] = (p.y - G.ref[3 * j + 1]) * sc;
            J.gz[r] = (p.z - G.ref[3 * j + 2]) * sc;
        }
    } else if (it.type == CV_PCA) {
        double q[1] = {0};
#pragma unroll 4
        for (int j = it.s0 + tid; j < it.s1; j += nt) {
            F3 p = pos(j);
            float dx = p.x - G.ref[3 * j], dy = p.y - G.ref[3 * j + 1], dz = p.z - G.ref[3 * j + 2];
            q[0] += (double)(dx * G.ev[3 * j] + dy * G.ev[3 * j + 1] + dz * G.ev[3 * j + 2]);
        }
        blockSum<1>(q, red);
        if (tid == 0) cvv[it.cv] = q[0];
        for (int j = it.s0 + tid; j < it.s1; j += nt) {
            int r = it.jac0 + j;
            J.gx[r] = G.ev[3 * j]; J.gy[r] = G.ev[3 * j + 1]; J.gz[r] = G.ev[3 * j + 2];
        }
    } else if (it.type == CV_PATH) {
        // Frames are 1-indexed in s (CommonGluedKernels.cpp:716-738); the frame
        // weights are cached as float like the reference's wBuf.
        const int M = it.s1 - it.s0, N = it.n;
        const float lam = it.f0;
        const int lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
        for (int f = warp; f < N; f += nw) {
            float acc = 0.0f;
            const float* rf = G.ref + 3 * (it.r0 + f * M);
            for (int j = lane; j < M; j += 32) {
                F3 p = pos(it.s0 + j);
                float dx = p.x - rf[3 * j], dy = p.y - rf[3 * j + 1], dz = p.z - rf[3 * j + 2];
                acc += dx * dx + dy * dy + dz * dz;
            }
            acc = warpSumF(acc);
            if (lane == 0) wbuf[f] = expf(-lam * (acc / (float)M));
        }
        __syncthreads();
        if (tid == 0) {
            double S = 0, sn = 0;
            for (int f = 0; f < N; f++) { S += wbuf[f]; sn += (double)(f + 1) * wbuf[f]; }
            double s = S > 1e-300 ? sn / S : 0.0;
            double z = S > 1e-300 ? -log(S) / lam : 0.0;
            cvv[it.cv] = s; cvv[it.cv + 1] = z;
            bc[0] = s; bc[1] = S;
        }
        __syncthreads();
        float s = (float)bc[0], S = (float)bc[1];
        float scS = -2.0f * lam / ((float)M * S), scZ = 2.0f / ((float)M * S);
        for (int j = tid; j < M; j += nt) {
            F3 p = pos(it.s0 + j);
            float sx = 0, sy = 0, sz = 0, zx = 0, zy = 0, zz = 0;
            for (int f = 0; f < N; f++) {
                const float* rf = G.ref + 3 * (it.r0 + f * M + j);
                float dx = p.x - rf[0], dy = p.y - rf[1], dz = p.z - rf[2];
                float w = wbuf[f], fs = ((float)(f + 1) - s) * w;
                sx += fs * dx; sy += fs * dy; sz += fs * dz;
                zx += w * dx; zy += w * dy; zz += w * dz;
            }
            int r = it.jac0 + 2 * j;
            J.gx[r] = scS * sx; J.gy[r] = scS * sy; J.gz[r] = scS * sz;
            J.gx[r + 1] = scZ * zx; J.gy[r + 1] = scZ * zy; J.gz[r + 1] = scZ * zz;
        }
    } else if (it.type == CV_CONTACTMAP) {
        double q[1] = {0};
        for (int p = it.s0 + tid; p < it.s1; p += nt) {
            int2 pr = G.cmPairs[p];
            float4 prm = G.cmParams[p];
            F3 d = minImage(sub3(loadPos(posq, u2g, pr.y), loadPos(posq, u2g, pr.x)), box);
            float dist = sqrtf(dot3(d, d));
            float idist = dist > 1e-10f ? 1.0f / dist : 0.0f;
            float ir0 = 1.0f / prm.x, x = dist * ir0;
            int nn = (int)prm.y, mm = (int)prm.z;
            float s, dsdd;
            if (nn >= 1 && mm >= 1 && nn <= 64 && mm <= 64) {
                // cancellation-free form of (1 - x^n)/(1 - x^m) (see ratioSwitch)
                float dsdx;
                ratioSwitch(x, nn, mm, s, dsdx);
                dsdd = dsdx * ir0;
            } else {
                // reference formula (CommonGluedKernels.cpp:1283-1300)
                float xn = 1.0f, xm = 1.0f, xn1 = 1.0f, xm1 = 1.0f;
                for (int k = 0; k < nn; k++) { xn1 = xn; xn *= x; }
                for (int k = 0; k < mm; k++) { xm1 = xm; xm *= x; }
                float num = 1.0f - xn, den = 1.0f - xm;
                if (fabsf(den) < 1e-8f) { s = (float)nn / (float)mm; dsdd = 0.0f; }
                else {
                    s = num / den;
                    float dxn = nn > 0 ? (float)nn * xn1 : 0.0f;
                    float dxm = mm > 0 ? (float)mm * xm1 : 0.0f;
                    dsdd = ((-dxn * den + dxm * num) / (den * den)) * ir0;
                }
            }
            q[0] += (double)(prm.w * s);
            float co = prm.w * dsdd * idist;
            int r = it.jac0 + 2 * (p - it.s0);
            J.gx[r] = -co * d.x; J.gy[r] = -co * d.y; J.gz[r] = -co * d.z;
            J.gx[r + 1] = co * d.x; J.gy[r + 1] = co * d.y; J.gz[r + 1] = co * d.z;
        }
        blockSum<1>(q, red);
        if (tid == 0) cvv[it.cv] = q[0];
    } else if (it.type == CV_RMSD_KABSCH) {
        // Optimal superposition RMSD: FP64 centroids and correlation matrix, the
        // quaternion 4x4 eigenproblem solved in FP64 by one thread (maxEigen4).
        const int na = it.s1 - it.s0;
        double v[6] = {0, 0, 0, 0, 0, 0};
        for (int j = it.s0 + tid; j < it.s1; j += nt) {
            F3 p = pos(j);
            v[0] += p.x; v[1] += p.y; v[2] += p.z;
            v[3] += G.ref[3 * j]; v[4] += G.ref[3 * j + 1]; v[5] += G.ref[3 * j + 2];
        }
        blockSum<6>(v, red);
        double xc[3] = {v[0] / na, v[1] / na, v[2] / na}, yc[3] = {v[3] / na, v[4] / na, v[5] / na};
        double c[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int j = it.s0 + tid; j < it.s1; j += nt) {
            F3 p = pos(j);
            double x[3] = {p.x - xc[0], p.y - xc[1], p.z - xc[2]};
            double y[3] = {G.ref[3 * j] - yc[0], G.ref[3 * j + 1] - yc[1], G.ref[3 * j + 2] - yc[2]};
            for (int a = 0; a < 3; a++) for (int b = 0; b < 3; b++) c[3 * a + b] += x[a] * y[b];
            c[9] += x[0] * x[0] + x[1] * x[1] + x[2] * x[2] + y[0] * y[0] + y[1] * y[1] + y[2] * y[2];
        }
        blockSum<10>(c, red);
        if (tid == 0) {
            double (*R)[3] = reinterpret_cast<double (*)[3]>(c);
            double F[4][4] = {
                {R[0][0] + R[1][1] + R[2][2], R[1][2] - R[2][1], R[2][0] - R[0][2], R[0][1] - R[1][0]},
                {R[1][2] - R[2][1], R[0][0] - R[1][1] - R[2][2], R[0][1] + R[1][0], R[0][2] + R[2][0]},
                {R[2][0] - R[0][2], R[0][1] + R[1][0], -R[0][0] + R[1][1] - R[2][2], R[1][2] + R[2][1]},
                {R[0][1] - R[1][0], R[0][2] + R[2][0], R[1][2] + R[2][1], -R[0][0] - R[1][1] + R[2][2]}};
            // largest eigenvalue (bounded above by (sum |x|^2 + sum |y|^2) / 2) and its
            // eigenvector
            double wm, q[4];
            maxEigen4(F, 0.5 * c[9], wm, q);
            const double q0 = q[0], q1 = q[1], q2 = q[2], q3 = q[3];
            // q rotates x onto y (correlation x y^T); bc[0..8] is its transpose,
            // the rotation that takes the reference y onto x
            bc[0] = q0 * q0 + q1 * q1 - q2 * q2 - q3 * q3; bc[1] = 2 * (q1 * q2 + q0 * q3); bc[2] = 2 * (q1 * q3 - q0 * q2);
            bc[3] = 2 * (q1 * q2 - q0 * q3); bc[4] = q0 * q0 - q1 * q1 + q2 * q2 - q3 * q3; bc[5] = 2 * (q2 * q3 + q0 * q1);
            bc[6] = 2 * (q1 * q3 + q0 * q2); bc[7] = 2 * (q2 * q3 - q0 * q1); bc[8] = q0 * q0 - q1 * q1 - q2 * q2 + q3 * q3;
            double msd = fmax(0.0, (c[9] - 2 * wm) / na);
            double rmsd = sqrt(msd);
            bc[9] = rmsd > 1e-10 ? 1.0 / (na * rmsd) : 0.0;
            cvv[it.cv] = rmsd;
        }
        __syncthreads();
        for (int j = it.s0 + tid; j < it.s1; j += nt) {
            F3 p = pos(j);
            double x[3] = {p.x - xc[0], p.y - xc[1], p.z - xc[2]};
            double y[3] = {G.ref[3 * j] - yc[0], G.ref[3 * j + 1] - yc[1], G.ref[3 * j + 2] - yc[2]};
            double g[3];
            for (int a = 0; a < 3; a++) g[a] = bc[9] * (x[a] - (bc[3 * a] * y[0] + bc[3 * a + 1] * y[1] + bc[3 * a + 2] * y[2]));
            int r = it.jac0 + j;
            J.gx[r] = (float)g[0]; J.gy[r] = (float)g[1]; J.gz[r] = (float)g[2];
        }
    }
    if constexpr (LATE) asm volatile("griddepcontrol.wait;" ::: "memory");
}

// setTestForce: mode 1 constant (scale,0,0); mode 2 (userAtom*scale,0,0);
// mode 3 PBC distance of user atoms 0,1 as force.x of slot 0.
__global__ void k_test_force(const float4* __restrict__ posq, const int* __restrict__ atomIndex,
                             unsigned long long* __restrict__ force, int padded, int numAtoms, int mode,
                             double scale, const BoxDev* __restrict__ boxp) {
    const double S = 4294967296.0;
    if (mode == 3) {
        if (blockIdx.x == 0 && threadIdx.x == 0 && numAtoms >= 2) {
            int g0 = atomIndex ? atomIndex[0] : 0, g1 = atomIndex ? atomIndex[1] : 1;
            float4 a = posq[g0], b = posq[g1];
            F3 d = minImage(f3(b.x - a.x, b.y - a.y, b.z - a.z), *boxp);
            float dist = sqrtf(dot3(d, d));
            atomicAdd(&force[0], (unsigned long long)(long long)((double)dist * S));
        }
        return;
    }
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < numAtoms; g += gridDim.x * blockDim.x) {
        double fx = mode == 1 ? scale : (double)(atomIndex ? atomIndex[g] : g) * scale;
        atomicAdd(&force[g], (unsigned long long)(long long)(fx * S));
    }
}

// ------------------------------------------------------------------ launchers
void launchInvertIndex(cudaStream_t s, const int* atomIndex, int* u2g, int n) {
    if (n > 0) k_invert_index<<<(n + 255) / 256, 256, 0, s>>>(atomIndex, u2g, n);
}

void launchComposeSimpleSlots(cudaStream_t s, SimpleItem* items, const int* u2g, int n) {
    if (n > 0) k_compose_simple_slots<<<(n + 127) / 128, 128, 0, s>>>(items, u2g, n);
}

void launchSimpleCVs(cudaStream_t s, const float4* posq, const int* u2g, const SimpleItem* items, int n,
                     const BoxDev* box, double* cvv, const JacDev& J, bool late) {
    if (n <= 0) return;
    if (late)
        launchPdl(k_simple_cvs<true>, dim3((n + 127) / 128), dim3(128), 0, s, posq, u2g, items, n, box, cvv, J);
    else
        launchPdl(k_simple_cvs<false>, dim3((n + 127) / 128), dim3(128), 0, s, posq, u2g, items, n, box, cvv, J);
}

// Cluster form of the slice-able group CVs (CommonGluedKernels.cpp:456-639,
// :796-881, :1633-1681). The atoms of the CV, [s0, s1) or [s0, s2) for a COM
// distance, are split into GROUP_CLUSTER contiguous slices, one per CTA of the
// cluster; a CTA gathers its slice into shared memory, sums it with the fixed
// block tree, and clusterSum adds the CTAs' sums in rank order through
// distributed shared memory. Each reduction has its own buffer, so one cluster
// barrier per reduction suffices; a last barrier keeps every CTA's buffers alive
// until the others have read them.
constexpr int GROUP_CLUSTER = 8;

namespace cg = cooperative_groups;

template <int NV>
__device__ __forceinline__ void clusterSum(double (&v)[NV], double* part, double* bcast) {
    cg::cluster_group cluster = cg::this_cluster();
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < NV; k++) part[k] = v[k];
    cluster.sync();
    if (threadIdx.x == 0) {
        double t[NV];
#pragma unroll
        for (int k = 0; k < NV; k++) t[k] = 0.0;
        for (int r = 0; r < GROUP_CLUSTER; r++) {
            const double* remote = cluster.map_shared_rank(part, r);
#pragma unroll
            for (int k = 0; k < NV; k++) t[k] += remote[k];
        }
#pragma unroll
        for (int k = 0; k < NV; k++) bcast[k] = t[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; k++) v[k] = bcast[k];
    __syncthreads();
}

__global__ void __cluster_dims__(GROUP_CLUSTER, 1, 1) __launch_bounds__(GROUP_THREADS)
    k_group_cvs_cluster(const float4* __restrict__ posq, const GroupDev G, const BoxDev* __restrict__ boxp,
                        double* __restrict__ cvv, JacDev J) {
    pdlEnter();
    extern __shared__ float4 sPos[];
    __shared__ double red[32 * 8];
    __shared__ double part[2][8];
    __shared__ double bcast[8];
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = (int)cluster.block_rank();
    const int gi = blockIdx.x / GROUP_CLUSTER;
    const GroupItem it = gi < G.nInl ? G.inl[gi] : G.items[gi];
    const BoxDev box = *boxp;
    const int tid = threadIdx.x, nt = blockDim.x;
    const int a0 = it.s0, a1 = it.type == CV_COM_DISTANCE ? it.s2 : it.s1;
    const int L = (a1 - a0 + GROUP_CLUSTER - 1) / GROUP_CLUSTER;
    const int b0 = min(a0 + rank * L, a1), b1 = min(b0 + L, a1);
    const bool cached = L <= GROUP_CACHE;
    const bool withMass = it.type == CV_COM_DISTANCE || it.type == CV_GYRATION;
    if (cached) {
        const int n = b1 - b0;
        for (int base = tid; base < n; base += nt * GATHER_U) {
            int slot[GATHER_U];
            float m[GATHER_U];
#pragma unroll
            for (int u = 0; u < GATHER_U; u++) {
                const int j = base + nt * u;
                slot[u] = j < n ? __ldg(G.slots + b0 + j) : -1;
                m[u] = (withMass && j < n) ? __ldg(G.mass + b0 + j) : 0.0f;
            }
#pragma unroll
            for (int u = 0; u < GATHER_U; u++)
                if (slot[u] >= 0) {
                    float4 p = __ldg(posq + slot[u]);
                    p.w = m[u];
                    sPos[base + nt * u] = p;
                }
        }
        __syncthreads();
    }
    auto pos = [&](int j) -> F3 {
        if (cached) { const float4 p = sPos[j - b0]; return f3(p.x, p.y, p.z); }
        return loadPos(posq, nullptr, G.slots[j]);
    };
    auto massAt = [&](int j) -> float { return cached ? sPos[j - b0].w : G.mass[j]; };
    const bool lead = rank == 0 && tid == 0;

    if (it.type == CV_COM_DISTANCE) {
        double v[6] = {0, 0, 0, 0, 0, 0};
        for (int j = b0 + tid; j < b1; j += nt) {
            F3 p = pos(j);
            double m = massAt(j);
            int o = j < it.s1 ? 0 : 3;
            v[o] += m * p.x; v[o + 1] += m * p.y; v[o + 2] += m * p.z;
        }
        blockSum<6>(v, red);
        clusterSum<6>(v, part[0], bcast);
        float i1 = 1.0f / it.f0, i2 = 1.0f / it.f1;
        F3 c1 = f3((float)v[0] * i1, (float)v[1] * i1, (float)v[2] * i1);
        F3 c2 = f3((float)v[3] * i2, (float)v[4] * i2, (float)v[5] * i2);
        F3 d = minImage(sub3(c2, c1), box);
        float dist = sqrtf(dot3(d, d));
        float inv = dist > 1e-10f ? 1.0f / dist : 0.0f;
        if (lead) cvv[it.cv] = (double)dist;
        for (int j = b0 + tid; j < b1; j += nt) {
            bool g1 = j < it.s1;
            float w = massAt(j) / (g1 ? it.f0 : it.f1);
            float sc = g1 ? -inv * w : inv * w;
            int r = it.jac0 + j;
            J.gx[r] = d.x * sc; J.gy[r] = d.y * sc; J.gz[r] = d.z * sc;
        }
    } else if (it.type == CV_GYRATION) {
        double v[3] = {0, 0, 0};
        for (int j = b0 + tid; j < b1; j += nt) {
            F3 p = pos(j);
            double m = massAt(j);
            v[0] += m * p.x; v[1] += m * p.y; v[2] += m * p.z;
        }
        blockSum<3>(v, red);
        clusterSum<3>(v, part[0], bcast);
        float iM = 1.0f / it.f0;
        F3 com = f3((float)v[0] * iM, (float)v[1] * iM, (float)v[2] * iM);
        double q[1] = {0};
        for (int j = b0 + tid; j < b1; j += nt) {
            F3 d = minImage(sub3(pos(j), com), box);
            q[0] += (double)massAt(j) * (double)dot3(d, d);
        }
        blockSum<1>(q, red);
        clusterSum<1>(q, part[1], bcast);
        float rg = (float)sqrt(q[0] / (double)it.f0);
        float irg = rg > 1e-10f ? 1.0f / rg : 0.0f;
        if (lead) cvv[it.cv] = (double)rg;
        for (int j = b0 + tid; j < b1; j += nt) {
            F3 d = minImage(sub3(pos(j), com), box);
            float w = massAt(j) / it.f0;
            int r = it.jac0 + j;
            J.gx[r] = w * d.x * irg; J.gy[r] = w * d.y * irg; J.gz[r] = w * d.z * irg;
        }
    } else if (it.type == CV_RMSD) {
        double q[1] = {0};
#pragma unroll 4
        for (int j = b0 + tid; j < b1; j += nt) {
            F3 p = pos(j);
            F3 d = f3(p.x - G.ref[3 * j], p.y - G.ref[3 * j + 1], p.z - G.ref[3 * j + 2]);
            q[0] += (double)dot3(d, d);
        }
        blockSum<1>(q, red);
        clusterSum<1>(q, part[0], bcast);
        int na = it.s1 - it.s0;
        float rmsd = (float)sqrt(q[0] / na);
        float sc = (rmsd > 1e-10f ? 1.0f / rmsd : 0.0f) / (float)na;
        if (lead) cvv[it.cv] = (double)rmsd;
#pragma unroll 4
        for (int j = b0 + tid; j < b1; j += nt) {
            F3 p = pos(j);
            int r = it.jac0 + j;
            J.gx[r] = (p.x - G.ref[3 * j]) * sc; J.gy[r] = (p.y - G.ref[3 * j + 1]) * sc;
            J.gz[r] = (p.z - G.ref[3 * j + 2]) * sc;
        }
    } else {  // CV_PCA
        double q[1] = {0};
#pragma unroll 4
        for (int j = b0 + tid; j < b1; j += nt) {
            F3 p = pos(j);
            float dx = p.x - G.ref[3 * j], dy = p.y - G.ref[3 * j + 1], dz = p.z - G.ref[3 * j + 2];
            q[0] += (double)(dx * G.ev[3 * j] + dy * G.ev[3 * j + 1] + dz * G.ev[3 * j + 2]);
        }
        blockSum<1>(q, red);
        clusterSum<1>(q, part[0], bcast);
        if (lead) cvv[it.cv] = q[0];
        for (int j = b0 + tid; j < b1; j += nt) {
            int r = it.jac0 + j;
            J.gx[r] = G.ev[3 * j]; J.gy[r] = G.ev[3 * j + 1]; J.gz[r] = G.ev[3 * j + 2];
        }
    }
    cluster.sync();
}

void launchGroupCVs(cudaStream_t s, const float4* posq, const int* u2g, const GroupDev& G, const BoxDev* box,
                    double* cvv, const JacDev& J, int maxCached, bool clustered, bool late) {
    if (G.numItems <= 0) return;
    if (clustered) {
        const int slice = (std::max(maxCached, 1) + GROUP_CLUSTER - 1) / GROUP_CLUSTER;
        const size_t smem = sizeof(float4) * (size_t)std::min(slice, GROUP_CACHE);
        static bool cattr = false;
        if (!cattr) {
            cudaCheck(cudaFuncSetAttribute((const void*)k_group_cvs_cluster,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)(sizeof(float4) * GROUP_CACHE)), "group CV shared memory");
            cattr = true;
        }
        launchPdl(k_group_cvs_cluster, dim3(G.numItems * GROUP_CLUSTER), dim3(GROUP_THREADS), smem, s, posq, G,
                  box, cvv, J);
        return;
    }
    const size_t smem = sizeof(float4) * (size_t)std::min(std::max(maxCached, 1), GROUP_CACHE);
    static bool attr = false;
    if (!attr) {
        for (const void* fn : {(const void*)k_group_cvs<false>, (const void*)k_group_cvs<true>})
            cudaCheck(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)(sizeof(float4) * GROUP_CACHE)), "group CV shared memory");
        attr = true;
    }
    if (late)
        launchPdl(k_group_cvs<true>, dim3(G.numItems), dim3(GROUP_THREADS), smem, s, posq, u2g, G, box, cvv, J);
    else
        launchPdl(k_group_cvs<false>, dim3(G.numItems), dim3(GROUP_THREADS), smem, s, posq, u2g, G, box, cvv, J);
}

void launchTestForce(cudaStream_t s, const float4* posq, const int* atomIndex, long long* force, int padded,
                     int numAtoms, int mode, double scale, const BoxDev* box) {
    int blocks = (numAtoms + 255) / 256;
    if (blocks < 1) blocks = 1;
    k_test_force<<<blocks, 256, 0, s>>>(posq, atomIndex, reinterpret_cast<unsigned long long*>(force), padded,
                                        numAtoms, mode, scale, box);
}

}  // namespace glued
