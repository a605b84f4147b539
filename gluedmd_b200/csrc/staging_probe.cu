// Hill-slice staging probe: the staging step of the batched hill evaluation
// (every CTA of a persistent grid copies its equal slice of the three float
// arrays x', y', h of the hill table into shared memory) timed alone, with the
// 16-byte cp.async copies the runs kernel uses and with one bulk copy per array
// (cp.async.bulk global -> shared of this GPU's own memory, completion counted
// on an mbarrier; no cluster, no multicast). Each timed launch follows an L2
// flush, as every batched step does. Used to decide which form the runs kernel
// uses; returns the mean microseconds per launch of each form.
#include <cuda_runtime.h>

#include "context.hpp"
#include "kernels.hpp"

namespace glued {

namespace {

constexpr int PROBE_HS = 512;       // hills staged per CTA at most (as the runs kernel)
constexpr int PROBE_THREADS = 512;
constexpr long long WAIT_LIMIT = 1ll << 24;

__device__ __forceinline__ unsigned sAddr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

}  // namespace

// mirror: [3][cap] floats (cap a multiple of 4, 16-byte aligned arrays); the
// CTA's slice is hill groups [g0, g1) of (count + 3) / 4. out[b] = a sum of the
// staged heights (keeps the copies observable); status bit 0: an mbarrier wait
// gave up (the kernel then stops waiting and exits without using the data).
template <bool BULK>
__global__ void __launch_bounds__(PROBE_THREADS) k_stage_probe(const float* __restrict__ mirror, int cap, int count,
                                                               float* __restrict__ out, int* __restrict__ status) {
    __shared__ __align__(128) float sh[3][PROBE_HS];
    __shared__ __align__(8) unsigned long long mbar;
    const int tid = threadIdx.x;
    const int groups = (count + 3) / 4;
    const int g0 = (int)((long long)groups * blockIdx.x / gridDim.x);
    const int g1 = min((int)((long long)groups * (blockIdx.x + 1) / gridDim.x), g0 + PROBE_HS / 4);
    const int n = g1 - g0;   // groups of 4 hills
    if (BULK) {
        if (tid == 0) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sAddr(&mbar)) : "memory");
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        __syncthreads();
        if (tid == 0) {
            const unsigned bytes = 16u * (unsigned)n;
            unsigned long long state;
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 %0, [%1], %2;"
                         : "=l"(state) : "r"(sAddr(&mbar)), "r"(3u * bytes) : "memory");
            (void)state;
            if (bytes > 0)
                for (int a = 0; a < 3; a++)
                    asm volatile(
                        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                            sAddr(&sh[a][0])),
                        "l"(mirror + (size_t)a * cap + 4 * (size_t)g0), "r"(bytes), "r"(sAddr(&mbar))
                        : "memory");
        }
        unsigned done = 0;
        for (long long it = 0; it < WAIT_LIMIT && !done; it++)
            asm volatile("{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0; selp.u32 %0, 1, 0, p; }"
                         : "=r"(done) : "r"(sAddr(&mbar)) : "memory");
        if (!done) {
            if (tid == 0) atomicOr(status, 1);
            return;
        }
    } else {
        for (int t = tid; t < 3 * n; t += PROBE_THREADS) {
            const int a = t / n, g = t - a * n;
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sAddr(&sh[a][4 * g])),
                         "l"(mirror + (size_t)a * cap + 4 * (size_t)(g0 + g))
                         : "memory");
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
        asm volatile("cp.async.wait_group 0;" ::: "memory");
    }
    __syncthreads();
    float s = 0.0f;
    for (int k = tid; k < 4 * n; k += PROBE_THREADS) s += sh[2][k] + sh[0][k] * sh[1][k];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((tid & 31) == 0) atomicAdd(out + blockIdx.x, s);
}

void measureHillStaging(int numHills, int ctas, int reps, double* usCpAsync, double* usBulk, int* status) {
    if (numHills < 1 || ctas < 1 || reps < 1) throw Error(GLUED_E_INVALID, "staging probe: sizes must be >= 1");
    const int cap = (numHills + 3) / 4 * 4;
    if ((long long)cap > (long long)PROBE_HS * ctas)
        throw Error(GLUED_E_INVALID, "staging probe: more than 512 hills per CTA");
    DBuf mirror, out, st, flush;
    mirror.alloc(sizeof(float) * 3 * (size_t)cap);
    std::vector<float> h(3 * (size_t)cap);
    for (size_t i = 0; i < h.size(); i++) h[i] = (float)((i * 2654435761u) % 1000u) * 1e-3f;
    cudaCheck(cudaMemcpy(mirror.p, h.data(), sizeof(float) * h.size(), cudaMemcpyHostToDevice), "probe");
    out.alloc(sizeof(float) * ctas);
    st.alloc(sizeof(int));
    flush.alloc((size_t)192 << 20);
    cudaEvent_t e0, e1;
    cudaCheck(cudaEventCreate(&e0), "event");
    cudaCheck(cudaEventCreate(&e1), "event");
    double tot[2] = {0, 0};
    for (int r = 0; r < reps + 1; r++)
        for (int v = 0; v < 2; v++) {
            cudaCheck(cudaMemsetAsync(flush.p, r & 0xff, flush.bytes), "flush");
            cudaCheck(cudaEventRecord(e0), "event");
            if (v == 0)
                k_stage_probe<false><<<ctas, PROBE_THREADS>>>(mirror.as<float>(), cap, numHills, out.as<float>(),
                                                              st.as<int>());
            else
                k_stage_probe<true><<<ctas, PROBE_THREADS>>>(mirror.as<float>(), cap, numHills, out.as<float>(),
                                                             st.as<int>());
            cudaCheck(cudaEventRecord(e1), "event");
            cudaCheck(cudaEventSynchronize(e1), "event");
            float ms = 0;
            cudaCheck(cudaEventElapsedTime(&ms, e0, e1), "event");
            if (r > 0) tot[v] += ms * 1e3;   // the first round warms the code
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaCheck(cudaMemcpy(status, st.p, sizeof(int), cudaMemcpyDeviceToHost), "probe");
    *usCpAsync = tot[0] / reps;
    *usBulk = tot[1] / reps;
}

}  // namespace glued
