// Programmatic dependent launches for the per-context kernel chain.
//
// Every kernel of a force evaluation (simple CVs, group CVs, coordination runs
// and finalize, kernel sums, biases, scatter) is launched as a programmatic
// dependent of the launch before it: the next kernel's CTAs may be scheduled
// once every CTA of the current kernel has executed
// griddepcontrol.launch_dependents (pdlEnter issues it right after the wait),
// and each kernel waits in hardware (griddepcontrol.wait) for the previous grid
// to complete, with its memory writes visible, before it reads anything a
// kernel of the step writes. The wait is transitive (a grid completes only after
// its own wait returned), so a kernel may read the output of any earlier launch;
// it returns at once for a plain launch. Every kernel of the chain starts after
// the chain's first kernel, or the plain-launched coordination grid, has passed
// its wait, so what was enqueued before the force evaluation (plan and bias
// records, tables written by the deposits, the caller's inputs) is complete by
// then and may be loaded before a kernel's own wait. What this saves is the
// launch and drain gap between two small dependent kernels, and the latency of
// those early loads.
#pragma once

#include <cuda_runtime.h>

#include "context.hpp"

namespace glued {

// First statement of every kernel launched with launchPdl.
__device__ __forceinline__ void pdlEnter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

template <typename... KArgs, typename... Args>
inline void launchPdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaCheck(cudaLaunchKernelEx(&cfg, kernel, args...), "launch");
}

}  // namespace glued
