// Programmatic dependent launches for the per-context kernel chain.
//
// Every kernel of a force evaluation (simple CVs, group CVs, coordination runs
// and finalize, kernel sums, biases, scatter) is launched as a programmatic
// dependent of the launch before it: the next kernel's CTAs may be scheduled
// once every CTA of the current kernel has started, and each kernel waits in
// hardware (griddepcontrol.wait) for the previous grid to complete, with its
// memory writes visible, before it reads anything. The wait is transitive
// (a grid completes only after its own wait returned), so a kernel may read the
// output of any earlier launch; it returns at once for a plain launch. What it
// saves is the launch and drain gap between two small dependent kernels.
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
