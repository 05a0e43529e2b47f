// Kernel launches with programmatic dependent launch (PDL).
//
// Every kernel of the hot path calls grid_dep_wait() (griddepcontrol.wait: returns once
// the preceding kernel in stream order has completed and its writes are visible) before
// it reads anything, and grid_dep_launch() (griddepcontrol.launch_dependents) once the
// next kernel's blocks may be scheduled: the short per-stage kernels trigger at their
// start, the long tile kernel only before its last pass, so waiting blocks of the next
// kernel do not sit beside it while it still works.  The ordering is that of a plain
// stream launch; inside a captured graph the dependency becomes a programmatic edge.
// FFB_PDL=0 in the environment launches without the attribute (the device instructions
// are then no-ops).
#pragma once

#include <cuda_runtime.h>

namespace ffb {

bool pdl_enabled();

__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void grid_dep_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <typename... KArgs, typename... Args>
inline cudaError_t launch_k(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                            Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl_enabled() ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

}  // namespace ffb
