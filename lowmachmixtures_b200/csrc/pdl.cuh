// pdl.cuh - programmatic dependent launch.
//
// A kernel launched with launch_pdl may be scheduled while the kernel before
// it on the stream drains; its first statement, pdl_enter(), waits for that
// kernel's completion and memory (griddepcontrol.wait) before any access,
// then lets the next kernel be scheduled (griddepcontrol.launch_dependents).
// Launched without the attribute, both instructions are no-ops.  Every
// kernel launched through launch_pdl starts with pdl_enter().
#pragma once
#include <cuda_runtime.h>

namespace lmm {

__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
template <class... KArgs, class... Args>
static inline void launch_pdl(void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, k, args...);
}

}  // namespace lmm
