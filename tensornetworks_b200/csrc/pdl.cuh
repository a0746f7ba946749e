// pdl.cuh -- programmatic dependent launch for chains of small dependent kernels.
//
// A kernel launched with launch_pdl() may be scheduled while its predecessor on
// the stream is still draining; it must call pdl_wait() before it reads
// anything the predecessor writes (or writes anything the predecessor reads).
// pdl_wait() returns once the predecessor grid has completed and its memory
// is visible; in a kernel launched the ordinary way it returns at once.  Each
// kernel in the chain waits before its own work, so the ordering is transitive.
// Captured into a CUDA graph, the launch becomes a programmatic edge.
#pragma once
#include <cuda_runtime.h>

#include "tn_internal.h"

namespace tnb {

__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Lets the next kernel on the stream (launched with launch_pdl) be scheduled
// once every CTA of this grid has passed here (or exited); it still waits in its
// own pdl_wait() for this grid's completion and memory flush, so calling this
// early only overlaps the next kernel's launch and prologue with this one.
__device__ __forceinline__ void pdl_launch_dependents() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

template <class... KArgs, class... Args>
int launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    TN_CUDA_CHECK(cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...));
    count_launch();
    return TN_OK;
}

}  // namespace tnb
