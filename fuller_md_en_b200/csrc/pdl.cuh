// pdl.cuh -- programmatic dependent launch for the kernels of one step.
//
// A kernel launched with launch_pdl may start (its blocks get scheduled and
// run their prologue) while the previous kernel in the stream is still
// draining; FMD_PDL_WAIT() at the top of every such kernel blocks until the
// previous kernel's memory operations are complete and visible, so the
// overlap only hides launch latency.  Captured into a CUDA graph, the
// dependency becomes a programmatic edge.  Without the launch attribute the
// wait is a no-op.
#pragma once
#include <cuda_runtime.h>

#include <utility>

#define FMD_PDL_WAIT() asm volatile("griddepcontrol.wait;" ::: "memory")

namespace fmd {

template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                       Args&&... args) {
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
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

}  // namespace fmd
