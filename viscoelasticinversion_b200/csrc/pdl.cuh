// pdl.cuh — programmatic dependent launch (PDL) between the kernels of one
// time loop.  A kernel launched with launch_pdl may be launched while the
// previous kernel in the stream is still finishing; pdl_wait() blocks until
// that grid has completed and its memory operations are visible.  Without
// an explicit pdl_release() the next grid is released as this grid's CTAs
// exit.
#pragma once

#include <cuda_runtime.h>

#include <utility>

namespace vb {

__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_release() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Launches kernel<<<grid, block, smem, st>>>(args...); with pdl set, the
// launch may overlap the tail of the previous kernel in the stream.
template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                       cudaStream_t st, bool pdl, Args &&...args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

}  // namespace vb
