// afda.cuh — the H-AFDA free surface (vi_config.free_surface == 2) inside
// the 4-cell step kernels: the z derivatives of the four rows below the
// surface whose 8th-order staggered stencils would reach above it, taken
// from the one-sided weights StepArgs::af (built on the host, capi.cu).
#pragma once

#include "common.cuh"
#include "vec.cuh"

namespace vb {

// sum_m af[OP][q][m] * sample(m) for the 4 cells of a group at the
// run-time surface distance q.  The table is read with a run-time row
// index, so the StepArgs it comes from must live in the parameter bank as
// a __grid_constant__ kernel parameter (or in global memory): a by-value
// copy indexed this way would move to the stack.
template <int OP, typename T, typename F>
__device__ __forceinline__ Q4<T> afda4(const StepArgs<T> &a, int q, F sample) {
  const T *w = &a.af[OP][q][0];
  Q4<T> acc = splat4<T>(T(0));
#pragma unroll
  for (int m = 0; m < kAfdaN; ++m) acc = fma4(splat4<T>(w[m]), sample(m), acc);
  return acc;
}

}  // namespace vb
