// vec.cuh — 4-wide vector loads/stores and staggered-row helpers shared by
// the split kernels.  Rows are multiples of 16 bytes and 4-cell groups start
// on multiples of 4 elements, so every vector access is 16-byte aligned.
#pragma once

#include <cuda_runtime.h>

namespace vb {

template <typename T>
struct Q4 {
  T v[4];
};

// shared memory
__device__ __forceinline__ Q4<float> lds4(const float *p) {
  const float4 q = *reinterpret_cast<const float4 *>(p);
  return {{q.x, q.y, q.z, q.w}};
}
__device__ __forceinline__ Q4<double> lds4(const double *p) {
  const double2 a = reinterpret_cast<const double2 *>(p)[0];
  const double2 b = reinterpret_cast<const double2 *>(p)[1];
  return {{a.x, a.y, b.x, b.y}};
}
// read-only global (non-coherent path)
__device__ __forceinline__ Q4<float> ldg4(const float *p) {
  const float4 q = __ldg(reinterpret_cast<const float4 *>(p));
  return {{q.x, q.y, q.z, q.w}};
}
__device__ __forceinline__ Q4<double> ldg4(const double *p) {
  const double2 a = __ldg(reinterpret_cast<const double2 *>(p));
  const double2 b = __ldg(reinterpret_cast<const double2 *>(p) + 1);
  return {{a.x, a.y, b.x, b.y}};
}
// coherent global loads of state the same kernel writes (own cells only)
__device__ __forceinline__ Q4<float> ldc4(const float *p) {
  const float4 q = *reinterpret_cast<const float4 *>(p);
  return {{q.x, q.y, q.z, q.w}};
}
__device__ __forceinline__ Q4<double> ldc4(const double *p) {
  const double2 a = reinterpret_cast<const double2 *>(p)[0];
  const double2 b = reinterpret_cast<const double2 *>(p)[1];
  return {{a.x, a.y, b.x, b.y}};
}
__device__ __forceinline__ void stg4(float *p, const Q4<float> &q) {
  *reinterpret_cast<float4 *>(p) = make_float4(q.v[0], q.v[1], q.v[2], q.v[3]);
}
__device__ __forceinline__ void stg4(double *p, const Q4<double> &q) {
  reinterpret_cast<double2 *>(p)[0] = make_double2(q.v[0], q.v[1]);
  reinterpret_cast<double2 *>(p)[1] = make_double2(q.v[2], q.v[3]);
}
// 2/s: correctly rounded reciprocal in FP32, division in FP64
__device__ __forceinline__ float two_over_s(float s) { return 2.0f * __frcp_rn(s); }
__device__ __forceinline__ double two_over_s(double s) { return 2.0 / s; }
// 2/s with the hardware approximate reciprocal (FP32, relative error of a
// few ulp, far inside the 1e-5 trace tolerance); FP64 divides
__device__ __forceinline__ float two_over_fast(float s) { return __fdividef(2.0f, s); }
__device__ __forceinline__ double two_over_fast(double s) { return 2.0 / s; }

// 2-wide forms (8-byte aligned for FP32, 16-byte for FP64)
template <typename T>
struct Q2 {
  T v[2];
};
__device__ __forceinline__ Q2<float> lds2(const float *p) {
  const float2 q = *reinterpret_cast<const float2 *>(p);
  return {{q.x, q.y}};
}
__device__ __forceinline__ Q2<double> lds2(const double *p) {
  const double2 q = *reinterpret_cast<const double2 *>(p);
  return {{q.x, q.y}};
}
__device__ __forceinline__ void stg2(float *p, const Q2<float> &q) {
  *reinterpret_cast<float2 *>(p) = make_float2(q.v[0], q.v[1]);
}
__device__ __forceinline__ void stg2(double *p, const Q2<double> &q) {
  *reinterpret_cast<double2 *>(p) = make_double2(q.v[0], q.v[1]);
}

// 12 consecutive values of a staged row starting at a 4-aligned column
template <typename T>
__device__ __forceinline__ void row12s(const T *p, T (&o)[12]) {
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const Q4<T> v = lds4(p + 4 * q);
#pragma unroll
    for (int k = 0; k < 4; ++k) o[4 * q + k] = v.v[k];
  }
}
// staggered sums over a row held in registers (c: the cell's index)
template <typename T>
__device__ __forceinline__ T dps(const T (&u)[12], int c, const T *D) {  // ddxp form
  return D[0] * (u[c + 1] - u[c]) + D[1] * (u[c + 2] - u[c - 1]) + D[2] * (u[c + 3] - u[c - 2]) +
         D[3] * (u[c + 4] - u[c - 3]);
}
template <typename T>
__device__ __forceinline__ T dms(const T (&u)[12], int c, const T *D) {  // ddxm form
  return D[0] * (u[c] - u[c - 1]) + D[1] * (u[c + 1] - u[c - 2]) + D[2] * (u[c + 2] - u[c - 3]) +
         D[3] * (u[c + 3] - u[c - 4]);
}

}  // namespace vb
