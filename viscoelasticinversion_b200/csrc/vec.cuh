// vec.cuh — 4-wide vector loads/stores and staggered-row helpers shared by
// the split kernels.  Rows are multiples of 16 bytes and 4-cell groups start
// on multiples of 4 elements, so every vector access is 16-byte aligned.
#pragma once

#include <cstdint>

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
// lane k (0..3, known only at run time) of a 4-cell group, without
// indexing the register array dynamically (which would move it to the stack)
template <typename T>
__device__ __forceinline__ T lane4(const Q4<T> &q, int k) {
  return k == 0 ? q.v[0] : k == 1 ? q.v[1] : k == 2 ? q.v[2] : q.v[3];
}
// q[k] += d as one rounded addition (never contracted with the product
// that formed d), so every kernel instantiation that inlines it adds a
// source term with the same bits
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }

// CPML memory and rate of one cell, with their roundings fixed (so the
// 4-cell and the cell-by-cell forms give the same bits): psi' = a d + b psi
// (the product b psi rounded, then one fused multiply-add), d' = d ik + psi'.
template <typename T>
__device__ __forceinline__ T cpml_mem(T b, T psi, T a, T d) {
  return fma_rn(a, d, mul_rn(b, psi));
}
template <typename T>
__device__ __forceinline__ T cpml_rate(T d, T ik, T p) {
  return fma_rn(d, ik, p);
}
template <typename T>
__device__ __forceinline__ void add_lane4(Q4<T> &q, int k, T d) {
#pragma unroll
  for (int i = 0; i < 4; ++i)
    if (i == k) q.v[i] = add_rn(q.v[i], d);
}
// ---- L2 eviction priority hints (createpolicy + .L2::cache_hint): lines
// re-read by the other pass of the step are kept (evict_last), lines that
// are read or written once per step go first (evict_first)
__device__ __forceinline__ uint64_t l2_keep() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t l2_stream() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ void sth4(float *p, const Q4<float> &q, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.v4.f32 [%0], {%1, %2, %3, %4}, %5;" ::"l"(p), "f"(q.v[0]), "f"(q.v[1]),
               "f"(q.v[2]), "f"(q.v[3]), "l"(pol)
               : "memory");
}
__device__ __forceinline__ void sth4(double *p, const Q4<double> &q, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.v2.f64 [%0], {%1, %2}, %3;" ::"l"(p), "d"(q.v[0]), "d"(q.v[1]), "l"(pol)
               : "memory");
  asm volatile("st.global.L2::cache_hint.v2.f64 [%0], {%1, %2}, %3;" ::"l"(p + 2), "d"(q.v[2]), "d"(q.v[3]), "l"(pol)
               : "memory");
}
__device__ __forceinline__ Q4<float> ldh4(const float *p, uint64_t pol) {
  Q4<float> q;
  asm volatile("ld.global.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
               : "=f"(q.v[0]), "=f"(q.v[1]), "=f"(q.v[2]), "=f"(q.v[3])
               : "l"(p), "l"(pol));
  return q;
}
__device__ __forceinline__ Q4<double> ldh4(const double *p, uint64_t pol) {
  Q4<double> q;
  asm volatile("ld.global.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;" : "=d"(q.v[0]), "=d"(q.v[1]) : "l"(p), "l"(pol));
  asm volatile("ld.global.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;" : "=d"(q.v[2]), "=d"(q.v[3]) : "l"(p + 2), "l"(pol));
  return q;
}
// State loaded before the PDL wait (written by the grid before the running
// one, which completed before this grid was released): read at L2, the
// coherence point, never from a line an earlier grid left in this SM's L1.
__device__ __forceinline__ Q4<float> ldcgh4(const float *p, uint64_t pol) {
  Q4<float> q;
  asm volatile("ld.global.cg.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
               : "=f"(q.v[0]), "=f"(q.v[1]), "=f"(q.v[2]), "=f"(q.v[3])
               : "l"(p), "l"(pol));
  return q;
}
__device__ __forceinline__ Q4<double> ldcgh4(const double *p, uint64_t pol) {
  Q4<double> q;
  asm volatile("ld.global.cg.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;" : "=d"(q.v[0]), "=d"(q.v[1]) : "l"(p), "l"(pol));
  asm volatile("ld.global.cg.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;" : "=d"(q.v[2]), "=d"(q.v[3]) : "l"(p + 2), "l"(pol));
  return q;
}
__device__ __forceinline__ Q4<float> ldcg4(const float *p) {
  const float4 q = __ldcg(reinterpret_cast<const float4 *>(p));
  return {{q.x, q.y, q.z, q.w}};
}
__device__ __forceinline__ Q4<double> ldcg4(const double *p) {
  const double2 a = __ldcg(reinterpret_cast<const double2 *>(p));
  const double2 b = __ldcg(reinterpret_cast<const double2 *>(p) + 1);
  return {{a.x, a.y, b.x, b.y}};
}
__device__ __forceinline__ Q4<float> ldgh4(const float *p, uint64_t pol) {  // read-only data
  Q4<float> q;
  asm volatile("ld.global.nc.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
               : "=f"(q.v[0]), "=f"(q.v[1]), "=f"(q.v[2]), "=f"(q.v[3])
               : "l"(p), "l"(pol));
  return q;
}
__device__ __forceinline__ Q4<double> ldgh4(const double *p, uint64_t pol) {
  Q4<double> q;
  asm volatile("ld.global.nc.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;" : "=d"(q.v[0]), "=d"(q.v[1]) : "l"(p), "l"(pol));
  asm volatile("ld.global.nc.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;" : "=d"(q.v[2]), "=d"(q.v[3]) : "l"(p + 2), "l"(pol));
  return q;
}
// Policies fixed per kernel instantiation (the hints pay when the kept
// set — the new v and sigma — fits in half the L2; beyond that kept lines
// thrash each other): with ON false both are evict_normal, so the accesses
// behave as plain ones.
__device__ __forceinline__ uint64_t l2_normal() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_normal.b64 %0, 1.0;" : "=l"(p));
  return p;
}
template <bool ON>
__device__ __forceinline__ uint64_t l2_keep_c() {
  return ON ? l2_keep() : l2_normal();
}
template <bool ON>
__device__ __forceinline__ uint64_t l2_stream_c() {
  return ON ? l2_stream() : l2_normal();
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
template <typename T>
__device__ __forceinline__ void add_lane2(Q2<T> &q, int k, T d) {
  if (k == 0)
    q.v[0] += d;
  else
    q.v[1] += d;
}
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

// ---- arithmetic on a 4-cell group.  FP32 pairs of cells use the packed
// FP32x2 instructions of sm_100 (each lane rounds as the scalar operation
// does); FP64 stays scalar.
__device__ __forceinline__ float2 lo2(const Q4<float> &a) { return make_float2(a.v[0], a.v[1]); }
__device__ __forceinline__ float2 hi2(const Q4<float> &a) { return make_float2(a.v[2], a.v[3]); }
__device__ __forceinline__ Q4<float> join2(float2 l, float2 h) { return {{l.x, l.y, h.x, h.y}}; }
template <typename T>
__device__ __forceinline__ Q4<T> splat4(T s) {
  return {{s, s, s, s}};
}
// a * b + c
__device__ __forceinline__ Q4<float> fma4(const Q4<float> &a, const Q4<float> &b, const Q4<float> &c) {
  return join2(__ffma2_rn(lo2(a), lo2(b), lo2(c)), __ffma2_rn(hi2(a), hi2(b), hi2(c)));
}
__device__ __forceinline__ Q4<double> fma4(const Q4<double> &a, const Q4<double> &b, const Q4<double> &c) {
  return {{fma(a.v[0], b.v[0], c.v[0]), fma(a.v[1], b.v[1], c.v[1]), fma(a.v[2], b.v[2], c.v[2]),
           fma(a.v[3], b.v[3], c.v[3])}};
}
__device__ __forceinline__ Q4<float> mul4(const Q4<float> &a, const Q4<float> &b) {
  return join2(__fmul2_rn(lo2(a), lo2(b)), __fmul2_rn(hi2(a), hi2(b)));
}
__device__ __forceinline__ Q4<double> mul4(const Q4<double> &a, const Q4<double> &b) {
  return {{a.v[0] * b.v[0], a.v[1] * b.v[1], a.v[2] * b.v[2], a.v[3] * b.v[3]}};
}
__device__ __forceinline__ Q4<float> add4(const Q4<float> &a, const Q4<float> &b) {
  return join2(__fadd2_rn(lo2(a), lo2(b)), __fadd2_rn(hi2(a), hi2(b)));
}
__device__ __forceinline__ Q4<double> add4(const Q4<double> &a, const Q4<double> &b) {
  return {{a.v[0] + b.v[0], a.v[1] + b.v[1], a.v[2] + b.v[2], a.v[3] + b.v[3]}};
}
template <typename T>
__device__ __forceinline__ Q4<T> sub4(const Q4<T> &a, const Q4<T> &b) {  // a - b, exact as one rounding
  return fma4(b, splat4<T>(T(-1)), a);
}
// ---- compensated accumulation of a 4-cell group (FP32 with a bfloat16
// residue per cell).  A float sigma updated 4000 times loses the low bits
// of every increment, and the part of that rounding noise that has no
// divergence never radiates away: it stays in sigma as a static field.
// Carrying each cell's rounding error in a residue plane and folding it
// into the next increment removes that drift.  hi + lo += d: x = d + lo,
// s = hi + x exactly split into s and its error e by Knuth's two-sum
// (six round-to-nearest additions, valid whatever the magnitudes), then
// hi = s and lo = e rounded to bfloat16 (8 more bits than the float).
__device__ __forceinline__ Q4<float> bf16x4_to_f32(uint2 u) {
  return {{__uint_as_float(u.x << 16), __uint_as_float(u.x & 0xffff0000u), __uint_as_float(u.y << 16),
           __uint_as_float(u.y & 0xffff0000u)}};
}
__device__ __forceinline__ uint32_t f32x2_to_bf16x2(float lo, float hi) {  // round to nearest even
  uint32_t d;
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(hi), "f"(lo));
  return d;
}
__device__ __forceinline__ uint2 f32_to_bf16x4(const Q4<float> &q) {
  return make_uint2(f32x2_to_bf16x2(q.v[0], q.v[1]), f32x2_to_bf16x2(q.v[2], q.v[3]));
}
__device__ __forceinline__ void two_sum_acc4(Q4<float> &hi, uint2 &lo, const Q4<float> &d) {
  const Q4<float> x = add4(d, bf16x4_to_f32(lo));
  const Q4<float> s = add4(hi, x);
  const Q4<float> bp = sub4(s, hi);
  const Q4<float> e = add4(sub4(hi, sub4(s, bp)), sub4(x, bp));
  hi = s;
  lo = f32_to_bf16x4(e);
}
__device__ __forceinline__ uint2 ldh_u2(const uint16_t *p, uint64_t pol) {
  uint2 q;
  asm volatile("ld.global.L2::cache_hint.v2.u32 {%0, %1}, [%2], %3;" : "=r"(q.x), "=r"(q.y) : "l"(p), "l"(pol));
  return q;
}
__device__ __forceinline__ void sth_u2(uint16_t *p, uint2 q, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.v2.u32 [%0], {%1, %2}, %3;" ::"l"(p), "r"(q.x), "r"(q.y), "l"(pol)
               : "memory");
}
// true when the 12 values of three groups are finite (a NaN or an
// infinity anywhere makes their sum non-finite; so does an overflowing sum,
// which is an unstable run as well)
template <typename T>
__device__ __forceinline__ bool finite3(const Q4<T> &a, const Q4<T> &b, const Q4<T> &c) {
  const Q4<T> s = add4(add4(a, b), c);
  return isfinite((s.v[0] + s.v[1]) + (s.v[2] + s.v[3]));
}
// window of 4 consecutive values of a 12-value row, starting at o
template <typename T>
__device__ __forceinline__ Q4<T> win4(const T (&u)[12], int o) {
  return {{u[o], u[o + 1], u[o + 2], u[o + 3]}};
}
// the ddxp / ddxm sums of dps / dms for the group's four cells (c = 4..7)
template <typename T>
__device__ __forceinline__ Q4<T> dps4(const T (&u)[12], const T *D) {
  Q4<T> acc = mul4(splat4<T>(D[0]), sub4(win4(u, 5), win4(u, 4)));
#pragma unroll
  for (int q = 1; q < 4; ++q) acc = fma4(splat4<T>(D[q]), sub4(win4(u, 5 + q), win4(u, 4 - q)), acc);
  return acc;
}
template <typename T>
__device__ __forceinline__ Q4<T> dms4(const T (&u)[12], const T *D) {
  Q4<T> acc = mul4(splat4<T>(D[0]), sub4(win4(u, 4), win4(u, 3)));
#pragma unroll
  for (int q = 1; q < 4; ++q) acc = fma4(splat4<T>(D[q]), sub4(win4(u, 4 + q), win4(u, 3 - q)), acc);
  return acc;
}

}  // namespace vb
