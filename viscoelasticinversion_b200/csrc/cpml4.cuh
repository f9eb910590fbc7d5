// cpml4.cuh — CPML memory updates of one 4-cell group of the split kernels.
//
// Each update covers two derivatives d0, d1 of the group (cells gi0 ..
// gi0 + 3 of row gj): psi_n' = a_n d_n + b_n psi_n, d_n' = d_n / kappa +
// psi_n', with the profile rows (b, a, 1/kappa) of derivative n in the
// plan's tables and its memory in psi plane Pn.  psi is read from `in` and,
// when `store`, written to `out` (the same set in place, the other set for
// the ping-pong forms).  A group whose four cells lie in one x strip with
// 16-byte aligned memory runs as 4-wide loads and stores; any other group
// cell by cell; both round the same way (cpml_mem / cpml_rate), so the
// results do not depend on the form.
#pragma once

#include "common.cuh"
#include "vec.cuh"

namespace vb {

struct CpmlRows {
  int p;        // psi plane of the derivative
  int b, a, k;  // table rows of b, a and 1/kappa
};

template <typename T>
__device__ __forceinline__ void cpml_x4(const StepArgs<T> &args, int gi0, int gj, CpmlRows r0, CpmlRows r1,
                                        const T *in, T *out, bool store, Q4<T> &d0, Q4<T> &d1) {
  const int nx = args.nx;
  const T *tb = args.tx;
  const long long pl = args.psix_plane;
  const int xs0 = strip_x(gi0, nx, args.Lx, args.Rx);
  const long long o0 = (long long)gj * args.wx + xs0;
  if (xs0 >= 0 && strip_x(gi0 + 3, nx, args.Lx, args.Rx) == xs0 + 3 && ((o0 | pl) & 3) == 0) {
    const Q4<T> q0 = ldc4(in + r0.p * pl + o0), q1 = ldc4(in + r1.p * pl + o0);
    const Q4<T> B0 = ldg4(tb + r0.b * nx + gi0), A0 = ldg4(tb + r0.a * nx + gi0), K0 = ldg4(tb + r0.k * nx + gi0);
    const Q4<T> B1 = ldg4(tb + r1.b * nx + gi0), A1 = ldg4(tb + r1.a * nx + gi0), K1 = ldg4(tb + r1.k * nx + gi0);
    Q4<T> p0, p1;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      p0.v[k] = cpml_mem(B0.v[k], q0.v[k], A0.v[k], d0.v[k]);
      p1.v[k] = cpml_mem(B1.v[k], q1.v[k], A1.v[k], d1.v[k]);
      d0.v[k] = cpml_rate(d0.v[k], K0.v[k], p0.v[k]);
      d1.v[k] = cpml_rate(d1.v[k], K1.v[k], p1.v[k]);
    }
    if (store) {
      stg4(out + r0.p * pl + o0, p0);
      stg4(out + r1.p * pl + o0, p1);
    }
    return;
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int gi = gi0 + k;
    const int xs = strip_x(gi, nx, args.Lx, args.Rx);
    if (xs >= 0) {
      const long long o = (long long)gj * args.wx + xs;
      const T p0 = cpml_mem(tb[r0.b * nx + gi], in[r0.p * pl + o], tb[r0.a * nx + gi], d0.v[k]);
      const T p1 = cpml_mem(tb[r1.b * nx + gi], in[r1.p * pl + o], tb[r1.a * nx + gi], d1.v[k]);
      if (store) {
        out[r0.p * pl + o] = p0;
        out[r1.p * pl + o] = p1;
      }
      d0.v[k] = cpml_rate(d0.v[k], tb[r0.k * nx + gi], p0);
      d1.v[k] = cpml_rate(d1.v[k], tb[r1.k * nx + gi], p1);
    }
  }
}

// z strips: zs is the row's index in the strip storage (strip_z >= 0); the
// profile is one value per row for the whole group.
template <typename T>
__device__ __forceinline__ void cpml_z4(const StepArgs<T> &args, int zs, int gi0, int gj, CpmlRows r0, CpmlRows r1,
                                        const T *in, T *out, bool store, Q4<T> &d0, Q4<T> &d1) {
  const int nx = args.nx, nz = args.nz;
  const T *tb = args.tz;
  const long long pl = args.psiz_plane;
  const long long o = (long long)zs * nx + gi0;
  const T B0 = tb[r0.b * nz + gj], A0 = tb[r0.a * nz + gj], K0 = tb[r0.k * nz + gj];
  const T B1 = tb[r1.b * nz + gj], A1 = tb[r1.a * nz + gj], K1 = tb[r1.k * nz + gj];
  Q4<T> q0, q1, p0, p1;
  const bool vec = ((o | pl) & 3) == 0;
  if (vec) {
    q0 = ldc4(in + r0.p * pl + o);
    q1 = ldc4(in + r1.p * pl + o);
  } else {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      q0.v[k] = in[r0.p * pl + o + k];
      q1.v[k] = in[r1.p * pl + o + k];
    }
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    p0.v[k] = cpml_mem(B0, q0.v[k], A0, d0.v[k]);
    p1.v[k] = cpml_mem(B1, q1.v[k], A1, d1.v[k]);
    d0.v[k] = cpml_rate(d0.v[k], K0, p0.v[k]);
    d1.v[k] = cpml_rate(d1.v[k], K1, p1.v[k]);
  }
  if (!store) return;
  if (vec) {
    stg4(out + r0.p * pl + o, p0);
    stg4(out + r1.p * pl + o, p1);
  } else {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      out[r0.p * pl + o + k] = p0.v[k];
      out[r1.p * pl + o + k] = p1.v[k];
    }
  }
}

}  // namespace vb
