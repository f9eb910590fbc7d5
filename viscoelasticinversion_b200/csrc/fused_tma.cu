// fused_tma.cu — the fused step with every operand of a tile staged in
// shared memory by TMA (cp.async.bulk.tensor) before any arithmetic.
//
// One elected thread issues all boxes of a tile (stresses + 8-cell halo,
// velocities + 4-cell halo, density, memory variables, stiffness, τ) on one
// mbarrier; the CTA then computes the velocity stage on the tile + halo and
// the SLS stress stage on the tile entirely from shared memory.  Only the
// CPML ψ strips, the per-tile source/receiver lists and the outputs touch
// global memory during compute.  With two stages the kernel is persistent:
// one CTA per SM walks the tiles round-robin and the boxes of its next tile
// load while the current tile computes.
#include <atomic>
#include <cudaTypedefs.h>

#include "fused_tma.cuh"
#include "plan.cuh"
#include "tma.cuh"

namespace vb {

__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Issues every TMA box of `tile` into stage buffer `sb` on barrier `bar`.
template <typename G, typename T>
__device__ __forceinline__ void issue_tile(T *sb, uint64_t *bar, const TmaMaps &maps, int x0,
                                           int z0) {
  constexpr int HVP = G::HVP, HSP = G::HSP, HV = G::HV, HS = G::HS;
  mbar_arrive_expect_tx(bar, G::TX_BYTES);
  tma_load_2d(sb + G::S_SXX, &maps.sxx, x0 - HSP, z0 - HS, bar);
  tma_load_2d(sb + G::S_SZZ, &maps.szz, x0 - HSP, z0 - HS, bar);
  tma_load_2d(sb + G::S_SXZ, &maps.sxz, x0 - HSP, z0 - HS, bar);
  tma_load_2d(sb + G::S_VX, &maps.vx, x0 - HVP, z0 - HV, bar);
  tma_load_2d(sb + G::S_VZ, &maps.vz, x0 - HVP, z0 - HV, bar);
  tma_load_2d(sb + G::S_RHO, &maps.rho, x0 - HVP, z0 - HV, bar);
  if constexpr (G::NM > 0) {
    tma_load_3d(sb + G::S_M, &maps.m, x0 + G::MX0, z0 + G::MZ0, 0, bar);
    if constexpr (G::TTI)
      tma_load_2d(sb + G::S_TAU, &maps.tau, x0 + G::MX0, z0 + G::MZ0, bar);
    else
      tma_load_2d(sb + G::S_TAU, &maps.tau, x0, z0, bar);
  }
#pragma unroll
  for (int c = 0; c < G::NC; ++c) tma_load_2d(sb + G::S_C + c * G::PC, &maps.c[c], x0, z0, bar);
}

// ---- 4-wide vectors of reals in shared and global memory (16-byte
// aligned: rows are multiples of 16 bytes and groups start on multiples
// of 4 elements) ----
template <typename T>
struct V4 {
  T v[4];
};
__device__ __forceinline__ V4<float> ld4(const float *p) {
  const float4 q = *reinterpret_cast<const float4 *>(p);
  return {{q.x, q.y, q.z, q.w}};
}
__device__ __forceinline__ V4<double> ld4(const double *p) {
  const double2 a = reinterpret_cast<const double2 *>(p)[0];
  const double2 b = reinterpret_cast<const double2 *>(p)[1];
  return {{a.x, a.y, b.x, b.y}};
}
__device__ __forceinline__ void st4(float *p, const V4<float> &q) {
  *reinterpret_cast<float4 *>(p) = make_float4(q.v[0], q.v[1], q.v[2], q.v[3]);
}
__device__ __forceinline__ void st4(double *p, const V4<double> &q) {
  reinterpret_cast<double2 *>(p)[0] = make_double2(q.v[0], q.v[1]);
  reinterpret_cast<double2 *>(p)[1] = make_double2(q.v[2], q.v[3]);
}
// 2/(a+b): correctly rounded reciprocal in FP32, division in FP64
__device__ __forceinline__ float two_over(float s) { return 2.0f * __frcp_rn(s); }
__device__ __forceinline__ double two_over(double s) { return 2.0 / s; }

// 12 consecutive values of a staged row starting at a 4-aligned column
template <typename T>
__device__ __forceinline__ void row12(const T *p, T (&o)[12]) {
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const V4<T> v = ld4(p + 4 * q);
#pragma unroll
    for (int k = 0; k < 4; ++k) o[4 * q + k] = v.v[k];
  }
}

// W-wide vectors (W = 2 or 4) for the stress stage
template <typename T, int W>
struct VW {
  T v[W];
};
// adds d to lane k (known only at run time) without indexing the register
// array dynamically (which would move it to the stack)
template <typename T, int W>
__device__ __forceinline__ void add_lanew(VW<T, W> &q, int k, T d) {
#pragma unroll
  for (int i = 0; i < W; ++i)
    if (i == k) q.v[i] += d;
}
template <typename T, int W>
__device__ __forceinline__ VW<T, W> ldw(const T *p) {
  VW<T, W> o;
  if constexpr (W == 4) {
    const V4<T> q = ld4(p);
#pragma unroll
    for (int k = 0; k < 4; ++k) o.v[k] = q.v[k];
  } else if constexpr (sizeof(T) == 4) {
    const float2 q = *reinterpret_cast<const float2 *>(p);
    o.v[0] = q.x;
    o.v[1] = q.y;
  } else {
    const double2 q = *reinterpret_cast<const double2 *>(p);
    o.v[0] = q.x;
    o.v[1] = q.y;
  }
  return o;
}
template <typename T, int W>
__device__ __forceinline__ void stw(T *p, const VW<T, W> &q) {
  if constexpr (W == 4) {
    st4(p, V4<T>{{q.v[0], q.v[1], q.v[2], q.v[3]}});
  } else if constexpr (sizeof(T) == 4) {
    *reinterpret_cast<float2 *>(p) = make_float2(q.v[0], q.v[1]);
  } else {
    *reinterpret_cast<double2 *>(p) = make_double2(q.v[0], q.v[1]);
  }
}
// W + 8 consecutive values of a staged row starting at a W-aligned column
template <typename T, int W>
__device__ __forceinline__ void roww(const T *p, T (&o)[W + 8]) {
#pragma unroll
  for (int q = 0; q < (W + 8) / W; ++q) {
    const VW<T, W> v = ldw<T, W>(p + W * q);
#pragma unroll
    for (int k = 0; k < W; ++k) o[W * q + k] = v.v[k];
  }
}
// staggered sums over a row held in registers; c is the cell's index
template <typename T, int N>
__device__ __forceinline__ T dpx(const T (&u)[N], int c, const T *D) {  // ddxp form
  return D[0] * (u[c + 1] - u[c]) + D[1] * (u[c + 2] - u[c - 1]) + D[2] * (u[c + 3] - u[c - 2]) +
         D[3] * (u[c + 4] - u[c - 3]);
}
template <typename T, int N>
__device__ __forceinline__ T dmx(const T (&u)[N], int c, const T *D) {  // ddxm form
  return D[0] * (u[c] - u[c - 1]) + D[1] * (u[c + 1] - u[c - 2]) + D[2] * (u[c + 2] - u[c - 3]) +
         D[3] * (u[c + 3] - u[c - 4]);
}

// Pointers and bounds of the tile being computed.
template <typename T>
struct TileCtx {
  T *s_sxx, *s_szz, *s_sxz, *s_vx, *s_vz, *s_rho, *s_m, *s_c, *s_tau, *s_exx, *s_ezz, *s_exz;
  int x0, z0, nx, nz, xe, ze, e0, e1;
};

// CPML-corrected rates of W cells whose first cell sits at velocity-box
// column vc (a multiple of W) and row vr, global (gi0.., gj); writes the
// psi output set when `own`.
template <typename G, typename T, int W>
__device__ __forceinline__ void rates_w(const StepArgs<T> &a, const TileCtx<T> &t, int vr, int vc,
                                        int gi0, int gj, bool own, T (&rxx)[W], T (&rzz)[W],
                                        T (&rxz)[W]) {
  constexpr int VWp = G::VWp;
  T hvx[W + 8], hvz[W + 8];
  roww<T, W>(t.s_vx + vr * VWp + vc - 4, hvx);
  roww<T, W>(t.s_vz + vr * VWp + vc - 4, hvz);
  // ddzm(vz) over rows -4..+3, ddzp(vx) over rows -3..+4, accumulated
  T zvz[W], zvx[W];
#pragma unroll
  for (int k = 0; k < W; ++k) zvz[k] = zvx[k] = T(0);
#pragma unroll
  for (int q = -4; q <= 4; ++q) {
    if (q <= 3) {
      const T cq = q >= 0 ? a.Dz[q] : -a.Dz[-q - 1];
      VW<T, W> v;
      if (q == 0) {
#pragma unroll
        for (int k = 0; k < W; ++k) v.v[k] = hvz[4 + k];
      } else {
        v = ldw<T, W>(t.s_vz + (vr + q) * VWp + vc);
      }
#pragma unroll
      for (int k = 0; k < W; ++k) zvz[k] += cq * v.v[k];
    }
    if (q >= -3) {
      const T cq = q >= 1 ? a.Dz[q - 1] : -a.Dz[-q];
      VW<T, W> v;
      if (q == 0) {
#pragma unroll
        for (int k = 0; k < W; ++k) v.v[k] = hvx[4 + k];
      } else {
        v = ldw<T, W>(t.s_vx + (vr + q) * VWp + vc);
      }
#pragma unroll
      for (int k = 0; k < W; ++k) zvx[k] += cq * v.v[k];
    }
  }
  const int nx = t.nx, nz = t.nz;
  const int zs = strip_z(gj, nz, a.Tz, a.Bz);
#pragma unroll
  for (int k = 0; k < W; ++k) {
    const int gi = gi0 + k;
    T dxvx = dmx(hvx, 4 + k, a.Dx);
    T dxvz = dpx(hvz, 4 + k, a.Dx);
    T dzvz = zvz[k], dzvx = zvx[k];
    const int xs = strip_x(gi, nx, a.Lx, a.Rx);
    if (xs >= 0) {
      const T *tb = a.tx;
      const long long o = (long long)gj * a.wx + xs;
      const T p0 = tb[T_B * nx + gi] * a.psix[PX_VX * a.psix_plane + o] + tb[T_A * nx + gi] * dxvx;
      const T p1 = tb[T_BH * nx + gi] * a.psix[PX_VZ * a.psix_plane + o] + tb[T_AH * nx + gi] * dxvz;
      if (own) {
        a.psix_o[PX_VX * a.psix_plane + o] = p0;
        a.psix_o[PX_VZ * a.psix_plane + o] = p1;
      }
      dxvx = dxvx * tb[T_IK * nx + gi] + p0;
      dxvz = dxvz * tb[T_IKH * nx + gi] + p1;
    }
    if (zs >= 0) {
      const T *tb = a.tz;
      const long long o = (long long)zs * nx + gi;
      const T p0 = tb[T_B * nz + gj] * a.psiz[PZ_VZ * a.psiz_plane + o] + tb[T_A * nz + gj] * dzvz;
      const T p1 = tb[T_BH * nz + gj] * a.psiz[PZ_VX * a.psiz_plane + o] + tb[T_AH * nz + gj] * dzvx;
      if (own) {
        a.psiz_o[PZ_VZ * a.psiz_plane + o] = p0;
        a.psiz_o[PZ_VX * a.psiz_plane + o] = p1;
      }
      dzvz = dzvz * tb[T_IK * nz + gj] + p0;
      dzvx = dzvx * tb[T_IKH * nz + gj] + p1;
    }
    rxx[k] = dxvx;
    rzz[k] = dzvz;
    rxz[k] = dzvx + dxvz;
  }
}

// effective SLS rates of W cells from the staged M (M-box index mi, a
// multiple of W) and tau
template <typename G, typename T, int NSLS, int W>
__device__ __forceinline__ void effective_w(const TileCtx<T> &t, int mi, const VW<T, W> &tau,
                                            const T (&rxx)[W], const T (&rzz)[W],
                                            const T (&rxz)[W], T (&exx)[W], T (&ezz)[W],
                                            T (&exz)[W]) {
  if constexpr (NSLS > 0) {
    constexpr int MP = G::MW * G::MH;
    T Sxx[W], Szz[W], Sxz[W];
#pragma unroll
    for (int k = 0; k < W; ++k) Sxx[k] = Szz[k] = Sxz[k] = T(0);
#pragma unroll
    for (int n = 0; n < NSLS; ++n) {
      const VW<T, W> mx = ldw<T, W>(t.s_m + (0 * NSLS + n) * MP + mi);
      const VW<T, W> mz = ldw<T, W>(t.s_m + (1 * NSLS + n) * MP + mi);
      const VW<T, W> mq = ldw<T, W>(t.s_m + (2 * NSLS + n) * MP + mi);
#pragma unroll
      for (int k = 0; k < W; ++k) {
        Sxx[k] += mx.v[k];
        Szz[k] += mz.v[k];
        Sxz[k] += mq.v[k];
      }
    }
#pragma unroll
    for (int k = 0; k < W; ++k) {
      const T tk = tau.v[k], t1 = T(1) + tk;
      exx[k] = t1 * rxx[k] + tk * Sxx[k];
      ezz[k] = t1 * rzz[k] + tk * Szz[k];
      exz[k] = t1 * rxz[k] + tk * Sxz[k];
    }
  } else {
#pragma unroll
    for (int k = 0; k < W; ++k) {
      exx[k] = rxx[k];
      ezz[k] = rzz[k];
      exz[k] = rxz[k];
    }
  }
}

// The velocity and stress stages of one staged tile.  The velocity stage
// works on groups of 4 x-adjacent cells of one row, the stress stage on
// groups of SWID cells: one vector load per staged row covers the x-taps
// of the group and each z-tap row is one vector.
template <typename G, typename T, int KIND, int NSLS>
__device__ __forceinline__ void compute_tile(const StepArgs<T> &a, const FusedExtras<T> &x,
                                             T *sb, T *s_e, int tile, int e0, int e1) {
  constexpr int TX = G::TX, TZ = G::TZ, NT = G::NT, HV = G::HV, HS = G::HS, HVP = G::HVP,
                HSP = G::HSP, SWp = G::SWp, VWp = G::VWp, VH = G::VH, RWp = G::RWp, MW = G::MW,
                CW = G::CW, EW = G::EW, EH = G::EH, PC = G::PC;
  constexpr int W = G::SWID;
  constexpr bool TTI = G::TTI;
  static_assert(HSP == HVP + 4, "sigma box must extend the velocity box by 4 columns");
  TileCtx<T> t;
  t.s_sxx = sb + G::S_SXX;
  t.s_szz = sb + G::S_SZZ;
  t.s_sxz = sb + G::S_SXZ;
  t.s_vx = sb + G::S_VX;
  t.s_vz = sb + G::S_VZ;
  t.s_rho = sb + G::S_RHO;
  t.s_m = sb + G::S_M;
  t.s_c = sb + G::S_C;
  t.s_tau = sb + G::S_TAU;
  t.s_exx = s_e;
  t.s_ezz = s_e + G::PE;
  t.s_exz = s_e + 2 * G::PE;
  constexpr int C11 = 0;
  constexpr int C13 = KIND == VI_MEDIUM_ISO ? 0 : 1;
  constexpr int C15 = 2;
  constexpr int C33 = KIND == VI_MEDIUM_VTI ? 2 : 3;
  constexpr int C35 = 4;
  constexpr int C55 = KIND == VI_MEDIUM_ISO ? 1 : (KIND == VI_MEDIUM_VTI ? 3 : 5);

  const int x0 = L + (tile % x.ntx) * TX;
  const int z0 = L + (tile / x.ntx) * TZ;
  const int nx = a.nx, nz = a.nz;
  const int xe = nx - L, ze = nz - L;
  t.x0 = x0;
  t.z0 = z0;
  t.nx = nx;
  t.nz = nz;
  t.xe = xe;
  t.ze = ze;
  t.e0 = e0;
  t.e1 = e1;
  const int tid = threadIdx.x;
  const T dt = a.dt;
  T *s_sxx = t.s_sxx, *s_szz = t.s_szz, *s_sxz = t.s_sxz, *s_vx = t.s_vx, *s_vz = t.s_vz;
  T *s_rho = t.s_rho, *s_m = t.s_m, *s_c = t.s_c, *s_tau = t.s_tau;
  T *s_exx = t.s_exx, *s_ezz = t.s_ezz, *s_exz = t.s_exz;

  // ---- 1. new velocities on the whole velocity box ----------------------
  constexpr int VG = VWp / 4;  // groups per row
  for (int item = tid; item < VG * VH; item += NT) {
    const int r = item / VG, lxv = 4 * (item - r * VG);
    const int gi0 = x0 - HVP + lxv, gj = z0 - HV + r;
    const int vb = r * VWp + lxv;
    V4<T> vxn = {{0, 0, 0, 0}}, vzn = {{0, 0, 0, 0}};
    if (gi0 >= L && gi0 < xe && gj >= L && gj < ze) {
      const int sbase = (r + HS - HV) * SWp + lxv;  // sigma row of the cells, 4-aligned start
      T hxx[12], hxz[12];
      row12(s_sxx + sbase, hxx);
      row12(s_sxz + sbase, hxz);
      // z derivatives of the 4 cells, accumulated row by row:
      // ddzm(sxz) over rows -4..+3, ddzp(szz) over rows -3..+4
      T zxz[4] = {0, 0, 0, 0}, zzz[4] = {0, 0, 0, 0};
#pragma unroll
      for (int q = -4; q <= 4; ++q) {
        if (q <= 3) {
          const T cq = q >= 0 ? a.Dz[q] : -a.Dz[-q - 1];
          const V4<T> v = q == 0 ? V4<T>{{hxz[4], hxz[5], hxz[6], hxz[7]}}
                                 : ld4(s_sxz + sbase + q * SWp + 4);
#pragma unroll
          for (int k = 0; k < 4; ++k) zxz[k] += cq * v.v[k];
        }
        if (q >= -3) {
          const T cq = q >= 1 ? a.Dz[q - 1] : -a.Dz[-q];
          const V4<T> v = ld4(s_szz + sbase + q * SWp + 4);
#pragma unroll
          for (int k = 0; k < 4; ++k) zzz[k] += cq * v.v[k];
        }
      }
      const V4<T> r0 = ld4(s_rho + r * RWp + lxv);
      const T r4 = s_rho[r * RWp + lxv + 4];
      const V4<T> r1 = ld4(s_rho + (r + 1) * RWp + lxv);
      const V4<T> vxi = ld4(s_vx + vb), vzi = ld4(s_vz + vb);
      const bool own_row = gj >= z0 && gj < z0 + TZ;
      const int zs = strip_z(gj, nz, a.Tz, a.Bz);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int gi = gi0 + k;
        T dxx = dpx(hxx, 4 + k, a.Dx);
        T dxxz = dmx(hxz, 4 + k, a.Dx);
        T dzxz = zxz[k];
        T dzz = zzz[k];
        const bool own = own_row && gi >= x0 && gi < x0 + TX;
        const int xs = strip_x(gi, nx, a.Lx, a.Rx);
        if (xs >= 0) {
          const T *tb = a.tx;
          const long long o = (long long)gj * a.wx + xs;
          const T p0 = tb[T_BH * nx + gi] * a.psix[PX_SXX * a.psix_plane + o] + tb[T_AH * nx + gi] * dxx;
          const T p1 = tb[T_B * nx + gi] * a.psix[PX_SXZ * a.psix_plane + o] + tb[T_A * nx + gi] * dxxz;
          if (own) {
            a.psix_o[PX_SXX * a.psix_plane + o] = p0;
            a.psix_o[PX_SXZ * a.psix_plane + o] = p1;
          }
          dxx = dxx * tb[T_IKH * nx + gi] + p0;
          dxxz = dxxz * tb[T_IK * nx + gi] + p1;
        }
        if (zs >= 0) {
          const T *tb = a.tz;
          const long long o = (long long)zs * nx + gi;
          const T p0 = tb[T_B * nz + gj] * a.psiz[PZ_SXZ * a.psiz_plane + o] + tb[T_A * nz + gj] * dzxz;
          const T p1 = tb[T_BH * nz + gj] * a.psiz[PZ_SZZ * a.psiz_plane + o] + tb[T_AH * nz + gj] * dzz;
          if (own) {
            a.psiz_o[PZ_SXZ * a.psiz_plane + o] = p0;
            a.psiz_o[PZ_SZZ * a.psiz_plane + o] = p1;
          }
          dzxz = dzxz * tb[T_IK * nz + gj] + p0;
          dzz = dzz * tb[T_IKH * nz + gj] + p1;
        }
        const T rx = k < 3 ? r0.v[k + 1] : r4;
        vxn.v[k] = vxi.v[k] + dt * two_over(r0.v[k] + rx) * (dxx + dzxz);
        vzn.v[k] = vzi.v[k] + dt * two_over(r0.v[k] + r1.v[k]) * (dxxz + dzz);
      }
    }
    st4(s_vx + vb, vxn);
    st4(s_vz + vb, vzn);
  }
  __syncthreads();

  if (e1 > e0) {
    // force sources (one thread: entries are few and may share a cell)
    if (tid == 0) {
      for (int e = e0; e < e1; ++e) {
        const int4 en = x.tile_ent[e];
        if (en.w != TL_FORCE_X && en.w != TL_FORCE_Z) continue;
        const int lx = en.x - (x0 - HVP), lz = en.y - (z0 - HV);
        const int sv = lz * VWp + lx;
        const int ri = lz * RWp + lx;
        const T w = x.it < x.wnt ? x.wavelet[(long long)en.z * x.wnt + x.it] : T(0);
        const T f = x.amp[en.z] * w;
        if (en.w == TL_FORCE_X)
          s_vx[sv] += dt * two_over(s_rho[ri] + s_rho[ri + 1]) * f;
        else
          s_vz[sv] += dt * two_over(s_rho[ri] + s_rho[ri + RWp]) * f;
      }
    }
    __syncthreads();
  }

  // ---- 2. write the tile's velocities; receivers sample them -------------
  constexpr int TG = TX / 4;  // 4-groups per tile row
  for (int item = tid; item < TG * TZ; item += NT) {
    const int r = item / TG, lx = 4 * (item - r * TG);
    const int gi0 = x0 + lx, gj = z0 + r;
    if (gi0 < xe && gj < ze) {
      const long long g = (long long)gj * nx + gi0;
      const int sv = (r + HV) * VWp + lx + HVP;
      st4(a.vx_o + g, ld4(s_vx + sv));
      st4(a.vz_o + g, ld4(s_vz + sv));
    }
  }
  if (x.traces && x.it < x.tnt) {
    for (int e = e0 + tid; e < e1; e += NT) {
      const int4 en = x.tile_ent[e];
      if (en.w != TL_RECEIVER) continue;
      const int sv = (en.y - z0 + HV) * VWp + en.x - x0 + HVP;
      x.traces[(long long)en.z * x.tnt + x.it] = s_vx[sv];
      x.traces[(long long)(x.nrec + en.z) * x.tnt + x.it] = s_vz[sv];
    }
  }

  // ---- 3. TTI: effective rates on the tile + ring, 4-aligned columns ----
  if constexpr (TTI) {
    // e box: origin (x0 - 4, z0 - 1), EW = TX + 8 columns, EH = TZ + 2 rows
    constexpr int EG = EW / 4;
    for (int item = tid; item < EG * EH; item += NT) {
      const int er = item / EG, ec = 4 * (item - er * EG);
      const int gi0 = x0 - 4 + ec, gj = z0 - 1 + er;
      T exx[4] = {0, 0, 0, 0}, ezz[4] = {0, 0, 0, 0}, exz[4] = {0, 0, 0, 0};
      if (gi0 >= L && gi0 < xe && gj >= L && gj < ze) {
        T rxx[4], rzz[4], rxz[4];
        rates_w<G, T, 4>(a, t, er - 1 + HV, ec + HVP - 4, gi0, gj, false, rxx, rzz, rxz);
        const int mi = er * MW + ec;  // M / tau ring box has the e-box origin
        VW<T, 4> tv;
        if constexpr (NSLS > 0) tv = ldw<T, 4>(s_tau + mi);
        effective_w<G, T, NSLS, 4>(t, mi, tv, rxx, rzz, rxz, exx, ezz, exz);
      }
      const int eb = er * EW + ec;
      st4(s_exx + eb, V4<T>{{exx[0], exx[1], exx[2], exx[3]}});
      st4(s_ezz + eb, V4<T>{{ezz[0], ezz[1], ezz[2], ezz[3]}});
      st4(s_exz + eb, V4<T>{{exz[0], exz[1], exz[2], exz[3]}});
    }
    __syncthreads();
    if (x.fs && z0 == L) {
      // tau_zz = 0 on the surface row (e row 1) for columns x0 .. x0+TX
      for (int lx = tid; lx <= TX; lx += NT) {
        const int gi = x0 + lx;
        if (gi >= xe) continue;
        const int e = EW + lx + 4;
        const T eb = T(0.25) * (s_exz[e] + s_exz[e - 1] + s_exz[e - EW] + s_exz[e - EW - 1]);
        s_ezz[e] = -(s_c[C13 * PC + lx] * s_exx[e] + s_c[C35 * PC + lx] * eb) / s_c[C33 * PC + lx];
      }
      __syncthreads();
    }
  }

  // ---- 4. stresses and memory variables on the tile, W-wide groups ------
  constexpr int SG = TX / W;  // W-groups per tile row
#pragma unroll 1
  for (int item = tid; item < SG * TZ; item += NT) {
    const int r = item / SG, lx = W * (item - r * SG);
    const int gi0 = x0 + lx, gj = z0 + r;
    if (gi0 >= xe || gj >= ze) continue;
    const long long g = (long long)gj * nx + gi0;
    const int ci = r * CW + lx;
    const int mi = TTI ? (r + 1) * MW + lx + 4 : r * MW + lx;
    T rxx[W], rzz[W], rxz[W], exx[W], ezz[W], exz[W];
    rates_w<G, T, W>(a, t, r + HV, lx + HVP, gi0, gj, true, rxx, rzz, rxz);
    const bool surf = x.fs && gj == L;
    const T *c55p = s_c + C55 * PC;
    const VW<T, W> c13 = ldw<T, W>(s_c + C13 * PC + ci);
    const VW<T, W> c55a = ldw<T, W>(c55p + ci), c55b = ldw<T, W>(c55p + ci + CW);
    const T c55aW = c55p[ci + W], c55bW = c55p[ci + CW + W];
    T dsxx[W], dszz[W], dsxz[W];
    if constexpr (TTI) {
      const int e = (r + 1) * EW + lx + 4;
      const T *c15p = s_c + C15 * PC, *c35p = s_c + C35 * PC;
      const VW<T, W> c11 = ldw<T, W>(s_c + C11 * PC + ci), c33 = ldw<T, W>(s_c + C33 * PC + ci);
      const VW<T, W> c15a = ldw<T, W>(c15p + ci), c15b = ldw<T, W>(c15p + ci + CW);
      const VW<T, W> c35a = ldw<T, W>(c35p + ci), c35b = ldw<T, W>(c35p + ci + CW);
      const T c15aW = c15p[ci + W], c15bW = c15p[ci + CW + W];
      const T c35aW = c35p[ci + W], c35bW = c35p[ci + CW + W];
      const VW<T, W> xx0 = ldw<T, W>(s_exx + e), xx1 = ldw<T, W>(s_exx + e + EW);
      const VW<T, W> zz0 = ldw<T, W>(s_ezz + e), zz1 = ldw<T, W>(s_ezz + e + EW);
      const VW<T, W> xz0 = ldw<T, W>(s_exz + e), xzm = ldw<T, W>(s_exz + e - EW);
      const T xx0W = s_exx[e + W], xx1W = s_exx[e + EW + W];
      const T zz0W = s_ezz[e + W], zz1W = s_ezz[e + EW + W];
      const T xz0m = s_exz[e - 1], xzmm = s_exz[e - EW - 1];
#pragma unroll
      for (int k = 0; k < W; ++k) {
        exx[k] = xx0.v[k];
        ezz[k] = zz0.v[k];
        exz[k] = xz0.v[k];
        const T xzl = k > 0 ? xz0.v[k - 1] : xz0m, xzml = k > 0 ? xzm.v[k - 1] : xzmm;
        const T ebxz = T(0.25) * (xz0.v[k] + xzl + xzm.v[k] + xzml);
        const T xxr = k < W - 1 ? xx0.v[k + 1] : xx0W, xx1r = k < W - 1 ? xx1.v[k + 1] : xx1W;
        const T zzr = k < W - 1 ? zz0.v[k + 1] : zz0W, zz1r = k < W - 1 ? zz1.v[k + 1] : zz1W;
        const T ebxx = T(0.25) * (xx0.v[k] + xxr + xx1.v[k] + xx1r);
        const T ebzz = T(0.25) * (zz0.v[k] + zzr + zz1.v[k] + zz1r);
        const T c55r = k < W - 1 ? c55a.v[k + 1] : c55aW, c55br = k < W - 1 ? c55b.v[k + 1] : c55bW;
        const T c15r = k < W - 1 ? c15a.v[k + 1] : c15aW, c15br = k < W - 1 ? c15b.v[k + 1] : c15bW;
        const T c35r = k < W - 1 ? c35a.v[k + 1] : c35aW, c35br = k < W - 1 ? c35b.v[k + 1] : c35bW;
        const T C55h = T(0.25) * (c55a.v[k] + c55r + c55b.v[k] + c55br);
        const T C15h = T(0.25) * (c15a.v[k] + c15r + c15b.v[k] + c15br);
        const T C35h = T(0.25) * (c35a.v[k] + c35r + c35b.v[k] + c35br);
        dsxx[k] = c11.v[k] * exx[k] + c13.v[k] * ezz[k] + c15a.v[k] * ebxz;
        dszz[k] = c13.v[k] * exx[k] + c33.v[k] * ezz[k] + c35a.v[k] * ebxz;
        dsxz[k] = C55h * exz[k] + C15h * ebxx + C35h * ebzz;
      }
    } else {
      VW<T, W> tv;
      if constexpr (NSLS > 0) tv = ldw<T, W>(s_tau + ci);
      effective_w<G, T, NSLS, W>(t, mi, tv, rxx, rzz, rxz, exx, ezz, exz);
      VW<T, W> c11, c33;
      if constexpr (KIND == VI_MEDIUM_ISO) {
#pragma unroll
        for (int k = 0; k < W; ++k) c11.v[k] = c33.v[k] = c13.v[k] + T(2) * c55a.v[k];
      } else {
        c11 = ldw<T, W>(s_c + C11 * PC + ci);
        c33 = ldw<T, W>(s_c + C33 * PC + ci);
      }
#pragma unroll
      for (int k = 0; k < W; ++k) {
        if (surf) ezz[k] = -(c13.v[k] * exx[k]) / c33.v[k];
        const T c55r = k < W - 1 ? c55a.v[k + 1] : c55aW, c55br = k < W - 1 ? c55b.v[k + 1] : c55bW;
        const T C55h = T(0.25) * (c55a.v[k] + c55r + c55b.v[k] + c55br);
        dsxx[k] = c11.v[k] * exx[k] + c13.v[k] * ezz[k];
        dszz[k] = c13.v[k] * exx[k] + c33.v[k] * ezz[k];
        dsxz[k] = C55h * exz[k];
      }
    }
    const int si = (r + HS) * SWp + lx + HSP;
    VW<T, W> sxx = ldw<T, W>(s_sxx + si), szz = ldw<T, W>(s_szz + si), sxz = ldw<T, W>(s_sxz + si);
#pragma unroll
    for (int k = 0; k < W; ++k) {
      sxx.v[k] += dt * dsxx[k];
      szz.v[k] += dt * dszz[k];
      sxz.v[k] += dt * dsxz[k];
    }
    if constexpr (NSLS > 0) {
      constexpr int MP = G::MW * G::MH;
#pragma unroll
      for (int n = 0; n < NSLS; ++n) {
        const T a1 = a.a1[n], a2 = a.a2[n];
        VW<T, W> mx = ldw<T, W>(s_m + (0 * NSLS + n) * MP + mi);
        VW<T, W> mz = ldw<T, W>(s_m + (1 * NSLS + n) * MP + mi);
        VW<T, W> mq = ldw<T, W>(s_m + (2 * NSLS + n) * MP + mi);
#pragma unroll
        for (int k = 0; k < W; ++k) {
          mx.v[k] = mx.v[k] + dt * (a1 * rxx[k] + a2 * mx.v[k]);
          mz.v[k] = surf ? T(0) : mz.v[k] + dt * (a1 * rzz[k] + a2 * mz.v[k]);
          mq.v[k] = mq.v[k] + dt * (a1 * rxz[k] + a2 * mq.v[k]);
        }
        stw<T, W>(a.m_o + (0 * NSLS + n) * a.mstride_o + g, mx);
        stw<T, W>(a.m_o + (1 * NSLS + n) * a.mstride_o + g, mz);
        stw<T, W>(a.m_o + (2 * NSLS + n) * a.mstride_o + g, mq);
      }
    }
    for (int e = e0; e < e1; ++e) {
      const int4 en = x.tile_ent[e];
      if (en.w != TL_EXPLOSIVE || en.y != gj || en.x < gi0 || en.x >= gi0 + W) continue;
      const T w = x.it < x.wnt ? x.wavelet[(long long)en.z * x.wnt + x.it] : T(0);
      add_lanew(sxx, en.x - gi0, dt * x.amp[en.z] * w);
      add_lanew(szz, en.x - gi0, dt * x.amp[en.z] * w);
    }
    if (surf) {
#pragma unroll
      for (int k = 0; k < W; ++k) szz.v[k] = T(0);
    }
    stw<T, W>(a.sxx_o + g, sxx);
    stw<T, W>(a.szz_o + g, szz);
    stw<T, W>(a.sxz_o + g, sxz);
    stw<T, W>(s_sxx + si, sxx);
    stw<T, W>(s_szz + si, szz);
    stw<T, W>(s_sxz + si, sxz);
  }

  // ---- 5. stress images above the free surface --------------------------
  if (x.fs && z0 == L) {
    __syncthreads();
    for (int lx = tid; lx < TX; lx += NT) {
      const int gi = x0 + lx;
      if (gi >= xe) continue;
#pragma unroll
      for (int k = 1; k <= L; ++k)
        a.szz_o[(long long)(L - k) * nx + gi] = -s_szz[(HS + k) * SWp + lx + HSP];
#pragma unroll
      for (int k = 0; k < L; ++k)
        a.sxz_o[(long long)(L - 1 - k) * nx + gi] = -s_sxz[(HS + k) * SWp + lx + HSP];
    }
  }
}

template <typename T, int KIND, int NSLS, bool PERSIST>
__global__ void __launch_bounds__(TmaPick<T, KIND, NSLS, PERSIST>::Lay::NT)
    k_fused_tma(const StepArgs<T> a, const FusedExtras<T> x, const __grid_constant__ TmaMaps maps,
                int ntiles) {
  using G = typename TmaPick<T, KIND, NSLS, PERSIST>::Lay;
  constexpr int ST = G::STAGES;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw);
  T *sm = reinterpret_cast<T *>(smem_raw);
  T *stage0 = sm + G::O_STAGE;
  T *s_e = sm + G::O_E;
  const int tid = threadIdx.x;
  const int G0 = gridDim.x;
  auto origin = [&](int tile, int &x0, int &z0) {
    x0 = L + (tile % x.ntx) * G::TX;
    z0 = L + (tile / x.ntx) * G::TZ;
  };

  if (tid == 0) {
    for (int s = 0; s < ST; ++s) mbar_init(&bars[s], 1);
  }
  __syncthreads();
  if (tid == 0) {
    for (int s = 0; s < ST; ++s) {
      const int t = blockIdx.x + s * G0;
      if (t < ntiles) {
        int x0, z0;
        origin(t, x0, z0);
        issue_tile<G, T>(stage0 + s * G::STAGE, &bars[s], maps, x0, z0);
      }
    }
  }
  int j = 0;
  for (int tile = blockIdx.x; tile < ntiles; tile += G0, ++j) {
    const int s = ST == 2 ? (j & 1) : 0;
    const uint32_t parity = ST == 2 ? ((j >> 1) & 1) : (j & 1);
    const int e0 = x.tile_off[tile], e1 = x.tile_off[tile + 1];  // loaded ahead of the wait
    const bool ok = mbar_wait_bounded(&bars[s], parity, 1u << 22);
    if (__syncthreads_or(!ok)) {
      // staging never completed: report, let the copies in flight land
      // (bounded), and stop
      if (tid == 0) {
        atomicExch(x.err, 1);
        mbar_wait_bounded(&bars[s], parity, 1u << 22);
        if (ST == 2 && tile + G0 < ntiles) mbar_wait_bounded(&bars[s ^ 1], ((j + 1) >> 1) & 1, 1u << 22);
      }
      return;
    }
    T *sb = stage0 + s * G::STAGE;
    compute_tile<G, T, KIND, NSLS>(a, x, sb, s_e, tile, e0, e1);
    __syncthreads();  // every thread is done with this stage
    if (tid == 0) {
      const int nt2 = tile + ST * G0;
      if (nt2 < ntiles) {
        fence_proxy_async_smem();  // generic writes to the stage before the async overwrite
        int x0, z0;
        origin(nt2, x0, z0);
        issue_tile<G, T>(sb, &bars[s], maps, x0, z0);
      }
    }
  }
}

// Many shots advancing one time step together: the launch covers the tiles
// of every active shot (shots sorted by step count, so the active ones are
// a prefix), each item reads its shot's arguments and tensor maps from
// device memory.  Same staging, pipeline and arithmetic as k_fused_tma.
template <typename T, int KIND, int NSLS, bool PERSIST>
__global__ void __launch_bounds__(TmaPick<T, KIND, NSLS, PERSIST>::Lay::NT)
    k_fused_tma_batch(const BatchDev<T> b, int it, int nitems) {
  using G = typename TmaPick<T, KIND, NSLS, PERSIST>::Lay;
  constexpr int ST = G::STAGES;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw);
  T *sm = reinterpret_cast<T *>(smem_raw);
  T *stage0 = sm + G::O_STAGE;
  T *s_e = sm + G::O_E;
  const int tid = threadIdx.x;
  const int G0 = gridDim.x;
  const int par = it & 1;
  auto locate = [&](int item, int &shot, int &tile) {
    int lo = 0, hi = b.nshots - 1;  // largest p with prefix[p] <= item
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (b.prefix[mid] <= item)
        lo = mid;
      else
        hi = mid - 1;
    }
    shot = b.order[lo];
    tile = item - b.prefix[lo];
  };
  auto issue_item = [&](int s, int item) {
    int shot, tile;
    locate(item, shot, tile);
    const int ntx = b.ext[shot].ntx;
    const int x0 = L + (tile % ntx) * G::TX, z0 = L + (tile / ntx) * G::TZ;
    issue_tile<G, T>(stage0 + s * G::STAGE, &bars[s], b.maps[2 * shot + par], x0, z0);
  };
  if (tid == 0)
    for (int s = 0; s < ST; ++s) mbar_init(&bars[s], 1);
  __syncthreads();
  if (tid == 0)
    for (int s = 0; s < ST; ++s)
      if (blockIdx.x + s * G0 < nitems) issue_item(s, blockIdx.x + s * G0);
  int j = 0;
  for (int item = blockIdx.x; item < nitems; item += G0, ++j) {
    const int s = ST == 2 ? (j & 1) : 0;
    const uint32_t parity = ST == 2 ? ((j >> 1) & 1) : (j & 1);
    int shot, tile;
    locate(item, shot, tile);
    FusedExtras<T> x = b.ext[shot];
    x.it = it;
    const int e0 = x.tile_off[tile], e1 = x.tile_off[tile + 1];
    const bool ok = mbar_wait_bounded(&bars[s], parity, 1u << 22);
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {
        atomicExch(b.err, 1);
        mbar_wait_bounded(&bars[s], parity, 1u << 22);
        if (ST == 2 && item + G0 < nitems) mbar_wait_bounded(&bars[s ^ 1], ((j + 1) >> 1) & 1, 1u << 22);
      }
      return;
    }
    compute_tile<G, T, KIND, NSLS>(b.args[2 * shot + par], x, stage0 + s * G::STAGE, s_e, tile, e0, e1);
    __syncthreads();
    if (tid == 0) {
      const int nxt = item + ST * G0;
      if (nxt < nitems) {
        fence_proxy_async_smem();
        issue_item(s, nxt);
      }
    }
  }
}

template <typename T, int KIND, int NSLS, bool PERSIST>
static int launch_batch_one(const BatchDev<T> &b, int it, int nitems, int nsm, cudaStream_t st) {
  if constexpr (!TmaPick<T, KIND, NSLS, PERSIST>::OK) {
    return set_error(VI_ERR_ARG, "TMA-staged step does not fit shared memory for this medium");
  } else {
    using G = typename TmaPick<T, KIND, NSLS, PERSIST>::Lay;
    static std::atomic<unsigned long long> attr_set{0};  // one bit per device set up (any thread)
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 64 && !(attr_set & (1ULL << dev))) {
      cudaError_t e = cudaFuncSetAttribute(k_fused_tma_batch<T, KIND, NSLS, PERSIST>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, G::BYTES);
      if (e != cudaSuccess) return cuda_check(e, "batch step smem attribute");
      attr_set |= 1ULL << dev;
    }
    int per = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_fused_tma_batch<T, KIND, NSLS, PERSIST>,
                                                      G::NT, G::BYTES) != cudaSuccess || per < 1) {
      cudaGetLastError();
      per = 1;
    }
    if (nitems <= 0) return VI_OK;  // attribute set-up only
    const int cap = G::STAGES == 2 ? per * nsm : nitems;
    const int grid = nitems < cap ? nitems : cap;
    k_fused_tma_batch<T, KIND, NSLS, PERSIST><<<grid, G::NT, G::BYTES, st>>>(b, it, nitems);
    return VI_OK;
  }
}

template <typename T>
int launch_fused_tma_batch(int kind, int nsls, const BatchDev<T> &b, int it, int nitems, int nsm,
                           bool persist, cudaStream_t st) {
  constexpr bool kSplit = sizeof(T) == 4;
#define VB_CASE(K, N)                                                                        \
  if (kind == K && nsls == N) {                                                              \
    if (kSplit && !persist) return launch_batch_one<T, K, N, !kSplit>(b, it, nitems, nsm, st); \
    return launch_batch_one<T, K, N, true>(b, it, nitems, nsm, st);                          \
  }
#define VB_KIND(K) VB_CASE(K, 0) VB_CASE(K, 1) VB_CASE(K, 2) VB_CASE(K, 3) VB_CASE(K, 4) VB_CASE(K, 5)
  VB_KIND(VI_MEDIUM_ISO)
  VB_KIND(VI_MEDIUM_VTI)
  VB_KIND(VI_MEDIUM_TTI)
#undef VB_KIND
#undef VB_CASE
  return set_error(VI_ERR_ARG, "unsupported medium / nsls combination");
}

template int launch_fused_tma_batch<float>(int, int, const BatchDev<float> &, int, int, int, bool,
                                           cudaStream_t);
template int launch_fused_tma_batch<double>(int, int, const BatchDev<double> &, int, int, int, bool,
                                            cudaStream_t);

template <typename T, int KIND, int NSLS, bool PERSIST>
static int launch_tma_one(const StepArgs<T> &a, const FusedExtras<T> &x, const TmaMaps &maps,
                          int ntiles, int nsm, cudaStream_t st) {
  if constexpr (!TmaPick<T, KIND, NSLS, PERSIST>::OK) {
    return set_error(VI_ERR_ARG, "TMA-staged step does not fit shared memory for this medium");
  } else {
    using G = typename TmaPick<T, KIND, NSLS, PERSIST>::Lay;
    static std::atomic<unsigned long long> attr_set{0};  // one bit per device set up (any thread)
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 64 && !(attr_set & (1ULL << dev))) {
      cudaError_t e = cudaFuncSetAttribute(k_fused_tma<T, KIND, NSLS, PERSIST>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, G::BYTES);
      if (e != cudaSuccess) return cuda_check(e, "TMA step smem attribute");
      attr_set |= 1ULL << dev;
    }
    const int grid = G::STAGES == 2 ? (ntiles < nsm ? ntiles : nsm) : ntiles;
    k_fused_tma<T, KIND, NSLS, PERSIST><<<grid, G::NT, G::BYTES, st>>>(a, x, maps, ntiles);
    return VI_OK;
  }
}

template <typename T>
int launch_fused_tma(int kind, const StepArgs<T> &a, const FusedExtras<T> &x, const TmaMaps &maps,
                     int ntiles, int nsm, bool persist, cudaStream_t st) {
  // the double-precision layouts are single-stage either way
  constexpr bool kSplit = sizeof(T) == 4;
#define VB_CASE(K, N)                                                                     \
  if (kind == K && a.nsls == N) {                                                         \
    if (kSplit && !persist) return launch_tma_one<T, K, N, !kSplit>(a, x, maps, ntiles, nsm, st); \
    return launch_tma_one<T, K, N, true>(a, x, maps, ntiles, nsm, st);                    \
  }
#define VB_KIND(K) VB_CASE(K, 0) VB_CASE(K, 1) VB_CASE(K, 2) VB_CASE(K, 3) VB_CASE(K, 4) VB_CASE(K, 5)
  VB_KIND(VI_MEDIUM_ISO)
  VB_KIND(VI_MEDIUM_VTI)
  VB_KIND(VI_MEDIUM_TTI)
#undef VB_KIND
#undef VB_CASE
  return set_error(VI_ERR_ARG, "unsupported medium / nsls combination");
}

template int launch_fused_tma<float>(int, const StepArgs<float> &, const FusedExtras<float> &,
                                     const TmaMaps &, int, int, bool, cudaStream_t);
template int launch_fused_tma<double>(int, const StepArgs<double> &, const FusedExtras<double> &,
                                      const TmaMaps &, int, int, bool, cudaStream_t);

template <typename Lay>
static TmaBoxes boxes_of(bool ok) {
  TmaBoxes b;
  b.TX = Lay::TX;
  b.TZ = Lay::TZ;
  b.HV = Lay::HV;
  b.HS = Lay::HS;
  b.HVP = Lay::HVP;
  b.HSP = Lay::HSP;
  b.SWp = Lay::SWp;
  b.SH = Lay::SH;
  b.VWp = Lay::VWp;
  b.VH = Lay::VH;
  b.RWp = Lay::RWp;
  b.RH = Lay::RH;
  b.MX0 = Lay::MX0;
  b.MZ0 = Lay::MZ0;
  b.MW = Lay::MW;
  b.MH = Lay::MH;
  b.NM = Lay::NM;
  b.CW = Lay::CW;
  b.CH = Lay::CH;
  b.NC = Lay::NC;
  b.STAGES = Lay::STAGES;
  b.NT = Lay::NT;
  b.ok = ok;
  return b;
}

template <typename T, int KIND, bool P>
static TmaBoxes boxes_kind(int nsls) {
#define VB_G(N)                                                            \
  if (nsls == N)                                                           \
    return boxes_of<typename TmaPick<T, KIND, N, P>::Lay>(TmaPick<T, KIND, N, P>::OK);
  VB_G(0) VB_G(1) VB_G(2) VB_G(3) VB_G(4) VB_G(5)
#undef VB_G
  TmaBoxes b{};
  b.ok = false;
  return b;
}

TmaBoxes tma_boxes(int kind, int nsls, int esize, bool persist) {
  if (esize == 4) {
    if (!persist) {
      if (kind == VI_MEDIUM_ISO) return boxes_kind<float, VI_MEDIUM_ISO, false>(nsls);
      if (kind == VI_MEDIUM_VTI) return boxes_kind<float, VI_MEDIUM_VTI, false>(nsls);
      return boxes_kind<float, VI_MEDIUM_TTI, false>(nsls);
    }
    if (kind == VI_MEDIUM_ISO) return boxes_kind<float, VI_MEDIUM_ISO, true>(nsls);
    if (kind == VI_MEDIUM_VTI) return boxes_kind<float, VI_MEDIUM_VTI, true>(nsls);
    return boxes_kind<float, VI_MEDIUM_TTI, true>(nsls);
  }
  if (kind == VI_MEDIUM_ISO) return boxes_kind<double, VI_MEDIUM_ISO, true>(nsls);
  if (kind == VI_MEDIUM_VTI) return boxes_kind<double, VI_MEDIUM_VTI, true>(nsls);
  return boxes_kind<double, VI_MEDIUM_TTI, true>(nsls);
}

static PFN_cuTensorMapEncodeTiled_v12000 encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault,
                                         &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

int encode_map(CUtensorMap *map, const void *base, int esize, int nx, int nz, long long depth,
               long long plane_stride_elems, int box_x, int box_z, int box_d) {
  auto fn = encoder();
  if (!fn) return set_error(VI_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
  const bool three = box_d > 1 || depth > 1;
  cuuint64_t dims[3] = {(cuuint64_t)nx, (cuuint64_t)nz, (cuuint64_t)(depth > 0 ? depth : 1)};
  cuuint64_t strides[2] = {(cuuint64_t)nx * esize, (cuuint64_t)plane_stride_elems * esize};
  cuuint32_t box[3] = {(cuuint32_t)box_x, (cuuint32_t)box_z, (cuuint32_t)(box_d > 0 ? box_d : 1)};
  cuuint32_t es[3] = {1, 1, 1};
  CUresult r = fn(map, esize == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64,
                  three ? 3 : 2, const_cast<void *>(base), dims, strides, box, es,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS)
    return set_error(VI_ERR_ARG, "cuTensorMapEncodeTiled failed (code " + std::to_string((int)r) + ")");
  return VI_OK;
}

}  // namespace vb
