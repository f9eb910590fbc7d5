// split_tiles.cuh — the per-tile device code of the split step: the
// velocity update of one 64 x 8 tile (direct loads or TMA-staged stress
// taps), its receiver sampling, and the ISO/VTI stress update of one tile.
// The one-launch-per-pass kernels (split.cu) and the wavefront kernel
// (wave.cu) run the same tile code, so their results are bitwise equal.
#pragma once

#include <cstdint>

#include "afda.cuh"
#include "cpml4.cuh"
#include "fused_tma.cuh"
#include "pdl.cuh"
#include "split.cuh"
#include "tma.cuh"
#include "vec.cuh"

namespace vb {

// ---------------------------------------------------------------- velocity
// Velocity pass with direct loads: every stress tap comes through the L1
// cache as an aligned 128-bit load (the 4-cell group and its 12-cell row
// windows start on multiples of 4), no shared-memory staging and no
// barrier, so a CTA's loads are all in flight at once and many CTAs fit
// on an SM.
// CPML, buoyancy, update, force sources, stores and receivers of one
// 4-cell group whose stress derivatives' raw parts are in hxx/hxz (row
// windows) and zxz/zzz (z derivatives).
// OOP: the new velocities go to a.vx_o / a.vz_o (a step from one state
// buffer into another); else in place.
template <typename T, bool PP, bool OOP, bool HINT>
__device__ __forceinline__ void split_vel_finish(const StepArgs<T> &a, const FusedExtras<T> &x, int tile,
                                                 int gi0, int gj, long long g, const Q4<T> &vxi,
                                                 const Q4<T> &vzi, const Q4<T> &r0, const Q4<T> &r1, T r4,
                                                 const T (&hxx)[12], const T (&hxz)[12], Q4<T> zxz,
                                                 Q4<T> zzz, T *psix_o, T *psiz_o, int e0, int e1) {
  const int nx = a.nx, nz = a.nz;
  const int zs = strip_z(gj, nz, a.Tz, a.Bz);
  const bool xstrip = gi0 < a.Lx || gi0 + 3 >= nx - a.Rx;
  Q4<T> dxx = dps4(hxx, a.Dx), dxxz = dms4(hxz, a.Dx);
  if (xstrip)
    cpml_x4(a, gi0, gj, CpmlRows{PX_SXX, T_BH, T_AH, T_IKH}, CpmlRows{PX_SXZ, T_B, T_A, T_IK}, a.psix, psix_o, true,
            dxx, dxxz);
  if (zs >= 0)
    cpml_z4(a, zs, gi0, gj, CpmlRows{PZ_SXZ, T_B, T_A, T_IK}, CpmlRows{PZ_SZZ, T_BH, T_AH, T_IKH}, a.psiz, psiz_o,
            true, zxz, zzz);
  const Q4<T> sx = add4(r0, Q4<T>{{r0.v[1], r0.v[2], r0.v[3], r4}}), sz = add4(r0, r1);
  Q4<T> bx, bz;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    bx.v[k] = two_over_s(sx.v[k]);
    bz.v[k] = two_over_s(sz.v[k]);
  }
  const Q4<T> dt4 = splat4<T>(a.dt);
  Q4<T> vxn = fma4(mul4(dt4, bx), add4(dxx, zxz), vxi);
  Q4<T> vzn = fma4(mul4(dt4, bz), add4(dxxz, zzz), vzi);
  for (int e = e0; e < e1; ++e) {  // force sources of this tile (listed first; e0, e1 loaded early)
    const int4 en = x.tile_ent[e];
    if (en.w > TL_FORCE_Z) break;
    if (en.y != gj || en.x < gi0 || en.x >= gi0 + 4) continue;
    const int k = en.x - gi0;
    const T w = x.it < x.wnt ? x.wavelet[(long long)en.z * x.wnt + x.it] : T(0);
    const T f = x.amp[en.z] * w;
    if (en.w == TL_FORCE_X)
      add_lane4(vxn, k, a.dt * two_over_s(lane4(r0, k) + (k < 3 ? lane4(r0, k + 1) : r4)) * f);
    else
      add_lane4(vzn, k, a.dt * two_over_s(lane4(r0, k) + lane4(r1, k)) * f);
  }
  // v is re-read by the stress pass of the same step: keep it in L2
  sth4((OOP ? a.vx_o : a.vx) + g, vxn, l2_keep_c<HINT>());
  sth4((OOP ? a.vz_o : a.vz) + g, vzn, l2_keep_c<HINT>());
}

// Receivers of the tile, one thread per entry, read back from the tile's
// new velocities after a barrier (every thread of the CTA calls it, after
// the tile's stores): a tile on a receiver line then costs one load per
// receiver instead of every thread scanning the whole list.
template <typename T, bool OOP = false>
__device__ __forceinline__ void split_vel_sample(const StepArgs<T> &a, const FusedExtras<T> &x, int tile) {
  if (!x.traces || x.it >= x.tnt) return;
  const int e0 = x.tile_off[tile], e1 = x.tile_off[tile + 1];
  if (e0 == e1) return;
  __syncthreads();
  const T *vx = OOP ? a.vx_o : a.vx, *vz = OOP ? a.vz_o : a.vz;
  for (int e = e0 + (int)threadIdx.x; e < e1; e += (int)blockDim.x) {
    const int4 en = x.tile_ent[e];
    if (en.w != TL_RECEIVER) continue;
    const long long c = (long long)en.y * a.nx + en.x;
    x.traces[(long long)en.z * x.tnt + x.it] = vx[c];
    x.traces[(long long)(x.nrec + en.z) * x.tnt + x.it] = vz[c];
  }
}

// PP: psi read from the input set and written to the output set (TTI);
// else in place on the input set.  OOP (implies PP): v written to the
// output state too.  AFDA: the grid has the H-AFDA free surface (a
// separate instantiation, so the others carry none of its registers).
template <typename T, bool PP, bool OOP, bool HINT, bool AFDA = false>
__device__ __forceinline__ void split_vel_tile(const StepArgs<T> &a, const FusedExtras<T> &x,
                                               int tile) {
  using G = SplitGeom<T>;
  constexpr int TX = G::TX, TZ = G::TZ;
  T *const psix_o = PP ? a.psix_o : a.psix, *const psiz_o = PP ? a.psiz_o : a.psiz;
  const int x0 = L + (tile % x.ntx) * TX, z0 = L + (tile / x.ntx) * TZ;
  const int nx = a.nx, nz = a.nz, xe = nx - L, ze = nz - L;
  const int tid = threadIdx.x;
  const int r = tid / (TX / 4), lx = 4 * (tid % (TX / 4));
  const int gi0 = x0 + lx, gj = z0 + r;
  if (gi0 >= xe || gj >= ze) return;
  const long long g = (long long)gj * nx + gi0;
  const Q4<T> vxi = ldc4(a.vx + g), vzi = ldc4(a.vz + g);
  const int e0 = x.tile_off[tile], e1 = x.tile_off[tile + 1];
  const Q4<T> r0 = ldg4(a.rho + g), r1 = ldg4(a.rho + g + nx);
  const T r4 = __ldg(a.rho + g + 4);
  T hxx[12], hxz[12];
#pragma unroll
  for (int q = 0; q < 3; ++q) {  // row windows [gi0-4, gi0+8)
    const Q4<T> u = ldg4(a.sxx + g - 4 + 4 * q), w = ldg4(a.sxz + g - 4 + 4 * q);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      hxx[4 * q + k] = u.v[k];
      hxz[4 * q + k] = w.v[k];
    }
  }
  Q4<T> zxz = splat4<T>(0), zzz = splat4<T>(0);
#pragma unroll
  for (int q = -4; q <= 4; ++q) {
    if (q <= 3) {  // ddzm(sxz)
      const T cq = q >= 0 ? a.Dz[q] : -a.Dz[-q - 1];
      const Q4<T> v = q == 0 ? win4(hxz, 4) : ldg4(a.sxz + g + (long long)q * nx);
      zxz = fma4(splat4<T>(cq), v, zxz);
    }
    if (q >= -3) {  // ddzp(szz)
      const T cq = q >= 1 ? a.Dz[q - 1] : -a.Dz[-q];
      const Q4<T> v = ldg4(a.szz + g + (long long)q * nx);
      zzz = fma4(splat4<T>(cq), v, zzz);
    }
  }
  if (AFDA && gj < L + 4) {  // one-sided z derivatives below the H-AFDA surface
    const int qs = gj - L;
    zxz = afda4<0>(a, qs, [&](int m) { return ldg4(a.sxz + (long long)(L + m) * nx + gi0); });
    if (qs < 3) zzz = afda4<1>(a, qs, [&](int m) { return ldg4(a.szz + (long long)(L + 1 + m) * nx + gi0); });
  }
  split_vel_finish<T, PP, OOP, HINT>(a, x, tile, gi0, gj, g, vxi, vzi, r0, r1, r4, hxx, hxz, zxz, zzz, psix_o, psiz_o,
                                     e0, e1);
}

// Tile height of the TMA-staged velocity pass (64 x 8: 34.8 Gpt/s on the
// 2048 x 1024 VTI step; 64 x 16: 34.3; 64 x 32: 33.0; with the L2 hints
// 64 x 8: 37.6, 64 x 16: 37.0).
constexpr int kVelTmaTZ = 8;

// Velocity pass with the stress taps staged by TMA (the default): one
// elected thread issues the tile's three stress boxes (sxx 72 x 8 from
// (x0-4, z0); sxz 72 x 16 from (x0-4, z0-4); szz 64 x 16 from (x0, z0-4))
// on one mbarrier, so all of a tile's DRAM reads are in flight at CTA
// start without holding registers, and the stencil reads come from shared
// memory (2048 x 1024 VTI: 34.8 vs 34.2 Gpt/s for the direct-load pass,
// which the batched step and the gradient's forward sweeps use).
template <typename T, int TZ_ = kVelTmaTZ>
struct SplitVelTmaT {
  static constexpr int TX = 64, TZ = TZ_, NT = TX / 4 * TZ;
  static constexpr int WX = TX + 8, WZ = TX;  // box widths of sxx/sxz and szz
  static constexpr int HZ = TZ + 8;           // rows of the sxz and szz boxes
  static constexpr int O_SXX = 128 / (int)sizeof(T);
  static constexpr int O_SXZ = O_SXX + WX * TZ;
  static constexpr int O_SZZ = O_SXZ + WX * HZ;
  static constexpr int BYTES_TX = (WX * TZ + WX * HZ + WZ * HZ) * (int)sizeof(T);
  static constexpr int SMEM = 128 + BYTES_TX;
  static_assert((WX * TZ * sizeof(T)) % 16 == 0 && (WX * HZ * sizeof(T)) % 16 == 0, "16-byte boxes");
};
template <typename T>
using SplitVelTma = SplitVelTmaT<T>;

template <typename T, bool PP, bool HINT, bool AFDA, typename G = SplitVelTma<T>>
__device__ __forceinline__ void split_vel_tma_tile(const StepArgs<T> &a, const FusedExtras<T> &x,
                                                   const SplitMaps &maps, int tile) {
  constexpr int TX = G::TX, WX = G::WX, WZ = G::WZ;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem_raw);
  const T *s_sxx = reinterpret_cast<T *>(smem_raw) + G::O_SXX;
  const T *s_sxz = reinterpret_cast<T *>(smem_raw) + G::O_SXZ;
  const T *s_szz = reinterpret_cast<T *>(smem_raw) + G::O_SZZ;
  T *const psix_o = PP ? a.psix_o : a.psix, *const psiz_o = PP ? a.psiz_o : a.psiz;
  const int x0 = L + (tile % x.ntx) * TX, z0 = L + (tile / x.ntx) * G::TZ;
  const int nx = a.nx, nz = a.nz, xe = nx - L, ze = nz - L;
  const int tid = threadIdx.x;
  if (tid == 0) mbar_init(bar, 1);
  __syncthreads();
  if (tid == 0) {
    pdl_wait();  // the previous stress pass is complete and visible
    mbar_arrive_expect_tx(bar, G::BYTES_TX);
    tma_load_2d(reinterpret_cast<T *>(smem_raw) + G::O_SXX, &maps.a, x0 - 4, z0, bar);
    tma_load_2d(reinterpret_cast<T *>(smem_raw) + G::O_SXZ, &maps.b, x0 - 4, z0 - 4, bar);
    tma_load_2d(reinterpret_cast<T *>(smem_raw) + G::O_SZZ, &maps.c, x0, z0 - 4, bar);
  }
  const int r = tid / (TX / 4), lx = 4 * (tid % (TX / 4));
  const int gi0 = x0 + lx, gj = z0 + r;
  const bool act = gi0 < xe && gj < ze;
  const long long g = (long long)gj * nx + gi0;
  // the other threads read v (last written by the previous velocity pass,
  // complete before the stress pass that precedes this grid was released)
  // and rho while that stress pass may still drain; sigma comes by TMA
  // after it has completed
  Q4<T> vxi{}, vzi{}, r0{}, r1{};
  T r4 = 0;
  if (act) {
    vxi = ldcg4(a.vx + g);
    vzi = ldcg4(a.vz + g);
    r0 = ldg4(a.rho + g);
    r1 = ldg4(a.rho + g + nx);
    r4 = __ldg(a.rho + g + 4);
  }
  const int e0 = x.tile_off[tile], e1 = x.tile_off[tile + 1];  // the tile's sources, while the boxes land
  pdl_wait();  // every thread, before its first store
  const bool ok = mbar_wait_bounded(bar, 0, 1u << 22);
  if (__syncthreads_or(!ok)) {
    if (tid == 0) {
      atomicOr(x.err, kErrTimeout);
      mbar_wait_bounded(bar, 0, 1u << 22);
    }
    return;
  }
  if (!act) return;
  T hxx[12], hxz[12];
  row12s(s_sxx + r * WX + lx, hxx);
  row12s(s_sxz + (r + 4) * WX + lx, hxz);
  Q4<T> zxz = splat4<T>(0), zzz = splat4<T>(0);
#pragma unroll
  for (int q = -4; q <= 4; ++q) {
    if (q <= 3) {  // ddzm(sxz)
      const T cq = q >= 0 ? a.Dz[q] : -a.Dz[-q - 1];
      const Q4<T> v = q == 0 ? win4(hxz, 4) : lds4(s_sxz + (r + 4 + q) * WX + lx + 4);
      zxz = fma4(splat4<T>(cq), v, zxz);
    }
    if (q >= -3) {  // ddzp(szz)
      const T cq = q >= 1 ? a.Dz[q - 1] : -a.Dz[-q];
      const Q4<T> v = lds4(s_szz + (r + 4 + q) * WZ + lx);
      zzz = fma4(splat4<T>(cq), v, zzz);
    }
  }
  static_assert(G::TZ >= 4, "the H-AFDA rows below the surface lie in the first tile row");
  if (AFDA && gj < L + 4) {  // one-sided z derivatives below the H-AFDA surface (z0 == L)
    const int qs = gj - L;
    zxz = afda4<0>(a, qs, [&](int m) { return lds4(s_sxz + (m + 4) * WX + lx + 4); });
    if (qs < 3) zzz = afda4<1>(a, qs, [&](int m) { return lds4(s_szz + (m + 5) * WZ + lx); });
  }
  split_vel_finish<T, PP, false, HINT>(a, x, tile, gi0, gj, g, vxi, vzi, r0, r1, r4, hxx, hxz, zxz, zzz, psix_o,
                                       psiz_o, e0, e1);
}

// ------------------------------------------------------------------ stress
// OOP: sigma, M and psi read from the input state and written to the
// output one (a.sxx_o.., a.m_o, a.psix_o/psiz_o; the v maps then cover the
// output velocities); else in place.  COMP (FP32, in place): sigma is
// accumulated with its rounding residue (a.slo, two_sum_acc4).  EARLY: the
// kernel's PDL wait comes after the loads of sigma, M and the medium (state
// the previous stress pass wrote: complete before the velocity pass that
// precedes this grid released it), and the next grid is released at once;
// else the wait comes first and the next grid is released at exit.
template <typename T, int KIND, int NSLS, bool OOP, bool HINT, bool COMP = false, bool AFDA = false,
          typename G = SplitStressGeom<T>, bool EARLY = false>
__device__ __forceinline__ void split_stress_tile(const StepArgs<T> &a, const FusedExtras<T> &x,
                                                  const SplitMaps &maps, int tile) {
  static_assert(!COMP || (sizeof(T) == 4 && !OOP), "compensated stress: FP32, in place");
  constexpr int TX = G::TX, TZ = G::TZ, SW = G::BW, PB = G::PB;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem_raw);
  T *s_vx = reinterpret_cast<T *>(smem_raw) + G::O0;
  T *s_vz = s_vx + PB;
  const int x0 = L + (tile % x.ntx) * TX, z0 = L + (tile / x.ntx) * TZ;
  const int nx = a.nx, nz = a.nz, xe = nx - L, ze = nz - L;
  const int tid = threadIdx.x;
  if constexpr (!EARLY) pdl_wait();  // the new velocities are complete and visible
  if (tid == 0) mbar_init(bar, 1);
  __syncthreads();
  if (tid == 0) {
    // EARLY: the issuing thread alone waits for the velocities here; the
    // others first issue the loads of their own state
    if constexpr (EARLY) pdl_wait();
    mbar_arrive_expect_tx(bar, 2 * G::BOX_BYTES);
    tma_load_2d(s_vx, &maps.a, x0 - 4, z0 - 4, bar);
    tma_load_2d(s_vz, &maps.b, x0 - 4, z0 - 4, bar);
  }
  const int r = tid / (TX / 4), lx = 4 * (tid % (TX / 4));
  const int gi0 = x0 + lx, gj = z0 + r;
  const bool act = gi0 < xe && gj < ze;
  const long long g = (long long)gj * nx + gi0;
  // every own-cell operand, issued before the arithmetic
  Q4<T> sxx{}, szz{}, sxz{}, c13{}, c55a{}, c55b{}, c11{}, c33{}, tau{};
  T c55a4 = 0, c55b4 = 0;
  Q4<T> m[3 * (NSLS > 0 ? NSLS : 1)];
  if (act) {
    sxx = EARLY ? ldcg4(a.sxx + g) : ldc4(a.sxx + g);
    szz = EARLY ? ldcg4(a.szz + g) : ldc4(a.szz + g);
    sxz = EARLY ? ldcg4(a.sxz + g) : ldc4(a.sxz + g);
    c13 = ldgh4(a.c13 + g, l2_stream_c<HINT>());
    c55a = ldg4(a.c55 + g);
    c55b = ldg4(a.c55 + g + nx);
    c55a4 = __ldg(a.c55 + g + 4);
    c55b4 = __ldg(a.c55 + g + nx + 4);
    if constexpr (KIND != VI_MEDIUM_ISO) {
      c11 = ldgh4(a.c11 + g, l2_stream_c<HINT>());
      c33 = ldgh4(a.c33 + g, l2_stream_c<HINT>());
    }
    if constexpr (NSLS > 0) {
      tau = ldgh4(a.tau + g, l2_stream_c<HINT>());
#pragma unroll
      for (int q = 0; q < 3 * NSLS; ++q)
        m[q] = EARLY ? ldcgh4(a.m + q * a.mstride + g, l2_stream_c<HINT>())
                     : ldh4(a.m + q * a.mstride + g, l2_stream_c<HINT>());
    }
  }
  if constexpr (EARLY) pdl_wait();  // every thread, before its first store
  uint2 lxx{}, lzz{}, lxz{};  // residues of sxx, szz, sxz (COMP)
  if constexpr (COMP) {
    if (act) {
      lxx = ldh_u2(a.slo + g, l2_stream_c<HINT>());
      lzz = ldh_u2(a.slo + a.slo_plane + g, l2_stream_c<HINT>());
      lxz = ldh_u2(a.slo + 2 * a.slo_plane + g, l2_stream_c<HINT>());
    }
  }
  const int e0 = x.tile_off[tile], e1 = x.tile_off[tile + 1];
  const bool ok = mbar_wait_bounded(bar, 0, 1u << 22);
  if (__syncthreads_or(!ok)) {
    if (tid == 0) {
      atomicOr(x.err, kErrTimeout);
      mbar_wait_bounded(bar, 0, 1u << 22);
    }
    return;
  }
  if (!act) return;
  // ---- strain rates from the staged velocities (cells at box column lx+4)
  const int vb = (r + 4) * SW + lx;
  T hvx[12], hvz[12];
  row12s(s_vx + vb, hvx);
  row12s(s_vz + vb, hvz);
  Q4<T> zvz = splat4<T>(0), zvx = splat4<T>(0);
#pragma unroll
  for (int q = -4; q <= 4; ++q) {
    if (q <= 3) {  // ddzm(vz)
      const T cq = q >= 0 ? a.Dz[q] : -a.Dz[-q - 1];
      const Q4<T> v = q == 0 ? win4(hvz, 4) : lds4(s_vz + vb + q * SW + 4);
      zvz = fma4(splat4<T>(cq), v, zvz);
    }
    if (q >= -3) {  // ddzp(vx)
      const T cq = q >= 1 ? a.Dz[q - 1] : -a.Dz[-q];
      const Q4<T> v = q == 0 ? win4(hvx, 4) : lds4(s_vx + vb + q * SW + 4);
      zvx = fma4(splat4<T>(cq), v, zvx);
    }
  }
  if (AFDA && gj < L + 4) {  // one-sided z derivatives below the H-AFDA surface (grid row L + m
    const int qs = gj - L;     // is box row L + m - (z0 - 4); on the surface row the tau_zz = 0
    const int b0 = L + 4 - z0; // relation sets e_zz)
    if (qs >= 1) zvz = afda4<2>(a, qs, [&](int m) { return lds4(s_vz + (m + b0) * SW + lx + 4); });
    if (qs < 3) zvx = afda4<3>(a, qs, [&](int m) { return lds4(s_vx + (m + b0) * SW + lx + 4); });
  }
  const int zs = strip_z(gj, nz, a.Tz, a.Bz);
  const bool xstrip = gi0 < a.Lx || gi0 + 3 >= nx - a.Rx;
  const bool surf = x.fs && gj == L;
  Q4<T> rxx = dms4(hvx, a.Dx), dxvz = dps4(hvz, a.Dx), rzz = zvz, dzvx = zvx;
  if (xstrip)
    cpml_x4(a, gi0, gj, CpmlRows{PX_VX, T_B, T_A, T_IK}, CpmlRows{PX_VZ, T_BH, T_AH, T_IKH}, a.psix,
            OOP ? a.psix_o : a.psix, true, rxx, dxvz);
  if (zs >= 0)
    cpml_z4(a, zs, gi0, gj, CpmlRows{PZ_VZ, T_B, T_A, T_IK}, CpmlRows{PZ_VX, T_BH, T_AH, T_IKH}, a.psiz,
            OOP ? a.psiz_o : a.psiz, true, rzz, dzvx);
  const Q4<T> rxz = add4(dzvx, dxvz);
  // ---- SLS effective rates and the stress update (4 cells at once)
  const T dt = a.dt;
  const Q4<T> dt4 = splat4<T>(dt);
  Q4<T> exx = rxx, ezz = rzz, exz = rxz;
  if constexpr (NSLS > 0) {
    Q4<T> Sxx = m[0], Szz = m[NSLS], Sxz = m[2 * NSLS];
#pragma unroll
    for (int n = 1; n < NSLS; ++n) {
      Sxx = add4(Sxx, m[0 * NSLS + n]);
      Szz = add4(Szz, m[1 * NSLS + n]);
      Sxz = add4(Sxz, m[2 * NSLS + n]);
    }
    const Q4<T> t1 = add4(tau, splat4<T>(T(1)));
    exx = fma4(t1, rxx, mul4(tau, Sxx));
    ezz = fma4(t1, rzz, mul4(tau, Szz));
    exz = fma4(t1, rxz, mul4(tau, Sxz));
  }
  const Q4<T> C13 = c13;
  const Q4<T> C11 = KIND == VI_MEDIUM_ISO ? fma4(splat4<T>(T(2)), c55a, c13) : c11;
  const Q4<T> C33 = KIND == VI_MEDIUM_ISO ? C11 : c33;
  if (surf) {
#pragma unroll
    for (int k = 0; k < 4; ++k) ezz.v[k] = -(C13.v[k] * exx.v[k]) / C33.v[k];
  }
  const Q4<T> c55r{{c55a.v[1], c55a.v[2], c55a.v[3], c55a4}}, c55br{{c55b.v[1], c55b.v[2], c55b.v[3], c55b4}};
  const Q4<T> C55h = mul4(splat4<T>(T(0.25)), add4(add4(add4(c55a, c55r), c55b), c55br));
  // increments (COMP) or the updated stresses
  Q4<T> ixx, izz, ixz;
  if constexpr (COMP) {
    ixx = mul4(dt4, fma4(C11, exx, mul4(C13, ezz)));
    izz = mul4(dt4, fma4(C13, exx, mul4(C33, ezz)));
    ixz = mul4(dt4, mul4(C55h, exz));
  } else {
    sxx = fma4(dt4, fma4(C11, exx, mul4(C13, ezz)), sxx);
    szz = fma4(dt4, fma4(C13, exx, mul4(C33, ezz)), szz);
    sxz = fma4(dt4, mul4(C55h, exz), sxz);
  }
  if constexpr (NSLS > 0) {
#pragma unroll
    for (int n = 0; n < NSLS; ++n) {
      const Q4<T> a1 = splat4<T>(a.a1[n]), a2 = splat4<T>(a.a2[n]);
      m[0 * NSLS + n] = fma4(dt4, fma4(a1, rxx, mul4(a2, m[0 * NSLS + n])), m[0 * NSLS + n]);
      m[1 * NSLS + n] = surf ? splat4<T>(0) : fma4(dt4, fma4(a1, rzz, mul4(a2, m[1 * NSLS + n])), m[1 * NSLS + n]);
      m[2 * NSLS + n] = fma4(dt4, fma4(a1, rxz, mul4(a2, m[2 * NSLS + n])), m[2 * NSLS + n]);
    }
#pragma unroll
    for (int q = 0; q < 3 * NSLS; ++q)
      sth4(OOP ? a.m_o + q * a.mstride_o + g : a.m + q * a.mstride + g, m[q], l2_stream_c<HINT>());
  }
  for (int e = e0; e < e1; ++e) {  // explosive sources (after the force ones, before receivers)
    const int4 en = x.tile_ent[e];
    if (en.w < TL_EXPLOSIVE) continue;
    if (en.w > TL_EXPLOSIVE) break;
    if (en.y != gj || en.x < gi0 || en.x >= gi0 + 4) continue;
    const T w = x.it < x.wnt ? x.wavelet[(long long)en.z * x.wnt + x.it] : T(0);
    add_lane4(COMP ? ixx : sxx, en.x - gi0, dt * x.amp[en.z] * w);
    add_lane4(COMP ? izz : szz, en.x - gi0, dt * x.amp[en.z] * w);
  }
  if constexpr (COMP) {
    two_sum_acc4(sxx, lxx, ixx);
    two_sum_acc4(szz, lzz, izz);
    two_sum_acc4(sxz, lxz, ixz);
    if (surf) lzz = make_uint2(0, 0);
    sth_u2(a.slo + g, lxx, l2_stream_c<HINT>());
    sth_u2(a.slo + a.slo_plane + g, lzz, l2_stream_c<HINT>());
    sth_u2(a.slo + 2 * a.slo_plane + g, lxz, l2_stream_c<HINT>());
  }
  if (surf) szz = Q4<T>{{0, 0, 0, 0}};
  if (!finite3(sxx, szz, sxz)) atomicOr(x.err, kErrNonFinite);
  T *const osxx = OOP ? a.sxx_o : a.sxx, *const oszz = OOP ? a.szz_o : a.szz, *const osxz = OOP ? a.sxz_o : a.sxz;
  // sigma is re-read by the next velocity pass: keep it in L2
  sth4(osxx + g, sxx, l2_keep_c<HINT>());
  sth4(oszz + g, szz, l2_keep_c<HINT>());
  sth4(osxz + g, sxz, l2_keep_c<HINT>());
  if (x.fs == kFsImaging) {
    // stress images: szz(L-k) = -szz(L+k), k = 1..4; sxz(L-1-k) = -sxz(L+k), k = 0..3
    const int k = gj - L;
    if (k >= 1 && k <= L) {
      Q4<T> im;
#pragma unroll
      for (int q = 0; q < 4; ++q) im.v[q] = -szz.v[q];
      stg4(oszz + (long long)(L - k) * nx + gi0, im);
    }
    if (k >= 0 && k < L) {
      Q4<T> im;
#pragma unroll
      for (int q = 0; q < 4; ++q) im.v[q] = -sxz.v[q];
      stg4(osxz + (long long)(L - 1 - k) * nx + gi0, im);
    }
  }
}

}  // namespace vb
