// split.cu — the step as two kernels per time step.
//
//   k_split_vel_tma: v += dt*b*(div sigma + f) on a 64 x 8 tile from TMA
//                    boxes of the stress taps (the default; below).
//   k_split_vel_ldg: the same update on a 64 x 8 tile where every
//                    stress tap is an aligned 128-bit load through L1 (the
//                    tile's loads all in flight at once, no staging).  Both
//                    velocity kernels serve every medium.
//   k_split_stress:  ISO/VTI SLS stress + memory variables on a 64 x 8 tile;
//                    the new velocities of the tile + 4-cell halo are staged
//                    by TMA, every own-cell operand (sigma, M, stiffness,
//                    tau) is a 128-bit load issued before the arithmetic.
//                    Threads on the rows below the free surface also write
//                    the stress images, so no separate mirror pass is needed.
//   k_split_stress_tti (split_tti.cu): the TTI stress pass.
//
// The kernels of one call are chained by programmatic dependent launch:
// each is launched while its predecessor drains and waits at entry for it
// to complete, which hides the launch latency between the two passes
// (2048 x 1024 VTI: 29.4 vs 28.0 Gpt/s on B200).  Issuing the independent
// loads (sigma, M, medium) before the wait measured slower.
//
// Each cell's operands cross the SMs' ports once per kernel: 8 planes for
// the velocity kernel (sigma 3 + v 2 + rho read, v written) and
// 2 + 2*(3 + 3N) + N_m for the stress kernel — 156 B per point per step
// for FP32 VTI with 3 SLS against 136 B for a single fused pass, but with
// a fraction of the fused kernel's arithmetic per byte.  When the new v
// and sigma fit in half the L2, their stores are marked evict_last and the
// memory variables and once-read stiffnesses evict_first (the HINT
// template parameter), so the other pass of the step finds v and sigma in
// L2: 235 MB per step then reach DRAM on 2048 x 1024 against 290 MB of
// operands (37.5 vs 35.0 Gpt/s).
// The out-of-place forms (OOP: the state read from one buffer and written
// to another) serve the gradient's segment recompute.
// In place is safe for ISO/VTI: the velocity kernel reads v only at its own
// cells and never writes sigma; the stress kernel reads v and writes sigma,
// M and psi only at its own cells.  The TTI stress pass also reads M and
// psi on a ring of neighbouring cells, so for TTI those two ping-pong
// between buffers every step (sigma and v stay in place).
#include <atomic>
#include <cudaTypedefs.h>

#include <cstdint>
#include <vector>

#include "afda.cuh"
#include "fused_tma.cuh"
#include "pdl.cuh"
#include "plan.cuh"
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
                                                 Q4<T> zzz, T *psix_o, T *psiz_o) {
  const int nx = a.nx, nz = a.nz;
  const int zs = strip_z(gj, nz, a.Tz, a.Bz);
  const bool xstrip = gi0 < a.Lx || gi0 + 3 >= nx - a.Rx;
  Q4<T> dxx = dps4(hxx, a.Dx), dxxz = dms4(hxz, a.Dx);
  if (xstrip) {  // CPML, cell by cell
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int gi = gi0 + k;
      const int xs = strip_x(gi, nx, a.Lx, a.Rx);
      if (xs >= 0) {
        const T *tb = a.tx;
        const long long o = (long long)gj * a.wx + xs;
        const T p0 = tb[T_BH * nx + gi] * a.psix[PX_SXX * a.psix_plane + o] + tb[T_AH * nx + gi] * dxx.v[k];
        const T p1 = tb[T_B * nx + gi] * a.psix[PX_SXZ * a.psix_plane + o] + tb[T_A * nx + gi] * dxxz.v[k];
        psix_o[PX_SXX * a.psix_plane + o] = p0;
        psix_o[PX_SXZ * a.psix_plane + o] = p1;
        dxx.v[k] = dxx.v[k] * tb[T_IKH * nx + gi] + p0;
        dxxz.v[k] = dxxz.v[k] * tb[T_IK * nx + gi] + p1;
      }
    }
  }
  if (zs >= 0) {
    const T *tb = a.tz;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const long long o = (long long)zs * nx + gi0 + k;
      const T p0 = tb[T_B * nz + gj] * a.psiz[PZ_SXZ * a.psiz_plane + o] + tb[T_A * nz + gj] * zxz.v[k];
      const T p1 = tb[T_BH * nz + gj] * a.psiz[PZ_SZZ * a.psiz_plane + o] + tb[T_AH * nz + gj] * zzz.v[k];
      psiz_o[PZ_SXZ * a.psiz_plane + o] = p0;
      psiz_o[PZ_SZZ * a.psiz_plane + o] = p1;
      zxz.v[k] = zxz.v[k] * tb[T_IK * nz + gj] + p0;
      zzz.v[k] = zzz.v[k] * tb[T_IKH * nz + gj] + p1;
    }
  }
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
  const int e0 = x.tile_off[tile], e1 = x.tile_off[tile + 1];
  for (int e = e0; e < e1; ++e) {  // force sources of this tile (listed first)
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
  split_vel_finish<T, PP, OOP, HINT>(a, x, tile, gi0, gj, g, vxi, vzi, r0, r1, r4, hxx, hxz, zxz, zzz, psix_o, psiz_o);
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
template <typename T>
struct SplitVelTma {
  static constexpr int TX = 64, TZ = kVelTmaTZ, NT = TX / 4 * TZ;
  static constexpr int WX = TX + 8, WZ = TX;  // box widths of sxx/sxz and szz
  static constexpr int HZ = TZ + 8;           // rows of the sxz and szz boxes
  static constexpr int O_SXX = 128 / (int)sizeof(T);
  static constexpr int O_SXZ = O_SXX + WX * TZ;
  static constexpr int O_SZZ = O_SXZ + WX * HZ;
  static constexpr int BYTES_TX = (WX * TZ + WX * HZ + WZ * HZ) * (int)sizeof(T);
  static constexpr int SMEM = 128 + BYTES_TX;
  static_assert((WX * TZ * sizeof(T)) % 16 == 0 && (WX * HZ * sizeof(T)) % 16 == 0, "16-byte boxes");
};

template <typename T, bool PP, bool HINT, bool AFDA>
__device__ __forceinline__ void split_vel_tma_tile(const StepArgs<T> &a, const FusedExtras<T> &x,
                                                   const SplitMaps &maps, int tile) {
  using G = SplitVelTma<T>;
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
    mbar_arrive_expect_tx(bar, G::BYTES_TX);
    tma_load_2d(reinterpret_cast<T *>(smem_raw) + G::O_SXX, &maps.a, x0 - 4, z0, bar);
    tma_load_2d(reinterpret_cast<T *>(smem_raw) + G::O_SXZ, &maps.b, x0 - 4, z0 - 4, bar);
    tma_load_2d(reinterpret_cast<T *>(smem_raw) + G::O_SZZ, &maps.c, x0, z0 - 4, bar);
  }
  const int r = tid / (TX / 4), lx = 4 * (tid % (TX / 4));
  const int gi0 = x0 + lx, gj = z0 + r;
  const bool act = gi0 < xe && gj < ze;
  const long long g = (long long)gj * nx + gi0;
  Q4<T> vxi{}, vzi{}, r0{}, r1{};
  T r4 = 0;
  if (act) {
    vxi = ldc4(a.vx + g);
    vzi = ldc4(a.vz + g);
    r0 = ldg4(a.rho + g);
    r1 = ldg4(a.rho + g + nx);
    r4 = __ldg(a.rho + g + 4);
  }
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
  split_vel_finish<T, PP, false, HINT>(a, x, tile, gi0, gj, g, vxi, vzi, r0, r1, r4, hxx, hxz, zxz, zzz, psix_o, psiz_o);
}

// AFDA: the grid has the H-AFDA free surface (a separate instantiation,
// so the others carry none of its code)
template <typename T, bool PP, bool HINT, bool AFDA>
__global__ void __launch_bounds__(SplitVelTma<T>::NT, (sizeof(T) == 4 ? 1024 : 512) / SplitVelTma<T>::NT)
    k_split_vel_tma(const __grid_constant__ StepArgs<T> a, const FusedExtras<T> x, const __grid_constant__ SplitMaps maps) {
  pdl_wait();  // the previous stress pass is complete and visible
  split_vel_tma_tile<T, PP, HINT, AFDA>(a, x, maps, blockIdx.x);
  split_vel_sample<T>(a, x, blockIdx.x);
}

template <typename T, bool PP, bool OOP, bool HINT, bool AFDA>
__global__ void __launch_bounds__(SplitGeom<T>::NT, (sizeof(T) == 4 ? 1024 : 512) / SplitGeom<T>::NT)
    k_split_vel_ldg(const __grid_constant__ StepArgs<T> a, const FusedExtras<T> x) {
  pdl_wait();  // the previous stress pass is complete and visible
  split_vel_tile<T, PP, OOP, HINT, AFDA>(a, x, blockIdx.x);
  split_vel_sample<T, OOP>(a, x, blockIdx.x);
}

// Batched: one tile of one shot per CTA; the step parity selects the shot's
// argument set (ping-pong buffers for TTI).  AFDA: some shot has the H-AFDA
// surface (each tile still checks its own shot's kind).
template <typename T, bool PP, bool AFDA>
__global__ void __launch_bounds__(SplitGeom<T>::NT, (sizeof(T) == 4 ? 1024 : 512) / SplitGeom<T>::NT)
    k_split_vel_batch(const BatchDev<T> b, int it) {
  pdl_wait();
  int shot, tile;
  batch_locate(b, blockIdx.x, shot, tile);
  FusedExtras<T> x = b.ext[shot];
  x.it = it;
  if (AFDA && x.fs == kFsAfda)
    split_vel_tile<T, PP, false, false, true>(b.args[2 * shot + (it & 1)], x, tile);
  else
    split_vel_tile<T, PP, false, false>(b.args[2 * shot + (it & 1)], x, tile);
  split_vel_sample<T>(b.args[2 * shot + (it & 1)], x, tile);
}

// ------------------------------------------------------------------ stress
// OOP: sigma, M and psi read from the input state and written to the
// output one (a.sxx_o.., a.m_o, a.psix_o/psiz_o; the v maps then cover the
// output velocities); else in place.  COMP (FP32, in place): sigma is
// accumulated with its rounding residue (a.slo, two_sum_acc4).
template <typename T, int KIND, int NSLS, bool OOP, bool HINT, bool COMP = false, bool AFDA = false,
          typename G = SplitStressGeom<T>>
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
  pdl_wait();  // the new velocities are complete and visible
  if (tid == 0) mbar_init(bar, 1);
  __syncthreads();
  if (tid == 0) {
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
    sxx = ldc4(a.sxx + g);
    szz = ldc4(a.szz + g);
    sxz = ldc4(a.sxz + g);
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
      for (int q = 0; q < 3 * NSLS; ++q) m[q] = ldh4(a.m + q * a.mstride + g, l2_stream_c<HINT>());
    }
  }
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
  if (xstrip) {  // CPML, cell by cell
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int gi = gi0 + k;
      const int xs = strip_x(gi, nx, a.Lx, a.Rx);
      if (xs >= 0) {
        const T *tb = a.tx;
        const long long o = (long long)gj * a.wx + xs;
        T *q = OOP ? a.psix_o : a.psix;
        const T p0 = tb[T_B * nx + gi] * a.psix[PX_VX * a.psix_plane + o] + tb[T_A * nx + gi] * rxx.v[k];
        const T p1 = tb[T_BH * nx + gi] * a.psix[PX_VZ * a.psix_plane + o] + tb[T_AH * nx + gi] * dxvz.v[k];
        q[PX_VX * a.psix_plane + o] = p0;
        q[PX_VZ * a.psix_plane + o] = p1;
        rxx.v[k] = rxx.v[k] * tb[T_IK * nx + gi] + p0;
        dxvz.v[k] = dxvz.v[k] * tb[T_IKH * nx + gi] + p1;
      }
    }
  }
  if (zs >= 0) {
    const T *tb = a.tz;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const long long o = (long long)zs * nx + gi0 + k;
      T *q = OOP ? a.psiz_o : a.psiz;
      const T p0 = tb[T_B * nz + gj] * a.psiz[PZ_VZ * a.psiz_plane + o] + tb[T_A * nz + gj] * rzz.v[k];
      const T p1 = tb[T_BH * nz + gj] * a.psiz[PZ_VX * a.psiz_plane + o] + tb[T_AH * nz + gj] * dzvx.v[k];
      q[PZ_VZ * a.psiz_plane + o] = p0;
      q[PZ_VX * a.psiz_plane + o] = p1;
      rzz.v[k] = rzz.v[k] * tb[T_IK * nz + gj] + p0;
      dzvx.v[k] = dzvx.v[k] * tb[T_IKH * nz + gj] + p1;
    }
  }
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

template <typename T, int KIND, int NSLS, bool OOP, bool HINT, bool COMP, bool AFDA>
__global__ void __launch_bounds__(SplitStressGeom<T>::NT, (sizeof(T) == 4 ? 512 : 256) / SplitStressGeom<T>::NT)
    k_split_stress(const __grid_constant__ StepArgs<T> a, const __grid_constant__ FusedExtras<T> x,
                   const __grid_constant__ SplitMaps maps) {
  split_stress_tile<T, KIND, NSLS, OOP, HINT, COMP, AFDA>(a, x, maps, blockIdx.x);
}

template <typename T, int KIND, int NSLS, bool COMP, bool AFDA>
__global__ void __launch_bounds__(SplitStressGeomBatch<T>::NT, (sizeof(T) == 4 ? 512 : 256) / SplitStressGeomBatch<T>::NT)
    k_split_stress_batch(const BatchDev<T> b, int it) {
  int shot, tile;
  batch_locate(b, blockIdx.x, shot, tile);
  FusedExtras<T> x = b.ext[shot];
  x.it = it;
  // COMP: compensated FP32 shots carry the stress residues, as the unbatched
  // split step; AFDA: some shot has the H-AFDA surface
  using G = SplitStressGeomBatch<T>;
  if (AFDA && x.fs == kFsAfda)
    split_stress_tile<T, KIND, NSLS, false, false, COMP, true, G>(b.args[2 * shot + (it & 1)], x, b.smaps[shot],
                                                                  tile);
  else
    split_stress_tile<T, KIND, NSLS, false, false, COMP, false, G>(b.args[2 * shot + (it & 1)], x, b.smaps[shot],
                                                                   tile);
}

// ------------------------------------------------------------------- host
template <typename T, int KIND, int NSLS, bool OOP, bool HINT, bool COMP = false, bool AFDA = false>
static int launch_stress_k(const StepArgs<T> &a, const FusedExtras<T> &x, const SplitMaps &m,
                           int ntiles, cudaStream_t st, bool pdl) {
  using SG = SplitStressGeom<T>;
  static std::atomic<unsigned long long> attr_set{0};  // one bit per device set up (any thread)
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && !(attr_set & (1ULL << dev))) {
    cudaError_t e = cudaFuncSetAttribute(k_split_stress<T, KIND, NSLS, OOP, HINT, COMP, AFDA>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, SG::SMEM);
    if (e != cudaSuccess) return cuda_check(e, "split stress smem attribute");
    attr_set |= 1ULL << dev;
  }
  return cuda_check(launch_pdl(k_split_stress<T, KIND, NSLS, OOP, HINT, COMP, AFDA>, dim3(ntiles), dim3(SG::NT),
                               (size_t)SG::SMEM, st, pdl, a, x, m),
                    "split stress launch");
}

// out of place when the caller set the output state (a.sxx_o); compensated
// (FP32, in place) when the caller set the residue planes (a.slo)
template <typename T, int KIND, int NSLS>
static int launch_stress(const StepArgs<T> &a, const FusedExtras<T> &x, const SplitMaps &m,
                         int ntiles, cudaStream_t st, bool pdl) {
  // the out-of-place form (the gradient's recompute) always hints
  if (a.sxx_o) return launch_stress_k<T, KIND, NSLS, true, true>(a, x, m, ntiles, st, pdl);
  if constexpr (sizeof(T) == 4) {
    if (a.slo) {
      if (x.fs == kFsAfda)
        return x.l2hint ? launch_stress_k<T, KIND, NSLS, false, true, true, true>(a, x, m, ntiles, st, pdl)
                        : launch_stress_k<T, KIND, NSLS, false, false, true, true>(a, x, m, ntiles, st, pdl);
      return x.l2hint ? launch_stress_k<T, KIND, NSLS, false, true, true>(a, x, m, ntiles, st, pdl)
                      : launch_stress_k<T, KIND, NSLS, false, false, true>(a, x, m, ntiles, st, pdl);
    }
  }
  if (x.fs == kFsAfda)
    return x.l2hint ? launch_stress_k<T, KIND, NSLS, false, true, false, true>(a, x, m, ntiles, st, pdl)
                    : launch_stress_k<T, KIND, NSLS, false, false, false, true>(a, x, m, ntiles, st, pdl);
  return x.l2hint ? launch_stress_k<T, KIND, NSLS, false, true>(a, x, m, ntiles, st, pdl)
                  : launch_stress_k<T, KIND, NSLS, false, false>(a, x, m, ntiles, st, pdl);
}

template <typename T, bool AFDA>
static cudaError_t launch_vel_ldg_k(const StepArgs<T> &a, const FusedExtras<T> &x, int ntiles, cudaStream_t st,
                                    bool pdl) {
  using G = SplitGeom<T>;
  const bool oop = a.vx_o != nullptr, pp = oop || a.psix_o != a.psix || a.psiz_o != a.psiz;
  return oop        ? launch_pdl(k_split_vel_ldg<T, true, true, true, AFDA>, dim3(ntiles), dim3(G::NT), 0, st, pdl, a, x)
         : pp       ? (x.l2hint ? launch_pdl(k_split_vel_ldg<T, true, false, true, AFDA>, dim3(ntiles), dim3(G::NT), 0, st, pdl, a, x)
                                : launch_pdl(k_split_vel_ldg<T, true, false, false, AFDA>, dim3(ntiles), dim3(G::NT), 0, st, pdl, a, x))
         : x.l2hint ? launch_pdl(k_split_vel_ldg<T, false, false, true, AFDA>, dim3(ntiles), dim3(G::NT), 0, st, pdl, a, x)
                    : launch_pdl(k_split_vel_ldg<T, false, false, false, AFDA>, dim3(ntiles), dim3(G::NT), 0, st, pdl, a, x);
}

template <typename T>
int launch_split_vel(const StepArgs<T> &a, const FusedExtras<T> &x, int ntiles, cudaStream_t st,
                     bool pdl) {
  const cudaError_t e = x.fs == kFsAfda ? launch_vel_ldg_k<T, true>(a, x, ntiles, st, pdl)
                                        : launch_vel_ldg_k<T, false>(a, x, ntiles, st, pdl);
  return cuda_check(e, "split velocity launch");
}

template <typename T>
int launch_split_stress(int kind, const StepArgs<T> &a, const FusedExtras<T> &x,
                        const SplitMaps &m, int ntiles, cudaStream_t st, bool pdl) {
#define VB_CASE(K, N) \
  if (kind == K && a.nsls == N) return launch_stress<T, K, N>(a, x, m, ntiles, st, pdl);
#define VB_KIND(K) VB_CASE(K, 0) VB_CASE(K, 1) VB_CASE(K, 2) VB_CASE(K, 3) VB_CASE(K, 4) VB_CASE(K, 5)
  VB_KIND(VI_MEDIUM_ISO)
  VB_KIND(VI_MEDIUM_VTI)
#undef VB_KIND
#undef VB_CASE
  return set_error(VI_ERR_ARG, "the split step covers ISO and VTI media");
}

template <typename T>
int launch_split_vel_batch(int kind, bool afda, const BatchDev<T> &b, int it, int nitems, cudaStream_t st,
                           bool pdl) {
  using G = SplitGeom<T>;
  if (nitems <= 0) return VI_OK;
  const bool tti = kind == VI_MEDIUM_TTI;
  const cudaError_t e =
      tti  ? (afda ? launch_pdl(k_split_vel_batch<T, true, true>, dim3(nitems), dim3(G::NT), 0, st, pdl, b, it)
                   : launch_pdl(k_split_vel_batch<T, true, false>, dim3(nitems), dim3(G::NT), 0, st, pdl, b, it))
           : (afda ? launch_pdl(k_split_vel_batch<T, false, true>, dim3(nitems), dim3(G::NT), 0, st, pdl, b, it)
                   : launch_pdl(k_split_vel_batch<T, false, false>, dim3(nitems), dim3(G::NT), 0, st, pdl, b, it));
  return cuda_check(e, "batched split velocity launch");
}

template <typename T, int KIND, int NSLS, bool COMP, bool AFDA>
static int launch_stress_batch_k(const BatchDev<T> &b, int it, int nitems, cudaStream_t st, bool pdl) {
  using SG = SplitStressGeomBatch<T>;
  static std::atomic<unsigned long long> attr_set{0};  // one bit per device set up (any thread)
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && !(attr_set & (1ULL << dev))) {
    cudaError_t e = cudaFuncSetAttribute(k_split_stress_batch<T, KIND, NSLS, COMP, AFDA>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, SG::SMEM);
    if (e != cudaSuccess) return cuda_check(e, "batched split stress smem attribute");
    attr_set |= 1ULL << dev;
  }
  if (nitems <= 0) return VI_OK;  // attribute set-up only
  return cuda_check(launch_pdl(k_split_stress_batch<T, KIND, NSLS, COMP, AFDA>, dim3(nitems), dim3(SG::NT),
                               (size_t)SG::SMEM, st, pdl, b, it),
                    "batched split stress launch");
}

template <typename T, int KIND, int NSLS>
static int launch_stress_batch(bool comp, bool afda, const BatchDev<T> &b, int it, int nitems, cudaStream_t st,
                               bool pdl) {
  if constexpr (sizeof(T) == 4)
    if (comp)
      return afda ? launch_stress_batch_k<T, KIND, NSLS, true, true>(b, it, nitems, st, pdl)
                  : launch_stress_batch_k<T, KIND, NSLS, true, false>(b, it, nitems, st, pdl);
  return afda ? launch_stress_batch_k<T, KIND, NSLS, false, true>(b, it, nitems, st, pdl)
              : launch_stress_batch_k<T, KIND, NSLS, false, false>(b, it, nitems, st, pdl);
}

template <typename T>
int launch_split_stress_batch(int kind, int nsls, bool comp, bool afda, const BatchDev<T> &b, int it, int nitems,
                              cudaStream_t st, bool pdl) {
  if (kind == VI_MEDIUM_TTI) return launch_split_stress_tti_batch<T>(nsls, comp, afda, b, it, nitems, st, pdl);
#define VB_CASE(K, N) \
  if (kind == K && nsls == N) return launch_stress_batch<T, K, N>(comp, afda, b, it, nitems, st, pdl);
#define VB_KIND(K) VB_CASE(K, 0) VB_CASE(K, 1) VB_CASE(K, 2) VB_CASE(K, 3) VB_CASE(K, 4) VB_CASE(K, 5)
  VB_KIND(VI_MEDIUM_ISO)
  VB_KIND(VI_MEDIUM_VTI)
#undef VB_KIND
#undef VB_CASE
  return set_error(VI_ERR_ARG, "batched split step: unknown medium or nsls");
}

static bool al16(const void *q) { return ((uintptr_t)q & 15) == 0; }

template <typename T>
bool split_eligible(const vi_plan *p, const StepArgs<T> &a) {
  const vi_config &c = p->cfg;
  if (c.nx % 4 != 0) return false;
  if (((size_t)c.nx * sizeof(T)) % 16 != 0) return false;
  const void *ptrs[] = {a.vx,  a.vz,  a.sxx, a.szz, a.sxz, a.rho, a.c11,
                        a.c13, a.c15, a.c33, a.c35, a.c55, a.tau, a.m};
  for (const void *q : ptrs)
    if (q && !al16(q)) return false;
  if (c.nsls > 0 && ((size_t)a.mstride * sizeof(T)) % 16 != 0) return false;
  return true;
}

template <typename T, bool AFDA>
static int launch_vel_tma_k(const StepArgs<T> &a, const FusedExtras<T> &x, const SplitMaps &m,
                            int ntiles, cudaStream_t st, bool pdl) {
  using G = SplitVelTma<T>;
  const bool pp = a.psix_o != a.psix || a.psiz_o != a.psiz;
  static std::atomic<unsigned long long> attr_set{0};  // one bit per device set up (any thread)
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && !(attr_set & (1ULL << dev))) {
    for (auto k : {k_split_vel_tma<T, true, true, AFDA>, k_split_vel_tma<T, false, true, AFDA>,
                   k_split_vel_tma<T, true, false, AFDA>, k_split_vel_tma<T, false, false, AFDA>}) {
      const cudaError_t ea = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM);
      if (ea != cudaSuccess) return cuda_check(ea, "split velocity (TMA) smem attribute");
    }
    attr_set |= 1ULL << dev;
  }
  const cudaError_t e =
      pp ? (x.l2hint ? launch_pdl(k_split_vel_tma<T, true, true, AFDA>, dim3(ntiles), dim3(G::NT), (size_t)G::SMEM, st, pdl, a, x, m)
                     : launch_pdl(k_split_vel_tma<T, true, false, AFDA>, dim3(ntiles), dim3(G::NT), (size_t)G::SMEM, st, pdl, a, x, m))
         : (x.l2hint ? launch_pdl(k_split_vel_tma<T, false, true, AFDA>, dim3(ntiles), dim3(G::NT), (size_t)G::SMEM, st, pdl, a, x, m)
                     : launch_pdl(k_split_vel_tma<T, false, false, AFDA>, dim3(ntiles), dim3(G::NT), (size_t)G::SMEM, st, pdl, a, x, m));
  return cuda_check(e, "split velocity (TMA) launch");
}

template <typename T>
static int launch_vel_tma(const StepArgs<T> &a, const FusedExtras<T> &x, const SplitMaps &m,
                          int ntiles, cudaStream_t st, bool pdl) {
  return x.fs == kFsAfda ? launch_vel_tma_k<T, true>(a, x, m, ntiles, st, pdl)
                         : launch_vel_tma_k<T, false>(a, x, m, ntiles, st, pdl);
}

template <typename T>
int split_steps(vi_plan *p, StepArgs<T> a, const vi_shot *s, int it0, int nsteps, cudaStream_t st,
                int mode) {
  const bool pipelined = mode == kSplitPipelined, vel_tma = mode == kSplitVelTma;
  using G = SplitGeom<T>;
  const vi_config &c = p->cfg;
  const bool tti = c.medium == VI_MEDIUM_TTI;
  if (!split_eligible<T>(p, a))
    return set_error(VI_ERR_ARG, "split step needs nx % 4 == 0 and 16-byte aligned planes");
  if (pipelined && tti)
    return set_error(VI_ERR_ARG, "the pipelined split step covers ISO and VTI media");
  if (pipelined && !split_p_fits(c.medium, c.nsls, (int)sizeof(T)))
    return set_error(VI_ERR_ARG, "pipelined split step does not fit shared memory for this medium");
  if (nsteps == 0) return VI_OK;
  const size_t np = (size_t)c.nx * c.nz;
  int rc = VI_OK;
  if constexpr (sizeof(T) == 4) {
    if (c.precision == VI_F32C) {
      if (pipelined)
        return set_error(VI_ERR_ARG, "compensated FP32 (VI_F32C) runs on the one-tile-per-CTA split pair");
      // compensated stress accumulation: the residue planes live in the plan
      if (!p->slo) {
        size_t have = 0;
        if ((rc = ensure_buffer(p, &p->slo, &have, 3 * np * sizeof(uint16_t)))) return rc;
        p->slo_valid = false;
      }
      if (!p->slo_valid) {
        if ((rc = cuda_check(cudaMemsetAsync(p->slo, 0, 3 * np * sizeof(uint16_t), st), "zero stress residues")))
          return rc;
        p->slo_valid = true;
      }
      a.slo = (uint16_t *)p->slo;
      a.slo_plane = (long long)np;
    }
  }
  T *user_m = a.m, *alt_m = nullptr;
  const long long user_ms = a.mstride;
  if (tti && c.nsls > 0) {
    // the plan's second state copy holds the other memory-variable set
    if (!p->alt) {
      const size_t bytes = (5 + 3 * (size_t)c.nsls) * np * sizeof(T);
      size_t have = 0;
      rc = ensure_buffer(p, &p->alt, &have, bytes);
      if (rc) return rc;
      rc = cuda_check(cudaMemsetAsync(p->alt, 0, bytes, st), "zero alt state");
      if (rc) return rc;
    }
    alt_m = (T *)p->alt + 5 * np;
  }
  // per-tile source/receiver lists of the velocity tiling and (pipelined:
  // its own 64 x 8 tiling) the stress tiling, in one buffer
  int vtx = G::TX, vtz = G::TZ, stx = SplitStressGeom<T>::TX, stz = SplitStressGeom<T>::TZ;
  if (vel_tma) {
    vtx = SplitVelTma<T>::TX;
    vtz = SplitVelTma<T>::TZ;
  }
  if (tti) {
    stx = SplitTtiGeom<T>::TX;
    stz = SplitTtiGeom<T>::TZ;
  }
  if (pipelined) split_p_tiles(vtx, vtz, stx, stz);
  int ntx, ntz, sntx, sntz;
  std::vector<int> off, soff;
  std::vector<int4> ent, sent;
  build_tile_lists(c.nx, c.nz, vtx, vtz, 0, s, off, ent, ntx, ntz);
  build_tile_lists(c.nx, c.nz, stx, stz, 0, s, soff, sent, sntx, sntz);
  const int nvoff = (int)off.size();
  for (int v : soff) off.push_back(v + (int)ent.size());
  ent.insert(ent.end(), sent.begin(), sent.end());
  int *d_off = nullptr;
  int4 *d_ent = nullptr;
  rc = stage_tile_lists(p, off, ent, st, &d_off, &d_ent);
  if (rc) return rc;
  const int e = sizeof(T);
  SplitMaps ms, mv;
  SplitPMaps pv, ps;
  if (pipelined) {
    if ((rc = encode_split_p<T>(c, a, pv, ps))) return rc;
  } else {
    const int bw = tti ? SplitTtiGeom<T>::BW : SplitStressGeom<T>::BW;
    const int bh = tti ? SplitTtiGeom<T>::BH : SplitStressGeom<T>::BH;
    if ((rc = encode_map(&ms.a, a.vx, e, c.nx, c.nz, 1, 0, bw, bh, 1))) return rc;
    if ((rc = encode_map(&ms.b, a.vz, e, c.nx, c.nz, 1, 0, bw, bh, 1))) return rc;
    ms.c = ms.b;
    if (vel_tma) {
      using VG = SplitVelTma<T>;
      if ((rc = encode_map(&mv.a, a.sxx, e, c.nx, c.nz, 1, 0, VG::WX, VG::TZ, 1))) return rc;
      if ((rc = encode_map(&mv.b, a.sxz, e, c.nx, c.nz, 1, 0, VG::WX, VG::HZ, 1))) return rc;
      if ((rc = encode_map(&mv.c, a.szz, e, c.nx, c.nz, 1, 0, VG::WZ, VG::HZ, 1))) return rc;
    }
  }
  FusedExtras<T> x;
  x.ntx = ntx;
  x.fs = c.free_surface;
  x.tile_off = d_off;
  x.tile_ent = d_ent;
  x.amp = (const T *)p->damp;
  x.wavelet = (s && s->nsrc) ? (const T *)s->wavelet_dev : nullptr;
  x.wnt = (s && s->nsrc) ? s->wavelet_nt : 0;
  x.traces = (s && s->nrec) ? (T *)s->traces_dev : nullptr;
  x.tnt = (s && s->nrec) ? s->traces_nt : 0;
  x.nrec = s ? s->nrec : 0;
  x.err = (int *)p->errflag;
  x.l2hint = l2_hints_fit(5LL * c.nx * c.nz * (long long)sizeof(T), p->l2_bytes);
  // ISO/VTI: in place on the current psi set; TTI: from the current set
  // to the other one, every step
  T *psix0 = a.psix ? (T *)p->psix : nullptr, *psiz0 = a.psiz ? (T *)p->psiz : nullptr;
  auto bind_psi = [&](int cur, int out) {
    if (psix0) {
      a.psix = psix0 + cur * kPsiPerSet * p->psix_plane;
      a.psix_o = psix0 + out * kPsiPerSet * p->psix_plane;
    }
    if (psiz0) {
      a.psiz = psiz0 + cur * kPsiPerSet * p->psiz_plane;
      a.psiz_o = psiz0 + out * kPsiPerSet * p->psiz_plane;
    }
  };
  if (!tti) bind_psi(p->psi_cur, p->psi_cur);
  const int ntiles = ntx * ntz, sntiles = sntx * sntz;
  FusedExtras<T> xs = x;
  xs.ntx = sntx;
  xs.tile_off = d_off + nvoff;
  for (int k = 0; k < nsteps; ++k) {
    x.it = xs.it = it0 + k;
    if (pipelined) {
      if ((rc = launch_split_vel_p<T>(a, x, pv, ntiles, p->nsm, st))) return rc;
      if ((rc = launch_split_stress_p<T>(c.medium, a, xs, ps, sntiles, p->nsm, st))) return rc;
    } else if (tti) {
      const bool from_user = k % 2 == 0;
      if (alt_m) {
        a.m = from_user ? user_m : alt_m;
        a.mstride = from_user ? user_ms : (long long)np;
        a.m_o = from_user ? alt_m : user_m;
        a.mstride_o = from_user ? (long long)np : user_ms;
      }
      const int cur = p->psi_cur;
      bind_psi(cur, 1 - cur);
      if ((rc = vel_tma ? launch_vel_tma<T>(a, x, mv, ntiles, st, k > 0)
                        : launch_split_vel<T>(a, x, ntiles, st, k > 0)))
        return rc;
      if ((rc = launch_split_stress_tti<T>(a, xs, ms, sntiles, st, true))) return rc;
      p->psi_cur = 1 - cur;
    } else {
      // the first kernel of the call starts after everything before it in
      // the stream; the others overlap the tail of their predecessor
      if ((rc = vel_tma ? launch_vel_tma<T>(a, x, mv, ntiles, st, k > 0)
                        : launch_split_vel<T>(a, x, ntiles, st, k > 0)))
        return rc;
      if ((rc = launch_split_stress<T>(c.medium, a, xs, ms, sntiles, st, true))) return rc;
    }
  }
  if (alt_m && nsteps % 2 == 1) {
    // the memory variables sit in the plan's copy: bring them back
    for (int q = 0; q < 3 * c.nsls; ++q) {
      rc = cuda_check(cudaMemcpyAsync(user_m + q * user_ms, alt_m + q * np, np * sizeof(T),
                                      cudaMemcpyDeviceToDevice, st),
                      "copy back memory variables");
      if (rc) return rc;
    }
  }
  return VI_OK;
}

template bool split_eligible<float>(const vi_plan *, const StepArgs<float> &);
template bool split_eligible<double>(const vi_plan *, const StepArgs<double> &);
template int split_steps<float>(vi_plan *, StepArgs<float>, const vi_shot *, int, int, cudaStream_t,
                                int);
template int split_steps<double>(vi_plan *, StepArgs<double>, const vi_shot *, int, int,
                                 cudaStream_t, int);

template int launch_split_vel_batch<float>(int, bool, const BatchDev<float> &, int, int, cudaStream_t, bool);
template int launch_split_vel_batch<double>(int, bool, const BatchDev<double> &, int, int, cudaStream_t,
                                            bool);
template int launch_split_stress_batch<float>(int, int, bool, bool, const BatchDev<float> &, int, int,
                                              cudaStream_t, bool);
template int launch_split_stress_batch<double>(int, int, bool, bool, const BatchDev<double> &, int, int,
                                               cudaStream_t, bool);
template int launch_split_vel<float>(const StepArgs<float> &, const FusedExtras<float> &, int,
                                     cudaStream_t, bool);
template int launch_split_vel<double>(const StepArgs<double> &, const FusedExtras<double> &, int,
                                      cudaStream_t, bool);
template int launch_split_stress<float>(int, const StepArgs<float> &, const FusedExtras<float> &,
                                        const SplitMaps &, int, cudaStream_t, bool);
template int launch_split_stress<double>(int, const StepArgs<double> &, const FusedExtras<double> &,
                                         const SplitMaps &, int, cudaStream_t, bool);

}  // namespace vb
