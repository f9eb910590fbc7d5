// split_p.cu — persistent, TMA-pipelined forms of the split step kernels.
//
// Each CTA walks tiles round-robin.  One elected thread keeps STAGES tiles'
// operand boxes in flight (every operand of a tile, halos included, is a
// TMA box); the CTA computes one staged tile while the next ones land, then
// refills the freed stage.  Compared with the one-tile-per-CTA split
// kernels, the HBM traffic is the same but no CTA ever waits on a load it
// has just issued.
//
//   velocity: 64 x 16 tiles, 4-cell groups, 256 threads, 3 stages (FP32)
//   stress:   64 x 8 tiles, 2-cell groups, 256 threads, 2 stages
#include <atomic>
#include <cudaTypedefs.h>

#include <cstdint>
#include <vector>

#include "fused_tma.cuh"
#include "plan.cuh"
#include "split.cuh"
#include "tma.cuh"
#include "vec.cuh"

namespace vb {

template <typename T>
constexpr int rnd128(int n) {
  return (int)(((long long)n * (long long)sizeof(T) + 127) / 128 * 128 / (long long)sizeof(T));
}

template <typename T>
struct VelP {
  static constexpr int TX = 64, TZ = 16, NT = 256, STAGES = sizeof(T) == 4 ? 3 : 2;
  static constexpr int BW = TX + 8, BH = TZ + 8;        // sigma box (4-cell halo)
  static constexpr int RW = TX + 4, RH = TZ + 1;        // rho box (+1 neighbours)
  static constexpr int PS = rnd128<T>(BW * BH), PV = rnd128<T>(TX * TZ), PR = rnd128<T>(RW * RH);
  static constexpr int S_SXX = 0, S_SZZ = PS, S_SXZ = 2 * PS, S_VX = 3 * PS, S_VZ = 3 * PS + PV,
                       S_RHO = 3 * PS + 2 * PV, STAGE = S_RHO + PR;
  static constexpr int O_STAGE = 128 / (int)sizeof(T);
  static constexpr int BYTES = (O_STAGE + STAGES * STAGE) * (int)sizeof(T);
  static constexpr int TXB = (int)sizeof(T) * (3 * BW * BH + 2 * TX * TZ + RW * RH);
};

template <typename T, int KIND, int NSLS>
struct StressP {
  static constexpr int TX = 64, TZ = 8, W = 2, NT = (TX / W) * TZ, STAGES = 2;
  static constexpr int NM = 3 * NSLS;
  static constexpr int NC = (KIND == VI_MEDIUM_ISO ? 2 : 4) + (NSLS > 0 ? 1 : 0);  // + tau
  static constexpr int BW = TX + 8, BH = TZ + 8;  // velocity box (4-cell halo)
  static constexpr int CW = TX + 4, CH = TZ + 1;  // coefficient boxes (+1 neighbours)
  static constexpr int PV = rnd128<T>(BW * BH), PT = rnd128<T>(TX * TZ), PC = rnd128<T>(CW * CH);
  static constexpr int PM = rnd128<T>(TX * TZ * (NM > 0 ? NM : 1));
  static constexpr int S_VX = 0, S_VZ = PV, S_SXX = 2 * PV, S_SZZ = 2 * PV + PT,
                       S_SXZ = 2 * PV + 2 * PT, S_M = 2 * PV + 3 * PT,
                       S_C = S_M + (NSLS > 0 ? PM : 0), STAGE = S_C + NC * PC;
  static constexpr int O_STAGE = 128 / (int)sizeof(T);
  static constexpr int BYTES = (O_STAGE + STAGES * STAGE) * (int)sizeof(T);
  static constexpr int TXB =
      (int)sizeof(T) * (2 * BW * BH + 3 * TX * TZ + (NSLS > 0 ? TX * TZ * NM : 0) + NC * CW * CH);
  static constexpr bool FITS = BYTES <= kSmemLimit;
};

// Runs the persistent tile loop: issue(stage, tile) queues a tile's boxes,
// compute(stage, tile) works on a landed stage.  Bounded waits: a stage that
// never lands sets the error word and ends the CTA after a bounded drain.
template <int STAGES, typename Issue, typename Compute>
__device__ __forceinline__ void tile_pipeline(uint64_t *bars, int ntiles, int *err, Issue issue,
                                              Compute compute) {
  const int tid = threadIdx.x, G0 = gridDim.x;
  if (tid == 0)
    for (int s = 0; s < STAGES; ++s) mbar_init(&bars[s], 1);
  __syncthreads();
  if (tid == 0)
    for (int s = 0; s < STAGES; ++s)
      if (blockIdx.x + s * G0 < ntiles) issue(s, blockIdx.x + s * G0, &bars[s]);
  int j = 0;
  for (int tile = blockIdx.x; tile < ntiles; tile += G0, ++j) {
    const int s = j % STAGES;
    const uint32_t parity = (j / STAGES) & 1;
    const bool ok = mbar_wait_bounded(&bars[s], parity, 1u << 22);
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {
        atomicExch(err, 1);
        for (int q = 0; q < STAGES; ++q) {  // drain what is still in flight
          const int jq = j + q;
          if (blockIdx.x + jq * G0 < ntiles)
            mbar_wait_bounded(&bars[jq % STAGES], (jq / STAGES) & 1, 1u << 22);
        }
      }
      return;
    }
    compute(s, tile);
    __syncthreads();  // every thread is done with stage s
    if (tid == 0) {
      const int nt = tile + STAGES * G0;
      if (nt < ntiles) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        issue(s, nt, &bars[s]);
      }
    }
  }
}

// ---------------------------------------------------------------- velocity
template <typename T>
__global__ void __launch_bounds__(VelP<T>::NT)
    k_split_vel_p(const StepArgs<T> a, const FusedExtras<T> x, const __grid_constant__ SplitPMaps maps,
                  int ntiles) {
  using G = VelP<T>;
  constexpr int TX = G::TX, TZ = G::TZ, BW = G::BW, RW = G::RW;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw);
  T *st0 = reinterpret_cast<T *>(smem_raw) + G::O_STAGE;
  const int nx = a.nx, nz = a.nz, xe = nx - L, ze = nz - L;
  const int tid = threadIdx.x;
  const int r = tid / (TX / 4), lx = 4 * (tid % (TX / 4));
  auto issue = [&](int s, int tile, uint64_t *bar) {
    const int x0 = L + (tile % x.ntx) * TX, z0 = L + (tile / x.ntx) * TZ;
    T *sb = st0 + s * G::STAGE;
    mbar_arrive_expect_tx(bar, G::TXB);
    tma_load_2d(sb + G::S_SXX, &maps.m[0], x0 - 4, z0 - 4, bar);
    tma_load_2d(sb + G::S_SZZ, &maps.m[1], x0 - 4, z0 - 4, bar);
    tma_load_2d(sb + G::S_SXZ, &maps.m[2], x0 - 4, z0 - 4, bar);
    tma_load_2d(sb + G::S_VX, &maps.m[3], x0, z0, bar);
    tma_load_2d(sb + G::S_VZ, &maps.m[4], x0, z0, bar);
    tma_load_2d(sb + G::S_RHO, &maps.m[5], x0, z0, bar);
  };
  auto compute = [&](int s, int tile) {
    const int x0 = L + (tile % x.ntx) * TX, z0 = L + (tile / x.ntx) * TZ;
    const int gi0 = x0 + lx, gj = z0 + r;
    if (gi0 >= xe || gj >= ze) return;
    const T *sb = st0 + s * G::STAGE;
    const T *s_sxx = sb + G::S_SXX, *s_szz = sb + G::S_SZZ, *s_sxz = sb + G::S_SXZ;
    const long long g = (long long)gj * nx + gi0;
    const int e0 = x.tile_off[tile], e1 = x.tile_off[tile + 1];
    const int bb = (r + 4) * BW + lx;  // box row of the cells; cells at box column lx+4
    T hxx[12], hxz[12];
    row12s(s_sxx + bb, hxx);
    row12s(s_sxz + bb, hxz);
    T zxz[4] = {0, 0, 0, 0}, zzz[4] = {0, 0, 0, 0};
#pragma unroll
    for (int q = -4; q <= 4; ++q) {
      if (q <= 3) {  // ddzm(sxz)
        const T cq = q >= 0 ? a.Dz[q] : -a.Dz[-q - 1];
        const Q4<T> v = q == 0 ? Q4<T>{{hxz[4], hxz[5], hxz[6], hxz[7]}} : lds4(s_sxz + bb + q * BW + 4);
#pragma unroll
        for (int k = 0; k < 4; ++k) zxz[k] += cq * v.v[k];
      }
      if (q >= -3) {  // ddzp(szz)
        const T cq = q >= 1 ? a.Dz[q - 1] : -a.Dz[-q];
        const Q4<T> v = lds4(s_szz + bb + q * BW + 4);
#pragma unroll
        for (int k = 0; k < 4; ++k) zzz[k] += cq * v.v[k];
      }
    }
    const Q4<T> vxi = lds4(sb + G::S_VX + r * TX + lx), vzi = lds4(sb + G::S_VZ + r * TX + lx);
    const Q4<T> r0 = lds4(sb + G::S_RHO + r * RW + lx), r1 = lds4(sb + G::S_RHO + (r + 1) * RW + lx);
    const T r4 = sb[G::S_RHO + r * RW + lx + 4];
    const int zs = strip_z(gj, nz, a.Tz, a.Bz);
    const bool xstrip = gi0 < a.Lx || gi0 + 3 >= nx - a.Rx;
    Q4<T> vxn, vzn;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int gi = gi0 + k;
      T dxx = dps(hxx, 4 + k, a.Dx), dxxz = dms(hxz, 4 + k, a.Dx);
      T dzxz = zxz[k], dzz = zzz[k];
      if (xstrip) {
        const int xs = strip_x(gi, nx, a.Lx, a.Rx);
        if (xs >= 0) {
          const T *tb = a.tx;
          const long long o = (long long)gj * a.wx + xs;
          T *p0 = a.psix + PX_SXX * a.psix_plane + o, *p1 = a.psix + PX_SXZ * a.psix_plane + o;
          *p0 = tb[T_BH * nx + gi] * *p0 + tb[T_AH * nx + gi] * dxx;
          *p1 = tb[T_B * nx + gi] * *p1 + tb[T_A * nx + gi] * dxxz;
          dxx = dxx * tb[T_IKH * nx + gi] + *p0;
          dxxz = dxxz * tb[T_IK * nx + gi] + *p1;
        }
      }
      if (zs >= 0) {
        const T *tb = a.tz;
        const long long o = (long long)zs * nx + gi;
        T *p0 = a.psiz + PZ_SXZ * a.psiz_plane + o, *p1 = a.psiz + PZ_SZZ * a.psiz_plane + o;
        *p0 = tb[T_B * nz + gj] * *p0 + tb[T_A * nz + gj] * dzxz;
        *p1 = tb[T_BH * nz + gj] * *p1 + tb[T_AH * nz + gj] * dzz;
        dzxz = dzxz * tb[T_IK * nz + gj] + *p0;
        dzz = dzz * tb[T_IKH * nz + gj] + *p1;
      }
      const T rx = k < 3 ? r0.v[k + 1] : r4;
      vxn.v[k] = vxi.v[k] + a.dt * two_over_fast(r0.v[k] + rx) * (dxx + dzxz);
      vzn.v[k] = vzi.v[k] + a.dt * two_over_fast(r0.v[k] + r1.v[k]) * (dxxz + dzz);
    }
    for (int e = e0; e < e1; ++e) {
      const int4 en = x.tile_ent[e];
      if ((en.w != TL_FORCE_X && en.w != TL_FORCE_Z) || en.y != gj || en.x < gi0 || en.x >= gi0 + 4)
        continue;
      const int k = en.x - gi0;
      const T w = x.it < x.wnt ? x.wavelet[(long long)en.z * x.wnt + x.it] : T(0);
      const T f = x.amp[en.z] * w;
      if (en.w == TL_FORCE_X)
        add_lane4(vxn, k, a.dt * two_over_fast(lane4(r0, k) + (k < 3 ? lane4(r0, k + 1) : r4)) * f);
      else
        add_lane4(vzn, k, a.dt * two_over_fast(lane4(r0, k) + lane4(r1, k)) * f);
    }
    stg4(a.vx + g, vxn);
    stg4(a.vz + g, vzn);
    if (x.traces && x.it < x.tnt) {
      for (int e = e0; e < e1; ++e) {
        const int4 en = x.tile_ent[e];
        if (en.w != TL_RECEIVER || en.y != gj || en.x < gi0 || en.x >= gi0 + 4) continue;
        x.traces[(long long)en.z * x.tnt + x.it] = lane4(vxn, en.x - gi0);
        x.traces[(long long)(x.nrec + en.z) * x.tnt + x.it] = lane4(vzn, en.x - gi0);
      }
    }
  };
  tile_pipeline<G::STAGES>(bars, ntiles, x.err, issue, compute);
}

// ------------------------------------------------------------------ stress
template <typename T, int KIND, int NSLS>
__global__ void __launch_bounds__(StressP<T, KIND, NSLS>::NT)
    k_split_stress_p(const StepArgs<T> a, const FusedExtras<T> x,
                     const __grid_constant__ SplitPMaps maps, int ntiles) {
  using G = StressP<T, KIND, NSLS>;
  constexpr int TX = G::TX, TZ = G::TZ, W = G::W, BW = G::BW, CW = G::CW, PC = G::PC;
  constexpr int C11 = 0;
  constexpr int C13 = KIND == VI_MEDIUM_ISO ? 0 : 1;
  constexpr int C33 = 2;
  constexpr int C55 = KIND == VI_MEDIUM_ISO ? 1 : 3;
  constexpr int CTAU = G::NC - 1;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw);
  T *st0 = reinterpret_cast<T *>(smem_raw) + G::O_STAGE;
  const int nx = a.nx, nz = a.nz, xe = nx - L, ze = nz - L;
  const int tid = threadIdx.x;
  const int r = tid / (TX / W), lx = W * (tid % (TX / W));
  auto issue = [&](int s, int tile, uint64_t *bar) {
    const int x0 = L + (tile % x.ntx) * TX, z0 = L + (tile / x.ntx) * TZ;
    T *sb = st0 + s * G::STAGE;
    mbar_arrive_expect_tx(bar, G::TXB);
    tma_load_2d(sb + G::S_VX, &maps.m[0], x0 - 4, z0 - 4, bar);
    tma_load_2d(sb + G::S_VZ, &maps.m[1], x0 - 4, z0 - 4, bar);
    tma_load_2d(sb + G::S_SXX, &maps.m[2], x0, z0, bar);
    tma_load_2d(sb + G::S_SZZ, &maps.m[3], x0, z0, bar);
    tma_load_2d(sb + G::S_SXZ, &maps.m[4], x0, z0, bar);
    if constexpr (NSLS > 0) tma_load_3d(sb + G::S_M, &maps.m[5], x0, z0, 0, bar);
#pragma unroll
    for (int c = 0; c < G::NC; ++c) tma_load_2d(sb + G::S_C + c * PC, &maps.m[6 + c], x0, z0, bar);
  };
  auto compute = [&](int s, int tile) {
    const int x0 = L + (tile % x.ntx) * TX, z0 = L + (tile / x.ntx) * TZ;
    const int gi0 = x0 + lx, gj = z0 + r;
    if (gi0 >= xe || gj >= ze) return;
    const T *sb = st0 + s * G::STAGE;
    const T *s_vx = sb + G::S_VX, *s_vz = sb + G::S_VZ;
    const long long g = (long long)gj * nx + gi0;
    const int e0 = x.tile_off[tile], e1 = x.tile_off[tile + 1];
    // strain rates of the W cells (cells at velocity-box column lx+4)
    const int vb = (r + 4) * BW + lx;
    T hvx[W + 8], hvz[W + 8];
#pragma unroll
    for (int q = 0; q < (W + 8) / 2; ++q) {
      const Q2<T> u = lds2(s_vx + vb + 2 * q), w = lds2(s_vz + vb + 2 * q);
      hvx[2 * q] = u.v[0];
      hvx[2 * q + 1] = u.v[1];
      hvz[2 * q] = w.v[0];
      hvz[2 * q + 1] = w.v[1];
    }
    T zvz[W] = {0, 0}, zvx[W] = {0, 0};
#pragma unroll
    for (int q = -4; q <= 4; ++q) {
      if (q <= 3) {  // ddzm(vz)
        const T cq = q >= 0 ? a.Dz[q] : -a.Dz[-q - 1];
        const Q2<T> v = q == 0 ? Q2<T>{{hvz[4], hvz[5]}} : lds2(s_vz + vb + q * BW + 4);
        zvz[0] += cq * v.v[0];
        zvz[1] += cq * v.v[1];
      }
      if (q >= -3) {  // ddzp(vx)
        const T cq = q >= 1 ? a.Dz[q - 1] : -a.Dz[-q];
        const Q2<T> v = q == 0 ? Q2<T>{{hvx[4], hvx[5]}} : lds2(s_vx + vb + q * BW + 4);
        zvx[0] += cq * v.v[0];
        zvx[1] += cq * v.v[1];
      }
    }
    const int zs = strip_z(gj, nz, a.Tz, a.Bz);
    const bool xstrip = gi0 < a.Lx || gi0 + W - 1 >= nx - a.Rx;
    const bool surf = x.fs && gj == L;
    T rxx[W], rzz[W], rxz[W];
#pragma unroll
    for (int k = 0; k < W; ++k) {
      const int gi = gi0 + k;
      const T *D = a.Dx;
      const int c = 4 + k;
      T dxvx = D[0] * (hvx[c] - hvx[c - 1]) + D[1] * (hvx[c + 1] - hvx[c - 2]) +
               D[2] * (hvx[c + 2] - hvx[c - 3]) + D[3] * (hvx[c + 3] - hvx[c - 4]);
      T dxvz = D[0] * (hvz[c + 1] - hvz[c]) + D[1] * (hvz[c + 2] - hvz[c - 1]) +
               D[2] * (hvz[c + 3] - hvz[c - 2]) + D[3] * (hvz[c + 4] - hvz[c - 3]);
      T dzvz = zvz[k], dzvx = zvx[k];
      if (xstrip) {
        const int xs = strip_x(gi, nx, a.Lx, a.Rx);
        if (xs >= 0) {
          const T *tb = a.tx;
          const long long o = (long long)gj * a.wx + xs;
          T *p0 = a.psix + PX_VX * a.psix_plane + o, *p1 = a.psix + PX_VZ * a.psix_plane + o;
          *p0 = tb[T_B * nx + gi] * *p0 + tb[T_A * nx + gi] * dxvx;
          *p1 = tb[T_BH * nx + gi] * *p1 + tb[T_AH * nx + gi] * dxvz;
          dxvx = dxvx * tb[T_IK * nx + gi] + *p0;
          dxvz = dxvz * tb[T_IKH * nx + gi] + *p1;
        }
      }
      if (zs >= 0) {
        const T *tb = a.tz;
        const long long o = (long long)zs * nx + gi;
        T *p0 = a.psiz + PZ_VZ * a.psiz_plane + o, *p1 = a.psiz + PZ_VX * a.psiz_plane + o;
        *p0 = tb[T_B * nz + gj] * *p0 + tb[T_A * nz + gj] * dzvz;
        *p1 = tb[T_BH * nz + gj] * *p1 + tb[T_AH * nz + gj] * dzvx;
        dzvz = dzvz * tb[T_IK * nz + gj] + *p0;
        dzvx = dzvx * tb[T_IKH * nz + gj] + *p1;
      }
      rxx[k] = dxvx;
      rzz[k] = dzvz;
      rxz[k] = dzvx + dxvz;
    }
    // staged own-cell operands
    const int ti = r * TX + lx, ci = r * CW + lx;
    Q2<T> sxx = lds2(sb + G::S_SXX + ti), szz = lds2(sb + G::S_SZZ + ti), sxz = lds2(sb + G::S_SXZ + ti);
    const T *cb = sb + G::S_C;
    const Q2<T> c13 = lds2(cb + C13 * PC + ci);
    const Q2<T> c55a = lds2(cb + C55 * PC + ci), c55b = lds2(cb + C55 * PC + ci + CW);
    const T c55a2 = cb[C55 * PC + ci + W], c55b2 = cb[C55 * PC + ci + CW + W];
    Q2<T> c11, c33, tau;
    if constexpr (KIND != VI_MEDIUM_ISO) {
      c11 = lds2(cb + C11 * PC + ci);
      c33 = lds2(cb + C33 * PC + ci);
    } else {
      c11.v[0] = c33.v[0] = c13.v[0] + T(2) * c55a.v[0];
      c11.v[1] = c33.v[1] = c13.v[1] + T(2) * c55a.v[1];
    }
    if constexpr (NSLS > 0) tau = lds2(cb + CTAU * PC + ci);
    Q2<T> m[NSLS > 0 ? 3 * NSLS : 1];
    if constexpr (NSLS > 0) {
#pragma unroll
      for (int q = 0; q < 3 * NSLS; ++q) m[q] = lds2(sb + G::S_M + q * (TX * TZ) + ti);
    }
    const T dt = a.dt;
#pragma unroll
    for (int k = 0; k < W; ++k) {
      T exx = rxx[k], ezz = rzz[k], exz = rxz[k];
      if constexpr (NSLS > 0) {
        T Sxx = 0, Szz = 0, Sxz = 0;
#pragma unroll
        for (int n = 0; n < NSLS; ++n) {
          Sxx += m[0 * NSLS + n].v[k];
          Szz += m[1 * NSLS + n].v[k];
          Sxz += m[2 * NSLS + n].v[k];
        }
        const T t = tau.v[k], t1 = T(1) + t;
        exx = t1 * rxx[k] + t * Sxx;
        ezz = t1 * rzz[k] + t * Szz;
        exz = t1 * rxz[k] + t * Sxz;
      }
      if (surf) ezz = -(c13.v[k] * exx) / c33.v[k];
      const T c55r = k < W - 1 ? c55a.v[k + 1] : c55a2, c55br = k < W - 1 ? c55b.v[k + 1] : c55b2;
      const T C55h = T(0.25) * (c55a.v[k] + c55r + c55b.v[k] + c55br);
      sxx.v[k] += dt * (c11.v[k] * exx + c13.v[k] * ezz);
      szz.v[k] += dt * (c13.v[k] * exx + c33.v[k] * ezz);
      sxz.v[k] += dt * (C55h * exz);
    }
    if constexpr (NSLS > 0) {
#pragma unroll
      for (int n = 0; n < NSLS; ++n) {
        const T a1 = a.a1[n], a2 = a.a2[n];
#pragma unroll
        for (int k = 0; k < W; ++k) {
          m[0 * NSLS + n].v[k] += dt * (a1 * rxx[k] + a2 * m[0 * NSLS + n].v[k]);
          m[1 * NSLS + n].v[k] =
              surf ? T(0) : m[1 * NSLS + n].v[k] + dt * (a1 * rzz[k] + a2 * m[1 * NSLS + n].v[k]);
          m[2 * NSLS + n].v[k] += dt * (a1 * rxz[k] + a2 * m[2 * NSLS + n].v[k]);
        }
      }
#pragma unroll
      for (int q = 0; q < 3 * NSLS; ++q) stg2(a.m + q * a.mstride + g, m[q]);
    }
    for (int e = e0; e < e1; ++e) {
      const int4 en = x.tile_ent[e];
      if (en.w != TL_EXPLOSIVE || en.y != gj || en.x < gi0 || en.x >= gi0 + W) continue;
      const T w = x.it < x.wnt ? x.wavelet[(long long)en.z * x.wnt + x.it] : T(0);
      add_lane2(sxx, en.x - gi0, dt * x.amp[en.z] * w);
      add_lane2(szz, en.x - gi0, dt * x.amp[en.z] * w);
    }
    if (surf) szz = Q2<T>{{0, 0}};
    stg2(a.sxx + g, sxx);
    stg2(a.szz + g, szz);
    stg2(a.sxz + g, sxz);
    if (x.fs) {
      // stress images: szz(L-k) = -szz(L+k), k = 1..4; sxz(L-1-k) = -sxz(L+k), k = 0..3
      const int k = gj - L;
      if (k >= 1 && k <= L) stg2(a.szz + (long long)(L - k) * nx + gi0, Q2<T>{{-szz.v[0], -szz.v[1]}});
      if (k >= 0 && k < L) stg2(a.sxz + (long long)(L - 1 - k) * nx + gi0, Q2<T>{{-sxz.v[0], -sxz.v[1]}});
    }
  };
  tile_pipeline<G::STAGES>(bars, ntiles, x.err, issue, compute);
}

// ------------------------------------------------------------------- host
template <typename K>
static int set_smem(K kern, int bytes, std::atomic<unsigned long long> &done) {
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && !(done.load() & (1ULL << dev))) {  // one bit per device set up (any thread)
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return cuda_check(e, "split pipeline smem attribute");
    done |= 1ULL << dev;
  }
  return VI_OK;
}

template <typename K>
static int persistent_grid(K kern, int nt, int bytes, int nsm, int ntiles) {
  int per = 1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, nt, bytes) != cudaSuccess || per < 1) {
    cudaGetLastError();
    per = 1;
  }
  const int g = per * nsm;
  return ntiles < g ? ntiles : g;
}

template <typename T, int KIND, int NSLS>
static int launch_stress_p(const StepArgs<T> &a, const FusedExtras<T> &x, const SplitPMaps &m,
                           int ntiles, int nsm, cudaStream_t st) {
  using G = StressP<T, KIND, NSLS>;
  if constexpr (!G::FITS) {
    return set_error(VI_ERR_ARG, "pipelined stress kernel does not fit shared memory");
  } else {
    static std::atomic<unsigned long long> done{0};
    int rc = set_smem(k_split_stress_p<T, KIND, NSLS>, G::BYTES, done);
    if (rc) return rc;
    const int grid = persistent_grid(k_split_stress_p<T, KIND, NSLS>, G::NT, G::BYTES, nsm, ntiles);
    k_split_stress_p<T, KIND, NSLS><<<grid, G::NT, G::BYTES, st>>>(a, x, m, ntiles);
    return VI_OK;
  }
}

template <typename T>
int launch_split_vel_p(const StepArgs<T> &a, const FusedExtras<T> &x, const SplitPMaps &m,
                       int ntiles, int nsm, cudaStream_t st) {
  using G = VelP<T>;
  static std::atomic<unsigned long long> done{0};
  int rc = set_smem(k_split_vel_p<T>, G::BYTES, done);
  if (rc) return rc;
  const int grid = persistent_grid(k_split_vel_p<T>, G::NT, G::BYTES, nsm, ntiles);
  k_split_vel_p<T><<<grid, G::NT, G::BYTES, st>>>(a, x, m, ntiles);
  return VI_OK;
}

template <typename T>
int launch_split_stress_p(int kind, const StepArgs<T> &a, const FusedExtras<T> &x,
                          const SplitPMaps &m, int ntiles, int nsm, cudaStream_t st) {
#define VB_CASE(K, N) \
  if (kind == K && a.nsls == N) return launch_stress_p<T, K, N>(a, x, m, ntiles, nsm, st);
#define VB_KIND(K) VB_CASE(K, 0) VB_CASE(K, 1) VB_CASE(K, 2) VB_CASE(K, 3) VB_CASE(K, 4) VB_CASE(K, 5)
  VB_KIND(VI_MEDIUM_ISO)
  VB_KIND(VI_MEDIUM_VTI)
#undef VB_KIND
#undef VB_CASE
  return set_error(VI_ERR_ARG, "the split step covers ISO and VTI media");
}

bool split_p_fits(int kind, int nsls, int esize) {
#define VB_F(K, N) \
  if (kind == K && nsls == N) return esize == 4 ? StressP<float, K, N>::FITS : StressP<double, K, N>::FITS;
#define VB_K(K) VB_F(K, 0) VB_F(K, 1) VB_F(K, 2) VB_F(K, 3) VB_F(K, 4) VB_F(K, 5)
  VB_K(VI_MEDIUM_ISO)
  VB_K(VI_MEDIUM_VTI)
#undef VB_K
#undef VB_F
  return false;
}

// Tensor maps of the pipelined kernels for the caller's (in-place) state.
template <typename T>
int encode_split_p(const vi_config &c, const StepArgs<T> &a, SplitPMaps &mv, SplitPMaps &ms) {
  const int e = sizeof(T), nx = c.nx, nz = c.nz;
  using V = VelP<T>;
  int rc;
  if ((rc = encode_map(&mv.m[0], a.sxx, e, nx, nz, 1, 0, V::BW, V::BH, 1))) return rc;
  if ((rc = encode_map(&mv.m[1], a.szz, e, nx, nz, 1, 0, V::BW, V::BH, 1))) return rc;
  if ((rc = encode_map(&mv.m[2], a.sxz, e, nx, nz, 1, 0, V::BW, V::BH, 1))) return rc;
  if ((rc = encode_map(&mv.m[3], a.vx, e, nx, nz, 1, 0, V::TX, V::TZ, 1))) return rc;
  if ((rc = encode_map(&mv.m[4], a.vz, e, nx, nz, 1, 0, V::TX, V::TZ, 1))) return rc;
  if ((rc = encode_map(&mv.m[5], a.rho, e, nx, nz, 1, 0, V::RW, V::RH, 1))) return rc;
  // stress (geometry is the same for every medium kind)
  using S = StressP<T, VI_MEDIUM_VTI, 1>;
  if ((rc = encode_map(&ms.m[0], a.vx, e, nx, nz, 1, 0, S::BW, S::BH, 1))) return rc;
  if ((rc = encode_map(&ms.m[1], a.vz, e, nx, nz, 1, 0, S::BW, S::BH, 1))) return rc;
  if ((rc = encode_map(&ms.m[2], a.sxx, e, nx, nz, 1, 0, S::TX, S::TZ, 1))) return rc;
  if ((rc = encode_map(&ms.m[3], a.szz, e, nx, nz, 1, 0, S::TX, S::TZ, 1))) return rc;
  if ((rc = encode_map(&ms.m[4], a.sxz, e, nx, nz, 1, 0, S::TX, S::TZ, 1))) return rc;
  if (c.nsls > 0 &&
      (rc = encode_map(&ms.m[5], a.m, e, nx, nz, 3 * c.nsls, a.mstride, S::TX, S::TZ, 3 * c.nsls)))
    return rc;
  const T *slots[5];
  int n = 0;
  if (c.medium == VI_MEDIUM_ISO) {
    slots[n++] = a.c13;
    slots[n++] = a.c55;
  } else {
    slots[n++] = a.c11;
    slots[n++] = a.c13;
    slots[n++] = a.c33;
    slots[n++] = a.c55;
  }
  if (c.nsls > 0) slots[n++] = a.tau;
  for (int k = 0; k < n; ++k)
    if ((rc = encode_map(&ms.m[6 + k], slots[k], e, nx, nz, 1, 0, S::CW, S::CH, 1))) return rc;
  return VI_OK;
}

void split_p_tiles(int &vtx, int &vtz, int &stx, int &stz) {
  vtx = VelP<float>::TX;
  vtz = VelP<float>::TZ;
  stx = StressP<float, VI_MEDIUM_VTI, 1>::TX;
  stz = StressP<float, VI_MEDIUM_VTI, 1>::TZ;
}

template int launch_split_vel_p<float>(const StepArgs<float> &, const FusedExtras<float> &,
                                       const SplitPMaps &, int, int, cudaStream_t);
template int launch_split_vel_p<double>(const StepArgs<double> &, const FusedExtras<double> &,
                                        const SplitPMaps &, int, int, cudaStream_t);
template int launch_split_stress_p<float>(int, const StepArgs<float> &, const FusedExtras<float> &,
                                          const SplitPMaps &, int, int, cudaStream_t);
template int launch_split_stress_p<double>(int, const StepArgs<double> &, const FusedExtras<double> &,
                                           const SplitPMaps &, int, int, cudaStream_t);
template int encode_split_p<float>(const vi_config &, const StepArgs<float> &, SplitPMaps &, SplitPMaps &);
template int encode_split_p<double>(const vi_config &, const StepArgs<double> &, SplitPMaps &, SplitPMaps &);

}  // namespace vb
