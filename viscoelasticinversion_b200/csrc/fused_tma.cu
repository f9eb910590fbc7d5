// fused_tma.cu — the fused step with every operand of a tile staged in
// shared memory by TMA (cp.async.bulk.tensor) before any arithmetic.
//
// One elected thread issues all boxes of the tile (stresses + 8-cell halo,
// velocities + 4-cell halo, density, memory variables, stiffness, τ) on one
// mbarrier; the CTA then computes the velocity stage on the tile + halo and
// the SLS stress stage on the tile entirely from shared memory.  Only the
// CPML ψ strips, the per-tile source/receiver lists and the outputs touch
// global memory during compute.  Two CTAs fit per SM (FP32 ISO/VTI), so one
// CTA's loads overlap the other's arithmetic.
#include <cudaTypedefs.h>

#include "fused_tma.cuh"
#include "plan.cuh"
#include "tma.cuh"

namespace vb {

template <typename T, int KIND, int NSLS>
__global__ void __launch_bounds__(256) k_fused_tma(const StepArgs<T> a, const FusedExtras<T> x,
                                                   const __grid_constant__ TmaMaps maps) {
  using G = typename TmaPick<T, KIND, NSLS>::Lay;
  constexpr int TX = G::TX, TZ = G::TZ, NT = G::NT, HV = G::HV, HS = G::HS, HVP = G::HVP,
                HSP = G::HSP, SWp = G::SWp, VWp = G::VWp, VW = G::VW, VH = G::VH, RWp = G::RWp,
                MW = G::MW, MH = G::MH, CW = G::CW, EW = G::EW, EH = G::EH, PC = G::PC;
  constexpr bool TTI = G::TTI;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem_raw);
  T *sm = reinterpret_cast<T *>(smem_raw);
  T *s_sxx = sm + G::O_SXX, *s_szz = sm + G::O_SZZ, *s_sxz = sm + G::O_SXZ;
  T *s_vx = sm + G::O_VX, *s_vz = sm + G::O_VZ, *s_rho = sm + G::O_RHO;
  T *s_m = sm + G::O_M, *s_c = sm + G::O_C, *s_tau = sm + G::O_TAU;
  T *s_exx = sm + G::O_E, *s_ezz = s_exx + G::PE, *s_exz = s_ezz + G::PE;
  // coefficient slots
  constexpr int C11 = 0;
  constexpr int C13 = KIND == VI_MEDIUM_ISO ? 0 : 1;
  constexpr int C15 = 2;
  constexpr int C33 = KIND == VI_MEDIUM_VTI ? 2 : 3;
  constexpr int C35 = 4;
  constexpr int C55 = KIND == VI_MEDIUM_ISO ? 1 : (KIND == VI_MEDIUM_VTI ? 3 : 5);

  const int tile = blockIdx.x;
  const int x0 = L + (tile % x.ntx) * TX;
  const int z0 = L + (tile / x.ntx) * TZ;
  const int nx = a.nx, nz = a.nz;
  const int xe = nx - L, ze = nz - L;
  const int tid = threadIdx.x;
  const T dt = a.dt;

  // ---- 0. stage the tile ------------------------------------------------
  if (tid == 0) mbar_init(bar, 1);
  __syncthreads();
  if (tid == 0) {
    mbar_arrive_expect_tx(bar, G::TX_BYTES);
    tma_load_2d(s_sxx, &maps.sxx, x0 - HSP, z0 - HS, bar);
    tma_load_2d(s_szz, &maps.szz, x0 - HSP, z0 - HS, bar);
    tma_load_2d(s_sxz, &maps.sxz, x0 - HSP, z0 - HS, bar);
    tma_load_2d(s_vx, &maps.vx, x0 - HVP, z0 - HV, bar);
    tma_load_2d(s_vz, &maps.vz, x0 - HVP, z0 - HV, bar);
    tma_load_2d(s_rho, &maps.rho, x0 - HVP, z0 - HV, bar);
    if constexpr (NSLS > 0) {
      tma_load_3d(s_m, &maps.m, x0 + G::MX0, z0 + G::MZ0, 0, bar);
      if constexpr (TTI)
        tma_load_2d(s_tau, &maps.tau, x0 + G::MX0, z0 + G::MZ0, bar);
      else
        tma_load_2d(s_tau, &maps.tau, x0, z0, bar);
    }
#pragma unroll
    for (int c = 0; c < G::NC; ++c) tma_load_2d(s_c + c * PC, &maps.c[c], x0, z0, bar);
  }
  const bool ok = mbar_wait_bounded(bar, 0, 1u << 22);
  if (__syncthreads_or(!ok)) {
    // the staging never completed: report, give the copies a bounded chance
    // to land, and leave this tile untouched
    if (tid == 0) {
      atomicExch(x.err, 1);
      mbar_wait_bounded(bar, 0, 1u << 22);
    }
    return;
  }

  // ---- 1. new velocities on the tile + HV halo --------------------------
  for (int idx = tid; idx < VW * VH; idx += NT) {
    const int lz = idx / VW, lx = idx - lz * VW;
    const int gi = x0 - HV + lx, gj = z0 - HV + lz;
    const int sv = lz * VWp + lx + (HVP - HV);
    T vxn = 0, vzn = 0;
    if (gi >= L && gi < xe && gj >= L && gj < ze) {
      const int si = (lz + HS - HV) * SWp + lx + (HSP - HV);
      T dxx = 0, dzxz = 0, dxxz = 0, dzz = 0;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int l = k + 1;
        dxx += a.Dx[k] * (s_sxx[si + l] - s_sxx[si - l + 1]);
        dzxz += a.Dz[k] * (s_sxz[si + (l - 1) * SWp] - s_sxz[si - l * SWp]);
        dxxz += a.Dx[k] * (s_sxz[si + l - 1] - s_sxz[si - l]);
        dzz += a.Dz[k] * (s_szz[si + l * SWp] - s_szz[si - (l - 1) * SWp]);
      }
      const bool own = gi >= x0 && gi < x0 + TX && gj >= z0 && gj < z0 + TZ;
      const int xs = strip_x(gi, nx, a.Lx, a.Rx);
      if (xs >= 0) {
        const T *t = a.tx;
        const long long o = (long long)gj * a.wx + xs;
        const T p0 = t[T_BH * nx + gi] * a.psix[PX_SXX * a.psix_plane + o] + t[T_AH * nx + gi] * dxx;
        const T p1 = t[T_B * nx + gi] * a.psix[PX_SXZ * a.psix_plane + o] + t[T_A * nx + gi] * dxxz;
        if (own) {
          a.psix_o[PX_SXX * a.psix_plane + o] = p0;
          a.psix_o[PX_SXZ * a.psix_plane + o] = p1;
        }
        dxx = dxx * t[T_IKH * nx + gi] + p0;
        dxxz = dxxz * t[T_IK * nx + gi] + p1;
      }
      const int zs = strip_z(gj, nz, a.Tz, a.Bz);
      if (zs >= 0) {
        const T *t = a.tz;
        const long long o = (long long)zs * nx + gi;
        const T p0 = t[T_B * nz + gj] * a.psiz[PZ_SXZ * a.psiz_plane + o] + t[T_A * nz + gj] * dzxz;
        const T p1 = t[T_BH * nz + gj] * a.psiz[PZ_SZZ * a.psiz_plane + o] + t[T_AH * nz + gj] * dzz;
        if (own) {
          a.psiz_o[PZ_SXZ * a.psiz_plane + o] = p0;
          a.psiz_o[PZ_SZZ * a.psiz_plane + o] = p1;
        }
        dzxz = dzxz * t[T_IK * nz + gj] + p0;
        dzz = dzz * t[T_IKH * nz + gj] + p1;
      }
      const int ri = lz * RWp + lx + (HVP - HV);
      const T r0 = s_rho[ri];
      vxn = s_vx[sv] + dt * (T(2) / (r0 + s_rho[ri + 1])) * (dxx + dzxz);
      vzn = s_vz[sv] + dt * (T(2) / (r0 + s_rho[ri + RWp])) * (dxxz + dzz);
    }
    s_vx[sv] = vxn;
    s_vz[sv] = vzn;
  }
  __syncthreads();

  const int e0 = x.tile_off[tile], e1 = x.tile_off[tile + 1];
  if (e1 > e0) {
    // force sources (one thread: entries are few and may share a cell)
    if (tid == 0) {
      for (int e = e0; e < e1; ++e) {
        const int4 en = x.tile_ent[e];
        if (en.w != TL_FORCE_X && en.w != TL_FORCE_Z) continue;
        const int lx = en.x - (x0 - HV), lz = en.y - (z0 - HV);
        const int sv = lz * VWp + lx + (HVP - HV);
        const int ri = lz * RWp + lx + (HVP - HV);
        const T w = x.it < x.wnt ? x.wavelet[(long long)en.z * x.wnt + x.it] : T(0);
        const T f = x.amp[en.z] * w;
        if (en.w == TL_FORCE_X)
          s_vx[sv] += dt * (T(2) / (s_rho[ri] + s_rho[ri + 1])) * f;
        else
          s_vz[sv] += dt * (T(2) / (s_rho[ri] + s_rho[ri + RWp])) * f;
      }
    }
    __syncthreads();
  }

  // ---- 2. write the tile's velocities; receivers sample them -------------
#pragma unroll
  for (int k = 0; k < TX * TZ / NT; ++k) {
    const int lx = tid % TX, lz = tid / TX + k * (NT / TX);
    const int gi = x0 + lx, gj = z0 + lz;
    if (gi < xe && gj < ze) {
      const long long g = (long long)gj * nx + gi;
      const int sv = (lz + HV) * VWp + lx + HVP;
      a.vx_o[g] = s_vx[sv];
      a.vz_o[g] = s_vz[sv];
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

  // CPML-corrected strain rates at a cell whose velocity-tile index is sv
  auto rates = [&](int sv, int gi, int gj, bool own, T &rxx, T &rzz, T &rxz) {
    T dxvx = 0, dzvz = 0, dzvx = 0, dxvz = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int l = k + 1;
      dxvx += a.Dx[k] * (s_vx[sv + l - 1] - s_vx[sv - l]);
      dzvz += a.Dz[k] * (s_vz[sv + (l - 1) * VWp] - s_vz[sv - l * VWp]);
      dzvx += a.Dz[k] * (s_vx[sv + l * VWp] - s_vx[sv - (l - 1) * VWp]);
      dxvz += a.Dx[k] * (s_vz[sv + l] - s_vz[sv - l + 1]);
    }
    const int xs = strip_x(gi, nx, a.Lx, a.Rx);
    if (xs >= 0) {
      const T *t = a.tx;
      const long long o = (long long)gj * a.wx + xs;
      const T p0 = t[T_B * nx + gi] * a.psix[PX_VX * a.psix_plane + o] + t[T_A * nx + gi] * dxvx;
      const T p1 = t[T_BH * nx + gi] * a.psix[PX_VZ * a.psix_plane + o] + t[T_AH * nx + gi] * dxvz;
      if (own) {
        a.psix_o[PX_VX * a.psix_plane + o] = p0;
        a.psix_o[PX_VZ * a.psix_plane + o] = p1;
      }
      dxvx = dxvx * t[T_IK * nx + gi] + p0;
      dxvz = dxvz * t[T_IKH * nx + gi] + p1;
    }
    const int zs = strip_z(gj, nz, a.Tz, a.Bz);
    if (zs >= 0) {
      const T *t = a.tz;
      const long long o = (long long)zs * nx + gi;
      const T p0 = t[T_B * nz + gj] * a.psiz[PZ_VZ * a.psiz_plane + o] + t[T_A * nz + gj] * dzvz;
      const T p1 = t[T_BH * nz + gj] * a.psiz[PZ_VX * a.psiz_plane + o] + t[T_AH * nz + gj] * dzvx;
      if (own) {
        a.psiz_o[PZ_VZ * a.psiz_plane + o] = p0;
        a.psiz_o[PZ_VX * a.psiz_plane + o] = p1;
      }
      dzvz = dzvz * t[T_IK * nz + gj] + p0;
      dzvx = dzvx * t[T_IKH * nz + gj] + p1;
    }
    rxx = dxvx;
    rzz = dzvz;
    rxz = dzvx + dxvz;
  };
  // effective SLS rates from staged M (index mi in the M box) and tau
  auto effective = [&](int mi, T tau, T rxx, T rzz, T rxz, T &exx, T &ezz, T &exz) {
    if constexpr (NSLS > 0) {
      constexpr int MP = MW * MH;
      T Sxx = 0, Szz = 0, Sxz = 0;
#pragma unroll
      for (int n = 0; n < NSLS; ++n) {
        Sxx += s_m[(0 * NSLS + n) * MP + mi];
        Szz += s_m[(1 * NSLS + n) * MP + mi];
        Sxz += s_m[(2 * NSLS + n) * MP + mi];
      }
      const T t1 = T(1) + tau;
      exx = t1 * rxx + tau * Sxx;
      ezz = t1 * rzz + tau * Szz;
      exz = t1 * rxz + tau * Sxz;
    } else {
      exx = rxx;
      ezz = rzz;
      exz = rxz;
    }
  };

  // ---- 3. TTI: effective rates on the tile + 1 ring ---------------------
  if constexpr (TTI) {
    for (int idx = tid; idx < EW * EH; idx += NT) {
      const int lz = idx / EW, lx = idx - lz * EW;
      const int gi = x0 - 1 + lx, gj = z0 - 1 + lz;
      T exx = 0, ezz = 0, exz = 0;
      if (gi >= L && gi < xe && gj >= L && gj < ze) {
        const int sv = (lz - 1 + HV) * VWp + lx - 1 + HVP;
        const int mi = lz * MW + lx + 3;  // ring box origin (x0 - 4, z0 - 1)
        T rxx, rzz, rxz;
        rates(sv, gi, gj, false, rxx, rzz, rxz);
        effective(mi, NSLS > 0 ? s_tau[mi] : T(0), rxx, rzz, rxz, exx, ezz, exz);
      }
      s_exx[idx] = exx;
      s_ezz[idx] = ezz;
      s_exz[idx] = exz;
    }
    __syncthreads();
    if (x.fs && z0 == L) {
      for (int lx = 1 + tid; lx < EW; lx += NT) {
        const int gi = x0 - 1 + lx;
        if (gi >= xe) continue;
        const int e = EW + lx;
        const int ci = lx - 1;  // coefficient box row 0 is the surface row
        const T eb = T(0.25) * (s_exz[e] + s_exz[e - 1] + s_exz[e - EW] + s_exz[e - EW - 1]);
        s_ezz[e] = -(s_c[C13 * PC + ci] * s_exx[e] + s_c[C35 * PC + ci] * eb) / s_c[C33 * PC + ci];
      }
      __syncthreads();
    }
  }

  // ---- 4. stresses and memory variables on the tile ---------------------
#pragma unroll 1
  for (int k = 0; k < TX * TZ / NT; ++k) {
    const int lx = tid % TX, lz = tid / TX + k * (NT / TX);
    const int gi = x0 + lx, gj = z0 + lz;
    if (gi >= xe || gj >= ze) continue;
    const long long g = (long long)gj * nx + gi;
    const int sv = (lz + HV) * VWp + lx + HVP;
    const int ci = lz * CW + lx;
    const int mi = TTI ? (lz + 1) * MW + lx + 4 : lz * MW + lx;
    T rxx, rzz, rxz, exx, ezz, exz;
    rates(sv, gi, gj, true, rxx, rzz, rxz);
    const bool surf = x.fs && gj == L;
    const T *c55 = s_c + C55 * PC;
    const T c13 = s_c[C13 * PC + ci];
    const T C55h = T(0.25) * (c55[ci] + c55[ci + 1] + c55[ci + CW] + c55[ci + CW + 1]);
    T dsxx, dszz, dsxz;
    if constexpr (TTI) {
      const int e = (lz + 1) * EW + lx + 1;
      exx = s_exx[e];
      ezz = s_ezz[e];
      exz = s_exz[e];
      const T *c15 = s_c + C15 * PC, *c35 = s_c + C35 * PC;
      const T ebxz = T(0.25) * (s_exz[e] + s_exz[e - 1] + s_exz[e - EW] + s_exz[e - EW - 1]);
      const T ebxx = T(0.25) * (s_exx[e] + s_exx[e + 1] + s_exx[e + EW] + s_exx[e + EW + 1]);
      const T ebzz = T(0.25) * (s_ezz[e] + s_ezz[e + 1] + s_ezz[e + EW] + s_ezz[e + EW + 1]);
      const T C15h = T(0.25) * (c15[ci] + c15[ci + 1] + c15[ci + CW] + c15[ci + CW + 1]);
      const T C35h = T(0.25) * (c35[ci] + c35[ci + 1] + c35[ci + CW] + c35[ci + CW + 1]);
      dsxx = s_c[C11 * PC + ci] * exx + c13 * ezz + c15[ci] * ebxz;
      dszz = c13 * exx + s_c[C33 * PC + ci] * ezz + c35[ci] * ebxz;
      dsxz = C55h * exz + C15h * ebxx + C35h * ebzz;
    } else {
      effective(mi, NSLS > 0 ? s_tau[ci] : T(0), rxx, rzz, rxz, exx, ezz, exz);
      const T c11 = KIND == VI_MEDIUM_ISO ? c13 + T(2) * c55[ci] : s_c[C11 * PC + ci];
      const T c33 = KIND == VI_MEDIUM_ISO ? c11 : s_c[C33 * PC + ci];
      if (surf) ezz = -(c13 * exx) / c33;
      dsxx = c11 * exx + c13 * ezz;
      dszz = c13 * exx + c33 * ezz;
      dsxz = C55h * exz;
    }
    const int si = (lz + HS) * SWp + lx + HSP;
    T sxx = s_sxx[si] + dt * dsxx;
    T szz = s_szz[si] + dt * dszz;
    T sxz = s_sxz[si] + dt * dsxz;
    if constexpr (NSLS > 0) {
      constexpr int MP = MW * MH;
#pragma unroll
      for (int n = 0; n < NSLS; ++n) {
        const T mxx = s_m[(0 * NSLS + n) * MP + mi];
        const T mzz = s_m[(1 * NSLS + n) * MP + mi];
        const T mxz = s_m[(2 * NSLS + n) * MP + mi];
        a.m_o[(0 * NSLS + n) * a.mstride_o + g] = mxx + dt * (a.a1[n] * rxx + a.a2[n] * mxx);
        a.m_o[(1 * NSLS + n) * a.mstride_o + g] =
            surf ? T(0) : mzz + dt * (a.a1[n] * rzz + a.a2[n] * mzz);
        a.m_o[(2 * NSLS + n) * a.mstride_o + g] = mxz + dt * (a.a1[n] * rxz + a.a2[n] * mxz);
      }
    }
    for (int e = e0; e < e1; ++e) {
      const int4 en = x.tile_ent[e];
      if (en.w != TL_EXPLOSIVE || en.x != gi || en.y != gj) continue;
      const T w = x.it < x.wnt ? x.wavelet[(long long)en.z * x.wnt + x.it] : T(0);
      sxx += dt * x.amp[en.z] * w;
      szz += dt * x.amp[en.z] * w;
    }
    if (surf) szz = T(0);
    a.sxx_o[g] = sxx;
    a.szz_o[g] = szz;
    a.sxz_o[g] = sxz;
    s_sxx[si] = sxx;
    s_szz[si] = szz;
    s_sxz[si] = sxz;
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

template <typename T, int KIND, int NSLS>
static int launch_tma_one(const StepArgs<T> &a, const FusedExtras<T> &x, const TmaMaps &maps,
                          int ntiles, cudaStream_t st) {
  if constexpr (!TmaPick<T, KIND, NSLS>::OK) {
    return set_error(VI_ERR_ARG, "TMA-staged step does not fit shared memory for this medium");
  } else {
    using G = typename TmaPick<T, KIND, NSLS>::Lay;
    static unsigned long long attr_set = 0;
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 64 && !(attr_set & (1ULL << dev))) {
      cudaError_t e = cudaFuncSetAttribute(k_fused_tma<T, KIND, NSLS>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, G::BYTES);
      if (e != cudaSuccess) return cuda_check(e, "TMA step smem attribute");
      attr_set |= 1ULL << dev;
    }
    k_fused_tma<T, KIND, NSLS><<<ntiles, G::NT, G::BYTES, st>>>(a, x, maps);
    return VI_OK;
  }
}

template <typename T>
int launch_fused_tma(int kind, const StepArgs<T> &a, const FusedExtras<T> &x, const TmaMaps &maps,
                     int ntiles, cudaStream_t st) {
#define VB_CASE(K, N) \
  if (kind == K && a.nsls == N) return launch_tma_one<T, K, N>(a, x, maps, ntiles, st);
#define VB_KIND(K) VB_CASE(K, 0) VB_CASE(K, 1) VB_CASE(K, 2) VB_CASE(K, 3) VB_CASE(K, 4) VB_CASE(K, 5)
  VB_KIND(VI_MEDIUM_ISO)
  VB_KIND(VI_MEDIUM_VTI)
  VB_KIND(VI_MEDIUM_TTI)
#undef VB_KIND
#undef VB_CASE
  return set_error(VI_ERR_ARG, "unsupported medium / nsls combination");
}

template int launch_fused_tma<float>(int, const StepArgs<float> &, const FusedExtras<float> &,
                                     const TmaMaps &, int, cudaStream_t);
template int launch_fused_tma<double>(int, const StepArgs<double> &, const FusedExtras<double> &,
                                      const TmaMaps &, int, cudaStream_t);

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
  b.ok = ok;
  return b;
}

template <typename T, int KIND>
static TmaBoxes boxes_kind(int nsls) {
#define VB_G(N) \
  if (nsls == N) return boxes_of<typename TmaPick<T, KIND, N>::Lay>(TmaPick<T, KIND, N>::OK);
  VB_G(0) VB_G(1) VB_G(2) VB_G(3) VB_G(4) VB_G(5)
#undef VB_G
  TmaBoxes b{};
  b.ok = false;
  return b;
}

TmaBoxes tma_boxes(int kind, int nsls, int esize) {
  if (esize == 4) {
    if (kind == VI_MEDIUM_ISO) return boxes_kind<float, VI_MEDIUM_ISO>(nsls);
    if (kind == VI_MEDIUM_VTI) return boxes_kind<float, VI_MEDIUM_VTI>(nsls);
    return boxes_kind<float, VI_MEDIUM_TTI>(nsls);
  }
  if (kind == VI_MEDIUM_ISO) return boxes_kind<double, VI_MEDIUM_ISO>(nsls);
  if (kind == VI_MEDIUM_VTI) return boxes_kind<double, VI_MEDIUM_VTI>(nsls);
  return boxes_kind<double, VI_MEDIUM_TTI>(nsls);
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
