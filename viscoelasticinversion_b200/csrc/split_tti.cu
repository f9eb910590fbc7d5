// split_tti.cu — the stress pass of the split step for TTI media.
//
// The TTI law couples the components: sigma_xx and sigma_zz need the shear
// effective rate at the integer node, sigma_xz the normal effective rates
// at the half node, each the mean of the four neighbouring rates
// (custom_solver/Model.jl:59-108).  A CTA computes the effective rates of
// its 64 x 8 tile and of the one-cell ring around it into shared memory,
// from a TMA box of the new velocities, and then updates its own cells.
// Ring cells belong to neighbouring CTAs, which update their memory
// variables and CPML psi at the same time, so M and psi are read from one
// buffer and written to the other (ping-pong per step); sigma is read and
// written only at the CTA's own cells, in place.  The velocity pass is the
// medium-independent one of split.cu (k_split_vel_tma by default), with psi
// read from one set and written to the other.
#include <atomic>
#include <cudaTypedefs.h>

#include <cstdint>

#include "afda.cuh"
#include "cpml4.cuh"
#include "pdl.cuh"
#include "plan.cuh"
#include "split.cuh"
#include "tma.cuh"
#include "vec.cuh"

namespace vb {

// CPML-corrected strain rates (ddxm vx, ddzm vz, ddzp vx + ddxp vz) of the
// 4 cells (gi0.., gj) whose 12-cell x window starts at v-box index wb.  psi
// is read from the input set and, for the CTA's own cells, written to the
// output set.
// AFDA: the grid has the H-AFDA surface, under which the z derivatives of
// the four rows below it are one-sided (v box row of grid row L + m:
// wb + (L + m - gj) * BW).
template <typename T, int BW, bool AFDA>
__device__ __forceinline__ void tti_rates4(const StepArgs<T> &a, const T *s_vx, const T *s_vz,
                                           int wb, int gi0, int gj, bool own, Q4<T> &rxx,
                                           Q4<T> &rzz, Q4<T> &rxz) {
  T hvx[12], hvz[12];
  row12s(s_vx + wb, hvx);
  row12s(s_vz + wb, hvz);
  Q4<T> zvz = splat4<T>(0), zvx = splat4<T>(0);
#pragma unroll
  for (int q = -4; q <= 4; ++q) {
    if (q <= 3) {  // ddzm(vz)
      const T cq = q >= 0 ? a.Dz[q] : -a.Dz[-q - 1];
      const Q4<T> v = q == 0 ? win4(hvz, 4) : lds4(s_vz + wb + q * BW + 4);
      zvz = fma4(splat4<T>(cq), v, zvz);
    }
    if (q >= -3) {  // ddzp(vx)
      const T cq = q >= 1 ? a.Dz[q - 1] : -a.Dz[-q];
      const Q4<T> v = q == 0 ? win4(hvx, 4) : lds4(s_vx + wb + q * BW + 4);
      zvx = fma4(splat4<T>(cq), v, zvx);
    }
  }
  if (AFDA && gj < L + 4) {  // on the surface row the tau_zz = 0 relation sets e_zz
    const int qs = gj - L;
    if (qs >= 1) zvz = afda4<2>(a, qs, [&](int m) { return lds4(s_vz + wb + (L + m - gj) * BW + 4); });
    if (qs < 3) zvx = afda4<3>(a, qs, [&](int m) { return lds4(s_vx + wb + (L + m - gj) * BW + 4); });
  }
  const int nx = a.nx, nz = a.nz;
  Q4<T> dxvx = dms4(hvx, a.Dx), dxvz = dps4(hvz, a.Dx), dzvz = zvz, dzvx = zvx;
  if (gi0 < a.Lx || gi0 + 3 >= nx - a.Rx)
    cpml_x4(a, gi0, gj, CpmlRows{PX_VX, T_B, T_A, T_IK}, CpmlRows{PX_VZ, T_BH, T_AH, T_IKH}, a.psix, a.psix_o, own,
            dxvx, dxvz);
  const int zs = strip_z(gj, nz, a.Tz, a.Bz);
  if (zs >= 0)
    cpml_z4(a, zs, gi0, gj, CpmlRows{PZ_VZ, T_B, T_A, T_IK}, CpmlRows{PZ_VX, T_BH, T_AH, T_IKH}, a.psiz, a.psiz_o,
            own, dzvz, dzvx);
  rxx = dxvx;
  rzz = dzvz;
  rxz = add4(dzvx, dxvz);
}

// Sums over the SLS of the memory variables (xx, zz, xz) of 4 cells whose
// memory variables start at m (plane stride ms).  They do not depend on the
// new velocities, so they are loaded while the velocity box is in flight.
template <typename T, int NSLS>
__device__ __forceinline__ void tti_msum4(const T *m, long long ms, long long g, Q4<T> &Sxx,
                                          Q4<T> &Szz, Q4<T> &Sxz) {
  Sxx = Szz = Sxz = splat4<T>(0);
#pragma unroll
  for (int n = 0; n < NSLS; ++n) {
    Sxx = add4(Sxx, ldc4(m + n * ms + g));
    Szz = add4(Szz, ldc4(m + (NSLS + n) * ms + g));
    Sxz = add4(Sxz, ldc4(m + (2 * NSLS + n) * ms + g));
  }
}

// Effective SLS rates e = (1 + tau) r + tau * sum_n M_n of 4 cells.
template <typename T, int NSLS>
__device__ __forceinline__ void tti_effective4(const Q4<T> &tau, const Q4<T> &Sxx,
                                               const Q4<T> &Szz, const Q4<T> &Sxz,
                                               const Q4<T> &rxx, const Q4<T> &rzz,
                                               const Q4<T> &rxz, Q4<T> &exx, Q4<T> &ezz,
                                               Q4<T> &exz) {
  if constexpr (NSLS > 0) {
    const Q4<T> t1 = add4(tau, splat4<T>(T(1)));
    exx = fma4(t1, rxx, mul4(tau, Sxx));
    ezz = fma4(t1, rzz, mul4(tau, Szz));
    exz = fma4(t1, rxz, mul4(tau, Sxz));
  } else {
    exx = rxx;
    ezz = rzz;
    exz = rxz;
  }
}

// [u1, u2, u3, w]: the group shifted one cell to the right's values
template <typename T>
__device__ __forceinline__ Q4<T> next4(const Q4<T> &u, T w) {
  return {{u.v[1], u.v[2], u.v[3], w}};
}
// [w, u0, u1, u2]: the group shifted one cell to the left's values
template <typename T>
__device__ __forceinline__ Q4<T> prev4(const Q4<T> &u, T w) {
  return {{w, u.v[0], u.v[1], u.v[2]}};
}
// mean of the four cells (i, j), (i+1, j), (i, j+1), (i+1, j+1) of a group
template <typename T>
__device__ __forceinline__ Q4<T> mean4_fwd(const Q4<T> &a, T a4, const Q4<T> &b, T b4) {
  return mul4(splat4<T>(T(0.25)), add4(add4(add4(a, next4(a, a4)), b), next4(b, b4)));
}

// COMP (FP32): sigma accumulated with its rounding residue (a.slo, two_sum_acc4).
template <typename T, int NSLS, bool HINT, bool COMP = false, bool AFDA = false, typename G = SplitTtiGeom<T>>
__device__ __forceinline__ void split_stress_tti_tile(const StepArgs<T> &a, const FusedExtras<T> &x,
                                                      const SplitMaps &maps, int tile) {
  static_assert(!COMP || sizeof(T) == 4, "compensated stress: FP32");
  constexpr int TX = G::TX, TZ = G::TZ, BW = G::BW, EW = G::EW, EG = G::EW / 4;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem_raw);
  T *s_vx = reinterpret_cast<T *>(smem_raw) + G::O0;
  T *s_vz = s_vx + G::PB;
  T *s_exx = s_vz + G::PB, *s_ezz = s_exx + G::PE, *s_exz = s_ezz + G::PE;
  const int x0 = L + (tile % x.ntx) * TX, z0 = L + (tile / x.ntx) * TZ;
  const int nx = a.nx, nz = a.nz, xe = nx - L, ze = nz - L;
  const int tid = threadIdx.x;
  pdl_wait();  // the new velocities are complete and visible
  if (tid == 0) mbar_init(bar, 1);
  __syncthreads();
  if (tid == 0) {
    // v box origin (x0 - 8, z0 - 5): the e box (x0 - 4, z0 - 1) with the
    // 4-cell stencil halo; x0 - 8 is a multiple of 4 elements
    mbar_arrive_expect_tx(bar, 2 * G::BOX_BYTES);
    tma_load_2d(s_vx, &maps.a, x0 - 8, z0 - 5, bar);
    tma_load_2d(s_vz, &maps.b, x0 - 8, z0 - 5, bar);
  }
  const int r = tid / (TX / 4), lx = 4 * (tid % (TX / 4));
  const int gi0 = x0 + lx, gj = z0 + r;
  const bool act = gi0 < xe && gj < ze;
  const long long g = (long long)gj * nx + gi0;
  Q4<T> tau = splat4<T>(0);
  if (act && NSLS > 0) tau = ldg4(a.tau + g);
  // the ring group of this thread (threads 0 .. NRING-1): e-box row/column
  int rr = -1, rc = 0;
  if (tid < 2 * EG) {
    rr = tid < EG ? 0 : TZ + 1;
    rc = 4 * (tid < EG ? tid : tid - EG);
  } else if (tid < G::NRING) {
    const int q = tid - 2 * EG;
    rr = 1 + (q < TZ ? q : q - TZ);
    rc = q < TZ ? 0 : EW - 4;
  }
  const int rgi0 = x0 - 4 + rc, rgj = z0 - 1 + rr;
  const bool ract = rr >= 0 && rgi0 >= L && rgi0 < xe && rgj >= L && rgj < ze;
  const long long rg = (long long)rgj * nx + rgi0;
  Q4<T> rtau = splat4<T>(0);
  if (ract && NSLS > 0) rtau = ldg4(a.tau + rg);
  // while the box is in flight: the memory-variable sums into registers
  Q4<T> mxx = splat4<T>(0), mzz = mxx, mxz = mxx, qmxx = mxx, qmzz = mxx, qmxz = mxx;
  if (act) tti_msum4<T, NSLS>(a.m, a.mstride, g, mxx, mzz, mxz);
  if (ract) tti_msum4<T, NSLS>(a.m, a.mstride, rg, qmxx, qmzz, qmxz);
  const int e0 = x.tile_off[tile], e1 = x.tile_off[tile + 1];
  const bool ok = mbar_wait_bounded(bar, 0, 1u << 22);
  if (__syncthreads_or(!ok)) {
    if (tid == 0) {
      atomicOr(x.err, kErrTimeout);
      mbar_wait_bounded(bar, 0, 1u << 22);
    }
    return;
  }
  // ---- effective rates: own group, then the ring group (zero outside U)
  Q4<T> rxx = splat4<T>(0), rzz = rxx, rxz = rxx;
  {
    Q4<T> exx = splat4<T>(0), ezz = exx, exz = exx;
    if (act) {
      tti_rates4<T, BW, AFDA>(a, s_vx, s_vz, (r + 5) * BW + lx + 4, gi0, gj, true, rxx, rzz, rxz);
      tti_effective4<T, NSLS>(tau, mxx, mzz, mxz, rxx, rzz, rxz, exx, ezz, exz);
    }
    const int e = (r + 1) * EW + lx + 4;
    stg4(s_exx + e, exx);
    stg4(s_ezz + e, ezz);
    stg4(s_exz + e, exz);
  }
  if (rr >= 0) {
    Q4<T> exx = splat4<T>(0), ezz = exx, exz = exx;
    if (ract) {
      Q4<T> qxx, qzz, qxz;
      tti_rates4<T, BW, AFDA>(a, s_vx, s_vz, (rr + 4) * BW + rc, rgi0, rgj, false, qxx, qzz, qxz);
      tti_effective4<T, NSLS>(rtau, qmxx, qmzz, qmxz, qxx, qzz, qxz, exx, ezz, exz);
    }
    const int e = rr * EW + rc;
    stg4(s_exx + e, exx);
    stg4(s_ezz + e, ezz);
    stg4(s_exz + e, exz);
  }
  __syncthreads();
  if (x.fs && z0 == L) {
    // tau_zz = 0 on the surface row (e row 1), columns x0 .. x0 + TX:
    // e_zz = -(C13 e_xx + C35 mean(e_xz)) / C33, e_xz above the surface 0
    for (int c = tid; c <= TX; c += G::NT) {
      const int gi = x0 + c;
      if (gi >= xe) continue;
      const int e = EW + c + 4;
      const long long gs = (long long)L * nx + gi;
      const T eb = T(0.25) * (s_exz[e] + s_exz[e - 1] + s_exz[e - EW] + s_exz[e - EW - 1]);
      s_ezz[e] = -(__ldg(a.c13 + gs) * s_exx[e] + __ldg(a.c35 + gs) * eb) / __ldg(a.c33 + gs);
    }
    __syncthreads();
  }
  if (!act) return;
  // ---- stresses and memory variables of the own group
  const T dt = a.dt;
  const Q4<T> dt4 = splat4<T>(dt);
  const bool surf = x.fs && gj == L;
  Q4<T> sxx = ldc4(a.sxx + g), szz = ldc4(a.szz + g), sxz = ldc4(a.sxz + g);
  // read once per step: streamed through L2 (ring-shared operands are not)
  const Q4<T> C11 = ldgh4(a.c11 + g, l2_stream_c<HINT>()), C13 = ldgh4(a.c13 + g, l2_stream_c<HINT>()),
              C33 = ldgh4(a.c33 + g, l2_stream_c<HINT>());
  const Q4<T> c15a = ldg4(a.c15 + g), c15b = ldg4(a.c15 + g + nx);
  const Q4<T> c35a = ldg4(a.c35 + g), c35b = ldg4(a.c35 + g + nx);
  const Q4<T> c55a = ldg4(a.c55 + g), c55b = ldg4(a.c55 + g + nx);
  const T c15a4 = __ldg(a.c15 + g + 4), c15b4 = __ldg(a.c15 + g + nx + 4);
  const T c35a4 = __ldg(a.c35 + g + 4), c35b4 = __ldg(a.c35 + g + nx + 4);
  const T c55a4 = __ldg(a.c55 + g + 4), c55b4 = __ldg(a.c55 + g + nx + 4);
  const int e = (r + 1) * EW + lx + 4;
  const Q4<T> exx = lds4(s_exx + e), ezz = lds4(s_ezz + e), exz = lds4(s_exz + e);
  // e_xz at the integer node: mean of (i-1/2, j-1/2) .. (i+1/2, j+1/2)
  const Q4<T> xzm = lds4(s_exz + e - EW);
  const Q4<T> ebxz = mul4(splat4<T>(T(0.25)),
                          add4(add4(add4(exz, prev4(exz, s_exz[e - 1])), xzm), prev4(xzm, s_exz[e - EW - 1])));
  // e_xx, e_zz at the half node: mean of (i, j) .. (i+1, j+1)
  const Q4<T> ebxx = mean4_fwd(exx, s_exx[e + 4], lds4(s_exx + e + EW), s_exx[e + EW + 4]);
  const Q4<T> ebzz = mean4_fwd(ezz, s_ezz[e + 4], lds4(s_ezz + e + EW), s_ezz[e + EW + 4]);
  const Q4<T> C15h = mean4_fwd(c15a, c15a4, c15b, c15b4);
  const Q4<T> C35h = mean4_fwd(c35a, c35a4, c35b, c35b4);
  const Q4<T> C55h = mean4_fwd(c55a, c55a4, c55b, c55b4);
  // increments (COMP) or the updated stresses
  Q4<T> ixx, izz, ixz;
  uint2 lxx{}, lzz{}, lxz{};
  if constexpr (COMP) {
    lxx = ldh_u2(a.slo + g, l2_stream_c<HINT>());
    lzz = ldh_u2(a.slo + a.slo_plane + g, l2_stream_c<HINT>());
    lxz = ldh_u2(a.slo + 2 * a.slo_plane + g, l2_stream_c<HINT>());
    ixx = mul4(dt4, fma4(C11, exx, fma4(C13, ezz, mul4(c15a, ebxz))));
    izz = mul4(dt4, fma4(C13, exx, fma4(C33, ezz, mul4(c35a, ebxz))));
    ixz = mul4(dt4, fma4(C55h, exz, fma4(C15h, ebxx, mul4(C35h, ebzz))));
  } else {
    sxx = fma4(dt4, fma4(C11, exx, fma4(C13, ezz, mul4(c15a, ebxz))), sxx);
    szz = fma4(dt4, fma4(C13, exx, fma4(C33, ezz, mul4(c35a, ebxz))), szz);
    sxz = fma4(dt4, fma4(C55h, exz, fma4(C15h, ebxx, mul4(C35h, ebzz))), sxz);
  }
  if constexpr (NSLS > 0) {
#pragma unroll
    for (int n = 0; n < NSLS; ++n) {
      const Q4<T> a1 = splat4<T>(a.a1[n]), a2 = splat4<T>(a.a2[n]);
      const Q4<T> mx = ldc4(a.m + (0 * NSLS + n) * a.mstride + g);
      const Q4<T> mz = ldc4(a.m + (1 * NSLS + n) * a.mstride + g);
      const Q4<T> mq = ldc4(a.m + (2 * NSLS + n) * a.mstride + g);
      sth4(a.m_o + (0 * NSLS + n) * a.mstride_o + g, fma4(dt4, fma4(a1, rxx, mul4(a2, mx)), mx), l2_stream_c<HINT>());
      sth4(a.m_o + (1 * NSLS + n) * a.mstride_o + g,
           surf ? splat4<T>(0) : fma4(dt4, fma4(a1, rzz, mul4(a2, mz)), mz), l2_stream_c<HINT>());
      sth4(a.m_o + (2 * NSLS + n) * a.mstride_o + g, fma4(dt4, fma4(a1, rxz, mul4(a2, mq)), mq), l2_stream_c<HINT>());
    }
  }
  for (int q = e0; q < e1; ++q) {  // explosive sources (after the force ones, before receivers)
    const int4 en = x.tile_ent[q];
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
  if (surf) szz = splat4<T>(0);
  if (!finite3(sxx, szz, sxz)) atomicOr(x.err, kErrNonFinite);
  // sigma is re-read by the next velocity pass: keep it in L2
  sth4(a.sxx + g, sxx, l2_keep_c<HINT>());
  sth4(a.szz + g, szz, l2_keep_c<HINT>());
  sth4(a.sxz + g, sxz, l2_keep_c<HINT>());
  if (x.fs == kFsImaging) {
    // stress images: szz(L-k) = -szz(L+k), k = 1..4; sxz(L-1-k) = -sxz(L+k), k = 0..3
    const int k = gj - L;
    if (k >= 1 && k <= L) stg4(a.szz + (long long)(L - k) * nx + gi0, mul4(splat4<T>(T(-1)), szz));
    if (k >= 0 && k < L) stg4(a.sxz + (long long)(L - 1 - k) * nx + gi0, mul4(splat4<T>(T(-1)), sxz));
  }
}

template <typename T, int NSLS, bool HINT, bool COMP, bool AFDA>
__global__ void __launch_bounds__(SplitTtiGeom<T>::NT, (sizeof(T) == 4 ? 512 : 256) / SplitTtiGeom<T>::NT)
    k_split_stress_tti(const __grid_constant__ StepArgs<T> a, const __grid_constant__ FusedExtras<T> x,
                       const __grid_constant__ SplitMaps maps) {
  split_stress_tti_tile<T, NSLS, HINT, COMP, AFDA>(a, x, maps, blockIdx.x);
}

// Batched: one tile of one shot per CTA; the step parity selects the
// shot's M / psi buffers.
template <typename T, int NSLS, bool COMP, bool AFDA>
__global__ void __launch_bounds__(SplitTtiGeomBatch<T>::NT, (sizeof(T) == 4 ? 512 : 256) / SplitTtiGeomBatch<T>::NT)
    k_split_stress_tti_batch(const BatchDev<T> b, int it) {
  int shot, tile;
  batch_locate(b, blockIdx.x, shot, tile);
  FusedExtras<T> x = b.ext[shot];
  x.it = it;
  // COMP: compensated FP32 shots carry the stress residues, as the unbatched
  // split step; AFDA: some shot has the H-AFDA surface
  using G = SplitTtiGeomBatch<T>;
  if (AFDA && x.fs == kFsAfda)
    split_stress_tti_tile<T, NSLS, false, COMP, true, G>(b.args[2 * shot + (it & 1)], x, b.smaps[shot], tile);
  else
    split_stress_tti_tile<T, NSLS, false, COMP, false, G>(b.args[2 * shot + (it & 1)], x, b.smaps[shot], tile);
}

template <typename T, int NSLS, bool HINT, bool COMP = false, bool AFDA = false>
static int launch_tti_k(const StepArgs<T> &a, const FusedExtras<T> &x, const SplitMaps &m, int ntiles,
                        cudaStream_t st, bool pdl) {
  using G = SplitTtiGeom<T>;
  static std::atomic<unsigned long long> attr_set{0};  // one bit per device set up (any thread)
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && !(attr_set & (1ULL << dev))) {
    cudaError_t e = cudaFuncSetAttribute(k_split_stress_tti<T, NSLS, HINT, COMP, AFDA>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM);
    if (e != cudaSuccess) return cuda_check(e, "split TTI stress smem attribute");
    attr_set |= 1ULL << dev;
  }
  return cuda_check(launch_pdl(k_split_stress_tti<T, NSLS, HINT, COMP, AFDA>, dim3(ntiles), dim3(G::NT),
                               (size_t)G::SMEM, st, pdl, a, x, m),
                    "split TTI stress launch");
}

// compensated (FP32) when the caller set the residue planes (a.slo)
template <typename T, int NSLS>
static int launch_tti(const StepArgs<T> &a, const FusedExtras<T> &x, const SplitMaps &m, int ntiles,
                      cudaStream_t st, bool pdl) {
  if constexpr (sizeof(T) == 4) {
    if (a.slo) {
      if (x.fs == kFsAfda)
        return x.l2hint ? launch_tti_k<T, NSLS, true, true, true>(a, x, m, ntiles, st, pdl)
                        : launch_tti_k<T, NSLS, false, true, true>(a, x, m, ntiles, st, pdl);
      return x.l2hint ? launch_tti_k<T, NSLS, true, true>(a, x, m, ntiles, st, pdl)
                      : launch_tti_k<T, NSLS, false, true>(a, x, m, ntiles, st, pdl);
    }
  }
  if (x.fs == kFsAfda)
    return x.l2hint ? launch_tti_k<T, NSLS, true, false, true>(a, x, m, ntiles, st, pdl)
                    : launch_tti_k<T, NSLS, false, false, true>(a, x, m, ntiles, st, pdl);
  return x.l2hint ? launch_tti_k<T, NSLS, true>(a, x, m, ntiles, st, pdl)
                  : launch_tti_k<T, NSLS, false>(a, x, m, ntiles, st, pdl);
}

template <typename T>
int launch_split_stress_tti(const StepArgs<T> &a, const FusedExtras<T> &x, const SplitMaps &m,
                            int ntiles, cudaStream_t st, bool pdl) {
  switch (a.nsls) {
    case 0: return launch_tti<T, 0>(a, x, m, ntiles, st, pdl);
    case 1: return launch_tti<T, 1>(a, x, m, ntiles, st, pdl);
    case 2: return launch_tti<T, 2>(a, x, m, ntiles, st, pdl);
    case 3: return launch_tti<T, 3>(a, x, m, ntiles, st, pdl);
    case 4: return launch_tti<T, 4>(a, x, m, ntiles, st, pdl);
    case 5: return launch_tti<T, 5>(a, x, m, ntiles, st, pdl);
    default: return set_error(VI_ERR_ARG, "nsls must be 0..5");
  }
}

template <typename T, int NSLS, bool COMP, bool AFDA>
static int launch_tti_batch_k(const BatchDev<T> &b, int it, int nitems, cudaStream_t st, bool pdl) {
  using G = SplitTtiGeomBatch<T>;
  static std::atomic<unsigned long long> attr_set{0};  // one bit per device set up (any thread)
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && !(attr_set & (1ULL << dev))) {
    cudaError_t e = cudaFuncSetAttribute(k_split_stress_tti_batch<T, NSLS, COMP, AFDA>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM);
    if (e != cudaSuccess) return cuda_check(e, "batched split TTI stress smem attribute");
    attr_set |= 1ULL << dev;
  }
  if (nitems <= 0) return VI_OK;  // attribute set-up only
  return cuda_check(launch_pdl(k_split_stress_tti_batch<T, NSLS, COMP, AFDA>, dim3(nitems), dim3(G::NT),
                               (size_t)G::SMEM, st, pdl, b, it),
                    "batched split TTI stress launch");
}

template <typename T, int NSLS>
static int launch_tti_batch(bool comp, bool afda, const BatchDev<T> &b, int it, int nitems, cudaStream_t st,
                            bool pdl) {
  if constexpr (sizeof(T) == 4)
    if (comp)
      return afda ? launch_tti_batch_k<T, NSLS, true, true>(b, it, nitems, st, pdl)
                  : launch_tti_batch_k<T, NSLS, true, false>(b, it, nitems, st, pdl);
  return afda ? launch_tti_batch_k<T, NSLS, false, true>(b, it, nitems, st, pdl)
              : launch_tti_batch_k<T, NSLS, false, false>(b, it, nitems, st, pdl);
}

template <typename T>
int launch_split_stress_tti_batch(int nsls, bool comp, bool afda, const BatchDev<T> &b, int it, int nitems,
                                  cudaStream_t st, bool pdl) {
  switch (nsls) {
    case 0: return launch_tti_batch<T, 0>(comp, afda, b, it, nitems, st, pdl);
    case 1: return launch_tti_batch<T, 1>(comp, afda, b, it, nitems, st, pdl);
    case 2: return launch_tti_batch<T, 2>(comp, afda, b, it, nitems, st, pdl);
    case 3: return launch_tti_batch<T, 3>(comp, afda, b, it, nitems, st, pdl);
    case 4: return launch_tti_batch<T, 4>(comp, afda, b, it, nitems, st, pdl);
    case 5: return launch_tti_batch<T, 5>(comp, afda, b, it, nitems, st, pdl);
    default: return set_error(VI_ERR_ARG, "nsls must be 0..5");
  }
}

template int launch_split_stress_tti_batch<float>(int, bool, bool, const BatchDev<float> &, int, int,
                                                  cudaStream_t, bool);
template int launch_split_stress_tti_batch<double>(int, bool, bool, const BatchDev<double> &, int, int,
                                                   cudaStream_t, bool);
template int launch_split_stress_tti<float>(const StepArgs<float> &, const FusedExtras<float> &,
                                            const SplitMaps &, int, cudaStream_t, bool);
template int launch_split_stress_tti<double>(const StepArgs<double> &, const FusedExtras<double> &,
                                             const SplitMaps &, int, cudaStream_t, bool);

}  // namespace vb
