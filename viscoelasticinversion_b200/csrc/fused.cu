// fused.cu — one kernel launch per time step.
//
// Each CTA owns a TX x TZ tile of the update region.  It stages the input
// stresses of the tile plus an (HV+4)-cell halo in shared memory, recomputes
// the new velocities on the tile plus an HV-cell halo (the redundant halo
// work replaces a grid-wide barrier between the velocity and stress stages),
// and then updates stresses, memory variables and CPML psi on its own cells.
// All state is ping-ponged (input set -> output set) so that halo
// recomputation never reads a value another CTA has already advanced.
// Per step each cell's state and medium cross HBM once: reads of v, sigma,
// M, psi and the medium, writes of v, sigma, M and psi.
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <vector>

#include "fused.cuh"
#include "fused_tma.cuh"
#include "plan.cuh"

namespace vb {

template <typename T, int KIND>
__device__ __forceinline__ T c11v(const StepArgs<T> &a, long long g) {
  return KIND == VI_MEDIUM_ISO ? a.c13[g] + T(2) * a.c55[g] : a.c11[g];
}
template <typename T, int KIND>
__device__ __forceinline__ T c33v(const StepArgs<T> &a, long long g) {
  return KIND == VI_MEDIUM_ISO ? a.c13[g] + T(2) * a.c55[g] : a.c33[g];
}

// CPML-corrected velocity-derivative rates at cell (gi, gj) from the staged
// new velocities (index sv in the VW-wide velocity tile).  Writes the psi
// output set when `own`.
template <typename T, int VW>
__device__ __forceinline__ void strain_rates(const StepArgs<T> &a, const T *s_vx, const T *s_vz,
                                             int sv, int gi, int gj, bool own, T &rxx, T &rzz,
                                             T &rxz) {
  T dxvx = 0, dzvz = 0, dzvx = 0, dxvz = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int l = k + 1;
    dxvx += a.Dx[k] * (s_vx[sv + l - 1] - s_vx[sv - l]);
    dzvz += a.Dz[k] * (s_vz[sv + (l - 1) * VW] - s_vz[sv - l * VW]);
    dzvx += a.Dz[k] * (s_vx[sv + l * VW] - s_vx[sv - (l - 1) * VW]);
    dxvz += a.Dx[k] * (s_vz[sv + l] - s_vz[sv - l + 1]);
  }
  const int nx = a.nx;
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
  const int zs = strip_z(gj, a.nz, a.Tz, a.Bz);
  if (zs >= 0) {
    const int nz = a.nz;
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
}

template <typename T, int NSLS>
__device__ __forceinline__ void sls_effective(const StepArgs<T> &a, long long g, T rxx, T rzz,
                                              T rxz, T &exx, T &ezz, T &exz) {
  if (NSLS > 0) {
    T Sxx = 0, Szz = 0, Sxz = 0;
#pragma unroll
    for (int n = 0; n < NSLS; ++n) {
      Sxx += a.m[(0 * NSLS + n) * a.mstride + g];
      Szz += a.m[(1 * NSLS + n) * a.mstride + g];
      Sxz += a.m[(2 * NSLS + n) * a.mstride + g];
    }
    const T t = a.tau[g];
    const T t1 = T(1) + t;
    exx = t1 * rxx + t * Sxx;
    ezz = t1 * rzz + t * Szz;
    exz = t1 * rxz + t * Sxz;
  } else {
    exx = rxx;
    ezz = rzz;
    exz = rxz;
  }
}

template <typename T, int KIND, int NSLS>
__global__ void __launch_bounds__(256) k_fused(const StepArgs<T> a, const FusedExtras<T> x) {
  using G = FusedGeom<KIND>;
  constexpr int TX = G::TX, TZ = G::TZ, NT = G::NT, HV = G::HV, HS = G::HS;
  constexpr int SW = G::SW, SH = G::SH, VW = G::VW, VH = G::VH, EW = G::EW, EH = G::EH;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *s_sxx = reinterpret_cast<T *>(smem_raw);
  T *s_szz = s_sxx + SW * SH;
  T *s_sxz = s_szz + SW * SH;
  T *s_vx = s_sxz + SW * SH;
  T *s_vz = s_vx + VW * VH;
  T *s_exx = s_vz + VW * VH;
  T *s_ezz = s_exx + EW * EH;
  T *s_exz = s_ezz + EW * EH;

  const int tile = blockIdx.x;
  const int x0 = L + (tile % x.ntx) * TX;
  const int z0 = L + (tile / x.ntx) * TZ;
  const int nx = a.nx, nz = a.nz;
  const int xe = nx - L, ze = nz - L;
  const int tid = threadIdx.x;
  const T dt = a.dt;

  // 1. stage the input stresses of the tile + HS halo
  for (int idx = tid; idx < SW * SH; idx += NT) {
    const int gi = x0 - HS + idx % SW, gj = z0 - HS + idx / SW;
    const bool ok = gi >= 0 && gi < nx && gj >= 0 && gj < nz;
    const long long g = (long long)gj * nx + gi;
    s_sxx[idx] = ok ? a.sxx[g] : T(0);
    s_szz[idx] = ok ? a.szz[g] : T(0);
    s_sxz[idx] = ok ? a.sxz[g] : T(0);
  }
  __syncthreads();

  // 2. new velocities on the tile + HV halo
  for (int idx = tid; idx < VW * VH; idx += NT) {
    const int lx = idx % VW, lz = idx / VW;
    const int gi = x0 - HV + lx, gj = z0 - HV + lz;
    T vxn = 0, vzn = 0;
    if (gi >= L && gi < xe && gj >= L && gj < ze) {
      const int si = (lz + HS - HV) * SW + lx + HS - HV;
      T dxx = 0, dzxz = 0, dxxz = 0, dzz = 0;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int l = k + 1;
        dxx += a.Dx[k] * (s_sxx[si + l] - s_sxx[si - l + 1]);
        dzxz += a.Dz[k] * (s_sxz[si + (l - 1) * SW] - s_sxz[si - l * SW]);
        dxxz += a.Dx[k] * (s_sxz[si + l - 1] - s_sxz[si - l]);
        dzz += a.Dz[k] * (s_szz[si + l * SW] - s_szz[si - (l - 1) * SW]);
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
      const long long g = (long long)gj * nx + gi;
      const T r0 = a.rho[g];
      vxn = a.vx[g] + dt * (T(2) / (r0 + a.rho[g + 1])) * (dxx + dzxz);
      vzn = a.vz[g] + dt * (T(2) / (r0 + a.rho[g + nx])) * (dxxz + dzz);
    }
    s_vx[idx] = vxn;
    s_vz[idx] = vzn;
  }
  __syncthreads();

  const int e0 = x.tile_off[tile], e1 = x.tile_off[tile + 1];
  // 2b. force sources (one thread: entries are few and may share a cell)
  if (tid == 0) {
    for (int e = e0; e < e1; ++e) {
      const int4 en = x.tile_ent[e];
      if (en.w != TL_FORCE_X && en.w != TL_FORCE_Z) continue;
      const int lx = en.x - (x0 - HV), lz = en.y - (z0 - HV);
      const long long g = (long long)en.y * nx + en.x;
      const T w = x.it < x.wnt ? x.wavelet[(long long)en.z * x.wnt + x.it] : T(0);
      const T f = x.amp[en.z] * w;
      if (en.w == TL_FORCE_X)
        s_vx[lz * VW + lx] += dt * (T(2) / (a.rho[g] + a.rho[g + 1])) * f;
      else
        s_vz[lz * VW + lx] += dt * (T(2) / (a.rho[g] + a.rho[g + nx])) * f;
    }
  }
  __syncthreads();

  // 2c. write the tile's new velocities; receivers sample them
  for (int k = 0; k < TX * TZ / NT; ++k) {
    const int lx = tid % TX, lz = tid / TX + k * (NT / TX);
    const int gi = x0 + lx, gj = z0 + lz;
    if (gi < xe && gj < ze) {
      const long long g = (long long)gj * nx + gi;
      const int sv = (lz + HV) * VW + lx + HV;
      a.vx_o[g] = s_vx[sv];
      a.vz_o[g] = s_vz[sv];
    }
  }
  if (x.traces && x.it < x.tnt) {
    for (int e = e0 + tid; e < e1; e += NT) {
      const int4 en = x.tile_ent[e];
      if (en.w != TL_RECEIVER) continue;
      const int sv = (en.y - z0 + HV) * VW + en.x - x0 + HV;
      x.traces[(long long)en.z * x.tnt + x.it] = s_vx[sv];
      x.traces[(long long)(x.nrec + en.z) * x.tnt + x.it] = s_vz[sv];
    }
  }

  // 3. TTI: effective SLS rates on the tile + 1 ring (neighbour averages)
  if constexpr (KIND == VI_MEDIUM_TTI) {
    for (int idx = tid; idx < EW * EH; idx += NT) {
      const int lx = idx % EW, lz = idx / EW;
      const int gi = x0 - 1 + lx, gj = z0 - 1 + lz;
      T exx = 0, ezz = 0, exz = 0;
      if (gi >= L && gi < xe && gj >= L && gj < ze) {
        const int sv = (lz - 1 + HV) * VW + lx - 1 + HV;
        T rxx, rzz, rxz;
        strain_rates<T, VW>(a, s_vx, s_vz, sv, gi, gj, false, rxx, rzz, rxz);
        sls_effective<T, NSLS>(a, (long long)gj * nx + gi, rxx, rzz, rxz, exx, ezz, exz);
      }
      s_exx[idx] = exx;
      s_ezz[idx] = ezz;
      s_exz[idx] = exz;
    }
    __syncthreads();
    if (x.fs && z0 == L) {
      // tau_zz = 0 on the surface row (lz = 1 of the ring)
      for (int lx = 1 + tid; lx < EW; lx += NT) {
        const int gi = x0 - 1 + lx;
        if (gi >= xe) continue;
        const int e = EW + lx;
        const long long g = (long long)L * nx + gi;
        const T eb = T(0.25) * (s_exz[e] + s_exz[e - 1] + s_exz[e - EW] + s_exz[e - EW - 1]);
        s_ezz[e] = -(a.c13[g] * s_exx[e] + a.c35[g] * eb) / a.c33[g];
      }
      __syncthreads();
    }
  }

  // 4. stresses and memory variables on the tile
  for (int k = 0; k < TX * TZ / NT; ++k) {
    const int lx = tid % TX, lz = tid / TX + k * (NT / TX);
    const int gi = x0 + lx, gj = z0 + lz;
    if (gi >= xe || gj >= ze) continue;
    const long long g = (long long)gj * nx + gi;
    const int sv = (lz + HV) * VW + lx + HV;
    T rxx, rzz, rxz, exx, ezz, exz;
    strain_rates<T, VW>(a, s_vx, s_vz, sv, gi, gj, true, rxx, rzz, rxz);
    const bool surf = x.fs && gj == L;
    const T C13 = a.c13[g];
    const T C55h = T(0.25) * (a.c55[g] + a.c55[g + 1] + a.c55[g + nx] + a.c55[g + nx + 1]);
    T dsxx, dszz, dsxz;
    if constexpr (KIND == VI_MEDIUM_TTI) {
      const int e = (lz + 1) * EW + lx + 1;
      exx = s_exx[e];
      ezz = s_ezz[e];
      exz = s_exz[e];
      const T ebxz = T(0.25) * (s_exz[e] + s_exz[e - 1] + s_exz[e - EW] + s_exz[e - EW - 1]);
      const T ebxx = T(0.25) * (s_exx[e] + s_exx[e + 1] + s_exx[e + EW] + s_exx[e + EW + 1]);
      const T ebzz = T(0.25) * (s_ezz[e] + s_ezz[e + 1] + s_ezz[e + EW] + s_ezz[e + EW + 1]);
      const T C15h = T(0.25) * (a.c15[g] + a.c15[g + 1] + a.c15[g + nx] + a.c15[g + nx + 1]);
      const T C35h = T(0.25) * (a.c35[g] + a.c35[g + 1] + a.c35[g + nx] + a.c35[g + nx + 1]);
      dsxx = a.c11[g] * exx + C13 * ezz + a.c15[g] * ebxz;
      dszz = C13 * exx + a.c33[g] * ezz + a.c35[g] * ebxz;
      dsxz = C55h * exz + C15h * ebxx + C35h * ebzz;
    } else {
      sls_effective<T, NSLS>(a, g, rxx, rzz, rxz, exx, ezz, exz);
      const T C33 = c33v<T, KIND>(a, g);
      if (surf) ezz = -(C13 * exx) / C33;
      dsxx = c11v<T, KIND>(a, g) * exx + C13 * ezz;
      dszz = C13 * exx + C33 * ezz;
      dsxz = C55h * exz;
    }
    const int si = (lz + HS) * SW + lx + HS;
    T sxx = s_sxx[si] + dt * dsxx;
    T szz = s_szz[si] + dt * dszz;
    T sxz = s_sxz[si] + dt * dsxz;
#pragma unroll
    for (int n = 0; n < NSLS; ++n) {
      const long long i0 = (0 * NSLS + n) * a.mstride + g, o0 = (0 * NSLS + n) * a.mstride_o + g;
      const long long i1 = (1 * NSLS + n) * a.mstride + g, o1 = (1 * NSLS + n) * a.mstride_o + g;
      const long long i2 = (2 * NSLS + n) * a.mstride + g, o2 = (2 * NSLS + n) * a.mstride_o + g;
      const T mxx = a.m[i0], mzz = a.m[i1], mxz = a.m[i2];
      a.m_o[o0] = mxx + dt * (a.a1[n] * rxx + a.a2[n] * mxx);
      a.m_o[o1] = surf ? T(0) : mzz + dt * (a.a1[n] * rzz + a.a2[n] * mzz);
      a.m_o[o2] = mxz + dt * (a.a1[n] * rxz + a.a2[n] * mxz);
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
    s_sxx[si] = sxx;  // the tile's own stresses are not read by others after step 2
    s_szz[si] = szz;
    s_sxz[si] = sxz;
  }

  // 5. stress images above the free surface
  if (x.fs && z0 == L) {
    __syncthreads();
    for (int lx = tid; lx < TX; lx += NT) {
      const int gi = x0 + lx;
      if (gi >= xe) continue;
#pragma unroll
      for (int k = 1; k <= L; ++k)
        a.szz_o[(long long)(L - k) * nx + gi] = -s_szz[(HS + k) * SW + lx + HS];
#pragma unroll
      for (int k = 0; k < L; ++k)
        a.sxz_o[(long long)(L - 1 - k) * nx + gi] = -s_sxz[(HS + k) * SW + lx + HS];
    }
  }
}

template <typename T, int KIND, int NSLS>
static int launch_fused(const StepArgs<T> &a, const FusedExtras<T> &x, int ntiles, cudaStream_t st) {
  using G = FusedGeom<KIND>;
  constexpr size_t smem = sizeof(T) * G::smem_elems;
  static std::atomic<unsigned long long> attr_set{0};  // one bit per device set up (any thread)
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && !(attr_set & (1ULL << dev))) {
    cudaError_t e = cudaFuncSetAttribute(k_fused<T, KIND, NSLS>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_check(e, "fused kernel smem attribute");
    attr_set |= 1ULL << dev;
  }
  k_fused<T, KIND, NSLS><<<ntiles, G::NT, smem, st>>>(a, x);
  return VI_OK;
}

template <typename T>
static int launch_fused_dispatch(int kind, const StepArgs<T> &a, const FusedExtras<T> &x,
                                 int ntiles, cudaStream_t st) {
#define VB_CASE(K, N) \
  if (kind == K && a.nsls == N) return launch_fused<T, K, N>(a, x, ntiles, st);
#define VB_KIND(K) VB_CASE(K, 0) VB_CASE(K, 1) VB_CASE(K, 2) VB_CASE(K, 3) VB_CASE(K, 4) VB_CASE(K, 5)
  VB_KIND(VI_MEDIUM_ISO)
  VB_KIND(VI_MEDIUM_VTI)
  VB_KIND(VI_MEDIUM_TTI)
#undef VB_KIND
#undef VB_CASE
  return set_error(VI_ERR_ARG, "unsupported medium / nsls combination");
}

// Builds the per-tile CSR list of sources and receivers for a TX x TZ
// tiling whose recomputed-velocity halo is HV cells.  Force sources are
// listed for every tile whose halo covers them; explosive sources and
// receivers only for the owning tile.
void build_tile_lists(int nx, int nz, int TX, int TZ, int HV, const vi_shot *s,
                      std::vector<int> &off, std::vector<int4> &ent, int &ntx, int &ntz) {
  ntx = (nx - 2 * L + TX - 1) / TX;
  ntz = (nz - 2 * L + TZ - 1) / TZ;
  const int ntiles = ntx * ntz;
  std::vector<std::vector<int4>> per(ntiles);
  auto own_tile = [&](int i, int j) { return ((j - L) / TZ) * ntx + (i - L) / TX; };
  if (s) {
    for (int q = 0; q < s->nsrc; ++q) {
      const vi_source &v = s->src_host[q];
      if (v.kind == VI_SRC_EXPLOSIVE) {
        per[own_tile(v.i, v.j)].push_back(make_int4(v.i, v.j, q, TL_EXPLOSIVE));
        continue;
      }
      const int kind = v.kind == VI_SRC_FORCE_X ? TL_FORCE_X : TL_FORCE_Z;
      const int bx0 = (v.i - L - HV) / TX - 1, bx1 = (v.i - L + HV) / TX;
      const int bz0 = (v.j - L - HV) / TZ - 1, bz1 = (v.j - L + HV) / TZ;
      for (int bz = bz0 < 0 ? 0 : bz0; bz <= bz1 && bz < ntz; ++bz)
        for (int bx = bx0 < 0 ? 0 : bx0; bx <= bx1 && bx < ntx; ++bx) {
          const int x0 = L + bx * TX, z0 = L + bz * TZ;
          if (v.i >= x0 - HV && v.i < x0 + TX + HV && v.j >= z0 - HV && v.j < z0 + TZ + HV)
            per[bz * ntx + bx].push_back(make_int4(v.i, v.j, q, kind));
        }
    }
    for (int r = 0; r < s->nrec; ++r) {
      const vi_receiver &v = s->rec_host[r];
      per[own_tile(v.i, v.j)].push_back(make_int4(v.i, v.j, r, TL_RECEIVER));
    }
  }
  off.assign(ntiles + 1, 0);
  ent.clear();
  for (int t = 0; t < ntiles; ++t) {
    // by kind (force, explosive, receiver), in their original order within
    // a kind: a loop over one kind stops at the first entry of the next
    std::stable_sort(per[t].begin(), per[t].end(), [](const int4 &u, const int4 &v) { return u.w < v.w; });
    off[t] = (int)ent.size();
    ent.insert(ent.end(), per[t].begin(), per[t].end());
  }
  off[ntiles] = (int)ent.size();
}

int stage_tile_lists(vi_plan *p, const std::vector<int> &off, const std::vector<int4> &ent,
                     cudaStream_t st, int **d_off, int4 **d_ent) {
  const size_t ent_off = (off.size() * sizeof(int) + 15) / 16 * 16;
  const size_t lbytes = ent_off + ent.size() * sizeof(int4) + 16;
  int rc = ensure_buffer(p, &p->tile_lists, &p->tile_lists_bytes, lbytes);
  if (rc) return rc;
  *d_off = (int *)p->tile_lists;
  *d_ent = (int4 *)((char *)p->tile_lists + ent_off);
  rc = cuda_check(cudaMemcpyAsync(*d_off, off.data(), off.size() * sizeof(int), cudaMemcpyHostToDevice, st),
                  "copy tile offsets");
  if (rc) return rc;
  if (!ent.empty()) {
    rc = cuda_check(cudaMemcpyAsync(*d_ent, ent.data(), ent.size() * sizeof(int4), cudaMemcpyHostToDevice, st),
                    "copy tile entries");
    if (rc) return rc;
  }
  // the host vectors die at return: wait for the pageable copies
  return cuda_check(cudaStreamSynchronize(st), "stage tile lists");
}

static bool aligned16(const void *ptr) { return ((uintptr_t)ptr & 15) == 0; }

// Tensor maps of one ping-pong parity: the input state (sigma, v, M) and the
// medium.
template <typename T>
int encode_parity(TmaMaps &m, const TmaBoxes &b, const vi_config &c, T *const in[5],
                         const T *min, long long mstride, const StepArgs<T> &a) {
  const int e = sizeof(T), nx = c.nx, nz = c.nz;
  int rc;
  if ((rc = encode_map(&m.sxx, in[2], e, nx, nz, 1, 0, b.SWp, b.SH, 1))) return rc;
  if ((rc = encode_map(&m.szz, in[3], e, nx, nz, 1, 0, b.SWp, b.SH, 1))) return rc;
  if ((rc = encode_map(&m.sxz, in[4], e, nx, nz, 1, 0, b.SWp, b.SH, 1))) return rc;
  if ((rc = encode_map(&m.vx, in[0], e, nx, nz, 1, 0, b.VWp, b.VH, 1))) return rc;
  if ((rc = encode_map(&m.vz, in[1], e, nx, nz, 1, 0, b.VWp, b.VH, 1))) return rc;
  if ((rc = encode_map(&m.rho, a.rho, e, nx, nz, 1, 0, b.RWp, b.RH, 1))) return rc;
  if (c.nsls > 0) {
    if ((rc = encode_map(&m.m, min, e, nx, nz, b.NM, mstride, b.MW, b.MH, b.NM))) return rc;
    const bool tti = c.medium == VI_MEDIUM_TTI;
    if ((rc = encode_map(&m.tau, a.tau, e, nx, nz, 1, 0, tti ? b.MW : b.CW, tti ? b.MH : b.CH, 1)))
      return rc;
  }
  const T *slots[6];
  int n = 0;
  if (c.medium == VI_MEDIUM_ISO) {
    slots[n++] = a.c13;
    slots[n++] = a.c55;
  } else if (c.medium == VI_MEDIUM_VTI) {
    slots[n++] = a.c11;
    slots[n++] = a.c13;
    slots[n++] = a.c33;
    slots[n++] = a.c55;
  } else {
    slots[n++] = a.c11;
    slots[n++] = a.c13;
    slots[n++] = a.c15;
    slots[n++] = a.c33;
    slots[n++] = a.c35;
    slots[n++] = a.c55;
  }
  for (int k = 0; k < n; ++k)
    if ((rc = encode_map(&m.c[k], slots[k], e, nx, nz, 1, 0, b.CW, b.CH, 1))) return rc;
  return VI_OK;
}

template <typename T>
int fused_steps(vi_plan *p, StepArgs<T> a, const vi_shot *s, int it0, int nsteps,
                cudaStream_t st, int mode) {
  const vi_config &c = p->cfg;
  const int kind = c.medium;
  const size_t np = (size_t)c.nx * c.nz;
  const int nstate = 5 + 3 * c.nsls;
  if (nsteps == 0) return VI_OK;
  if (c.free_surface && c.nz - 2 * L < L + 1)
    return set_error(VI_ERR_ARG, "free surface needs at least 5 rows in the update region");
  // second state copy, zero outside the update region (only ever written inside it)
  if (!p->alt) {
    size_t have = 0;
    int rc = ensure_buffer(p, &p->alt, &have, nstate * np * sizeof(T));
    if (rc) return rc;
    rc = cuda_check(cudaMemsetAsync(p->alt, 0, nstate * np * sizeof(T), st), "zero alt state");
    if (rc) return rc;
  }
  T *user[5] = {a.vx, a.vz, a.sxx, a.szz, a.sxz};
  T *user_m = a.m;
  const long long user_ms = a.mstride;
  T *alt = (T *)p->alt;
  T *alt_st[5];
  for (int q = 0; q < 5; ++q) alt_st[q] = alt + q * np;

  // TMA eligibility: 16-byte aligned rows, planes and bases
  const bool persist = mode != 4;
  const TmaBoxes bx = tma_boxes(kind, c.nsls, (int)sizeof(T), persist);
  // (4-cell groups never straddle the update-region edge when nx % 4 == 0)
  bool use_tma = mode != 2 && bx.ok && c.nx % 4 == 0 && ((size_t)c.nx * sizeof(T)) % 16 == 0 &&
                 (np * sizeof(T)) % 16 == 0;
  const void *ptrs[] = {user[0], user[1], user[2], user[3], user[4], a.rho, a.c11, a.c13,
                        a.c15,   a.c33,   a.c35,   a.c55,   a.tau,   user_m};
  for (const void *q : ptrs)
    if (q && !aligned16(q)) use_tma = false;
  if (c.nsls > 0 && ((size_t)user_ms * sizeof(T)) % 16 != 0) use_tma = false;
  if ((mode == 3 || mode == 4) && !use_tma)
    return set_error(VI_ERR_ARG, "TMA-staged step needs 16-byte aligned rows and planes");

  int TX, TZ, HV;
  if (use_tma) {
    TX = bx.TX;
    TZ = bx.TZ;
    HV = bx.HV;
  } else if (kind == VI_MEDIUM_TTI) {
    TX = FusedGeom<VI_MEDIUM_TTI>::TX;
    TZ = FusedGeom<VI_MEDIUM_TTI>::TZ;
    HV = FusedGeom<VI_MEDIUM_TTI>::HV;
  } else {
    TX = FusedGeom<VI_MEDIUM_ISO>::TX;
    TZ = FusedGeom<VI_MEDIUM_ISO>::TZ;
    HV = FusedGeom<VI_MEDIUM_ISO>::HV;
  }
  int ntx, ntz;
  std::vector<int> off;
  std::vector<int4> ent;
  build_tile_lists(c.nx, c.nz, TX, TZ, HV, s, off, ent, ntx, ntz);
  const int ntiles = ntx * ntz;
  int *d_off = nullptr;
  int4 *d_ent = nullptr;
  int rc = stage_tile_lists(p, off, ent, st, &d_off, &d_ent);
  if (rc) return rc;

  TmaMaps maps[2];
  if (use_tma) {
    if ((rc = encode_parity<T>(maps[0], bx, c, user, user_m, user_ms, a))) return rc;
    if ((rc = encode_parity<T>(maps[1], bx, c, alt_st, alt + 5 * np, (long long)np, a))) return rc;
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

  T *psix0 = (T *)p->psix, *psiz0 = (T *)p->psiz;
  for (int k = 0; k < nsteps; ++k) {
    const bool from_user = (k % 2) == 0;
    T *const *in = from_user ? user : alt_st;
    T *const *out = from_user ? alt_st : user;
    a.vx = in[0]; a.vz = in[1]; a.sxx = in[2]; a.szz = in[3]; a.sxz = in[4];
    a.vx_o = out[0]; a.vz_o = out[1]; a.sxx_o = out[2]; a.szz_o = out[3]; a.sxz_o = out[4];
    a.m = from_user ? user_m : alt + 5 * np;
    a.mstride = from_user ? user_ms : (long long)np;
    a.m_o = from_user ? alt + 5 * np : user_m;
    a.mstride_o = from_user ? (long long)np : user_ms;
    const int cur = p->psi_cur;
    a.psix = psix0 ? psix0 + cur * kPsiPerSet * p->psix_plane : nullptr;
    a.psix_o = psix0 ? psix0 + (1 - cur) * kPsiPerSet * p->psix_plane : nullptr;
    a.psiz = psiz0 ? psiz0 + cur * kPsiPerSet * p->psiz_plane : nullptr;
    a.psiz_o = psiz0 ? psiz0 + (1 - cur) * kPsiPerSet * p->psiz_plane : nullptr;
    x.it = it0 + k;
    rc = use_tma ? launch_fused_tma<T>(kind, a, x, maps[from_user ? 0 : 1], ntiles, p->nsm, persist, st)
                 : launch_fused_dispatch<T>(kind, a, x, ntiles, st);
    if (rc) return rc;
    p->psi_cur = 1 - cur;
  }
  if (nsteps % 2 == 1) {
    // result sits in the plan's copy: bring it back to the caller's fields
    for (int q = 0; q < 5; ++q) {
      rc = cuda_check(cudaMemcpyAsync(user[q], alt_st[q], np * sizeof(T), cudaMemcpyDeviceToDevice, st),
                      "copy back fields");
      if (rc) return rc;
    }
    for (int q = 0; q < 3 * c.nsls; ++q) {
      rc = cuda_check(cudaMemcpyAsync(user_m + q * user_ms, alt + (5 + q) * np, np * sizeof(T),
                                      cudaMemcpyDeviceToDevice, st),
                      "copy back memory variables");
      if (rc) return rc;
    }
  }
  p->last_used_tma = use_tma;
  return VI_OK;
}

template int encode_parity<float>(TmaMaps &, const TmaBoxes &, const vi_config &, float *const[5],
                                  const float *, long long, const StepArgs<float> &);
template int encode_parity<double>(TmaMaps &, const TmaBoxes &, const vi_config &, double *const[5],
                                   const double *, long long, const StepArgs<double> &);
template int fused_steps<float>(vi_plan *, StepArgs<float>, const vi_shot *, int, int, cudaStream_t, int);
template int fused_steps<double>(vi_plan *, StepArgs<double>, const vi_shot *, int, int, cudaStream_t, int);

}  // namespace vb
