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
// (2048 x 1024 VTI: 29.4 vs 28.0 Gpt/s on B200).  In the velocity pass
// and the ISO/VTI stress pass only the thread that issues the TMA boxes
// waits first; the others issue their loads of state the running grid does
// not write (v and rho; sigma, M and the medium) before waiting: 54.5 ->
// 54.0 us per 2048 x 1024 VTI step, 17.1 -> 16.5 at 1024 x 512.  Releasing
// the next grid early (griddepcontrol.launch_dependents after the wait)
// measured slower (55.2), as did loads before the wait in every thread
// ahead of the TMA issue on the TTI stress pass (76.7 vs 73.4 us).
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
#include "split_tiles.cuh"
#include "vec.cuh"

namespace vb {


// AFDA: the grid has the H-AFDA free surface (a separate instantiation,
// so the others carry none of its code)
template <typename T, bool PP, bool HINT, bool AFDA>
__global__ void __launch_bounds__(SplitVelTma<T>::NT, (sizeof(T) == 4 ? 1024 : 512) / SplitVelTma<T>::NT)
    k_split_vel_tma(const __grid_constant__ StepArgs<T> a, const FusedExtras<T> x, const __grid_constant__ SplitMaps maps) {
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

template <typename T, int KIND, int NSLS, bool OOP, bool HINT, bool COMP, bool AFDA>
__global__ void __launch_bounds__(SplitStressGeom<T>::NT, (sizeof(T) == 4 ? 512 : 256) / SplitStressGeom<T>::NT)
    k_split_stress(const __grid_constant__ StepArgs<T> a, const __grid_constant__ FusedExtras<T> x,
                   const __grid_constant__ SplitMaps maps) {
  split_stress_tile<T, KIND, NSLS, OOP, HINT, COMP, AFDA, SplitStressGeom<T>, true>(a, x, maps, blockIdx.x);
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
