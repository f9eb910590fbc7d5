// wave.cu — the time-blocked split step: one persistent kernel runs the
// velocity and stress passes of many time steps as a wavefront over bands
// of the grid, so a band's state is re-read from L2 by the next steps
// instead of from HBM.
//
// The grid's update region is cut into bands of 8 rows: one row of 64 x 8
// velocity tiles, two rows of 128 x 4 stress tiles.  A unit of work is one
// tile of one pass q = 2 (s - s0) + p (p = 0 velocity, 1 stress) of a time
// step s of a sweep of K steps starting at s0.  Within a sweep the units
// are ordered by the virtual time tau = b + D q (b the band, D the lag in
// bands between consecutive passes), so band b is visited by the sweep's K
// steps at tau = b, b + 2D, ..., while the bands touched in between (about
// 4 D K band-passes) stay in L2; sweeps follow each other.  A CTA takes the
// next unit from a global ticket counter, waits until the units it reads
// are complete, runs the same tile code as the one-launch-per-pass split
// pair (split_tiles.cuh: bitwise equal results) and counts the unit done
// for its band:
//   velocity (s, b) reads sigma of bands b-1..b+1 written by stress (s-1)
//     and overwrites v, which stress (s-1) of those bands reads;
//   stress (s, b) reads v of bands b-1..b+1 written by velocity (s) and
//     overwrites sigma, which velocity (s) of those bands reads;
// so each waits for the other pass's three neighbouring bands; own-cell
// state (v, sigma, M, psi) follows by transitivity.  Every dependency has
// an earlier ticket (D >= 2), tickets are taken in order by running CTAs,
// so the unit with the smallest outstanding ticket can always proceed: no
// co-residency is assumed.  Each wait is bounded; a wait that gives up
// sets the plan's error word and an abort flag the other CTAs poll, and
// the kernel returns.
//
// The per-band completion counters grow monotonically within a launch
// (a band's units of step s+1 start only after all of step s's are done),
// so "m passes of band b complete" is done[p][b] >= m * units(p, b).
// Producer: stores, barrier, then one thread's gpu-scope fence and
// increment; consumer: one thread's acquire load, a proxy fence for its TMA
// loads, then a barrier.  ISO/VTI media, FP32 and FP64, imaging or no
// free surface; the H-AFDA surface, compensated FP32 and TTI run on the
// split pair.
#include <atomic>
#include <climits>
#include <cstdint>
#include <vector>

#include "nvtx.cuh"
#include "plan.cuh"
#include "split.cuh"
#include "split_tiles.cuh"

namespace vb {

constexpr int kWaveBand = 8;  // rows per band: one velocity tile row
constexpr int kWaveThreads = 128;
template <typename T>
using WaveVelGeom = SplitVelTmaT<T, kWaveBand>;
template <typename T>
using WaveStressGeom = SplitStressGeomT<T, 128, kWaveBand / 2>;
static_assert(WaveVelGeom<float>::NT == kWaveThreads && WaveStressGeom<float>::NT == kWaveThreads,
              "both passes run on CTAs of the same size");
static_assert(WaveVelGeom<float>::TZ == kWaveBand && 2 * WaveStressGeom<float>::TZ == kWaveBand,
              "a band is one velocity tile row and two stress tile rows");
constexpr int kWaveCtlPad = 8;        // ints per counter (one 32-byte sector each)
constexpr int kWaveCtlHead = 32;      // ticket, abort flag
constexpr unsigned kWaveSpin = 1u << 22;  // polls of one dependency before giving up
constexpr int kWaveMaxSmem = 96 * 1024;   // tile staging + the sweep's prefix tables

struct WaveSched {
  int nb;            // bands
  int ntx_v, ntx_s;  // velocity / stress tiles per tile row
  int ntz_s;         // stress tile rows
  int slots;         // tickets per band-pass: max(ntx_v, 2 ntx_s)
  int k, d;          // steps per sweep, band lag between passes
  int it0, nsteps;
  int nfull;         // full sweeps (k steps each)
  long long per_full;  // band-passes of a full sweep: 2 k nb
  int *ctl;          // [0] ticket, [1] abort, then done[2][nb] (padded)
};

// band-passes of a sweep of 2k passes ordered before virtual time tau
__device__ __forceinline__ int wave_before(int tau, int twok, int d, int nb) {
  int s = 0;
  for (int q = 0; q < twok; ++q) s += min(max(tau - d * q, 0), nb);
  return s;
}

__device__ __forceinline__ int wave_units(const WaveSched &w, int p, int b) {
  return p == 0 ? w.ntx_v : w.ntx_s * min(2, w.ntz_s - 2 * b);
}

__device__ __forceinline__ int ld_acquire_gpu(const int *p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Prefix table of a sweep of 2k passes: tab[tau] = band-passes ordered
// before virtual time tau (wave_before), tau = 0 .. wave_tab_len - 1.
__host__ __device__ inline int wave_tab_len(int nb, int twok, int d) { return nb + d * (twok - 1) + 1; }

// Unit of ticket t (< 2^31): pass p of step s on band b, tile slot u.
// tabf / tabp: prefix tables of the full sweeps and of the last, shorter
// one.  False when the ticket names no unit (a slot beyond the band's
// tiles).
__device__ __forceinline__ bool wave_decode(const WaveSched &w, unsigned t, const int *tabf, const int *tabp,
                                            int &s, int &p, int &b, int &u) {
  const unsigned r = t / (unsigned)w.slots;
  u = (int)(t - r * (unsigned)w.slots);
  const unsigned full = (unsigned)w.nfull * (unsigned)w.per_full;
  const unsigned sweep = r < full ? r / (unsigned)w.per_full : (unsigned)w.nfull;
  const int rr = (int)(r - sweep * (unsigned)w.per_full);
  const int ks = sweep < (unsigned)w.nfull ? w.k : w.nsteps - w.nfull * w.k;
  const int twok = 2 * ks;
  if (ks <= 0 || rr >= twok * w.nb) return false;
  const int *tab = sweep < (unsigned)w.nfull ? tabf : tabp;
  // the largest tau with tab[tau] <= rr
  int lo = 0, hi = wave_tab_len(w.nb, twok, w.d) - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (tab[mid] <= rr) lo = mid;
    else hi = mid - 1;
  }
  const int tau = lo;
  const int qlo = tau - w.nb + 1 > 0 ? (tau - w.nb + 1 + w.d - 1) / w.d : 0;
  const int q = qlo + (rr - tab[tau]);
  b = tau - w.d * q;
  s = w.it0 + (int)sweep * w.k + q / 2;
  p = q & 1;
  return u < wave_units(w, p, b);
}

// Shared memory of the tile code (its barrier slot first), then the two
// prefix tables.
template <typename T>
__host__ __device__ constexpr int wave_tile_smem() {
  return WaveVelGeom<T>::SMEM > WaveStressGeom<T>::SMEM ? WaveVelGeom<T>::SMEM : WaveStressGeom<T>::SMEM;
}

template <typename T, int KIND, int NSLS>
__global__ void __launch_bounds__(kWaveThreads, (sizeof(T) == 4 ? 512 : 256) / kWaveThreads)
    k_wave(const __grid_constant__ StepArgs<T> a, const __grid_constant__ FusedExtras<T> xv,
           const __grid_constant__ FusedExtras<T> xs, const __grid_constant__ SplitMaps mv,
           const __grid_constant__ SplitMaps ms, const __grid_constant__ WaveSched w, unsigned total) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem_raw);  // the tile code's barrier slot
  int *tabf = reinterpret_cast<int *>(smem_raw + wave_tile_smem<T>());
  const int lenf = wave_tab_len(w.nb, 2 * w.k, w.d);
  int *tabp = tabf + lenf;
  const int kp = w.nsteps - w.nfull * w.k, lenp = kp > 0 ? wave_tab_len(w.nb, 2 * kp, w.d) : 0;
  __shared__ int s_unit[5];  // go, s, p, b, u
  unsigned long long *ticket = reinterpret_cast<unsigned long long *>(w.ctl);
  volatile int *abort_flag = w.ctl + 2;
  const int tid = threadIdx.x, lane = tid & 31;
  for (int i = tid; i < lenf + lenp; i += kWaveThreads)
    tabf[i] = i < lenf ? wave_before(i, 2 * w.k, w.d, w.nb) : wave_before(i - lenf, 2 * kp, w.d, w.nb);
  __syncthreads();
  unsigned next = 0;
  if (tid == 0) next = (unsigned)atomicAdd(ticket, 1ULL);
  for (;;) {
    if (tid < 32) {
      int go = 0, s = 0, p = 0, b = 0, u = 0;
      if (lane == 0) {
        while (next < total && !*abort_flag) {
          const unsigned t = next;
          next = (unsigned)atomicAdd(ticket, 1ULL);  // the following ticket, fetched ahead
          if (wave_decode(w, t, tabf, tabp, s, p, b, u)) {
            go = 1;
            break;
          }
        }
      }
      go = __shfl_sync(0xffffffffu, go, 0);
      s = __shfl_sync(0xffffffffu, s, 0);
      p = __shfl_sync(0xffffffffu, p, 0);
      b = __shfl_sync(0xffffffffu, b, 0);
      // lanes 0..2 poll the other pass's bands b-1, b, b+1 at once: m
      // passes of each complete
      const int o = 1 - p, m = p == 0 ? s - w.it0 : s - w.it0 + 1, bb = b - 1 + lane;
      const bool mine = go && m > 0 && lane < 3 && bb >= 0 && bb < w.nb;
      const int *c = w.ctl + kWaveCtlHead + (o * w.nb + (mine ? bb : 0)) * kWaveCtlPad;
      const int target = mine ? m * wave_units(w, o, bb) : 0;
      unsigned n = 0;
      for (;;) {
        const bool ok = !mine || ld_acquire_gpu(c) >= target;
        if (__all_sync(0xffffffffu, ok)) break;
        if (__any_sync(0xffffffffu, *abort_flag != 0) || ++n >= kWaveSpin) {
          if (lane == 0 && n >= kWaveSpin) {
            atomicOr(xv.err, kErrTimeout);
            atomicExch(w.ctl + 2, 1);
          }
          go = 0;
          break;
        }
        __nanosleep(64);
      }
      if (lane == 0) {
        s_unit[0] = go;
        s_unit[1] = s;
        s_unit[2] = p;
        s_unit[3] = b;
        s_unit[4] = u;
      }
    }
    __syncthreads();
    if (!s_unit[0]) break;
    const int s = s_unit[1], p = s_unit[2], b = s_unit[3], u = s_unit[4];
    if (tid == 0) fence_proxy_async();  // the acquired sigma / v before this thread's TMA loads of them
    if (p == 0) {
      FusedExtras<T> x = xv;
      x.it = s;
      const int tile = b * w.ntx_v + u;
      split_vel_tma_tile<T, false, false, false, WaveVelGeom<T>>(a, x, mv, tile);
      split_vel_sample<T>(a, x, tile);
    } else {
      FusedExtras<T> x = xs;
      x.it = s;
      split_stress_tile<T, KIND, NSLS, false, false, false, false, WaveStressGeom<T>, true>(
          a, x, ms, 2 * b * w.ntx_s + u);
    }
    __syncthreads();  // every store of the unit issued, every read of its staging done
    if (tid == 0) {
      mbar_inval(bar);
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // before the next unit's TMA writes
      __threadfence();
      atomicAdd(w.ctl + kWaveCtlHead + (p * w.nb + b) * kWaveCtlPad, 1);
      if (*(volatile int *)xv.err & kErrTimeout) atomicExch(w.ctl + 2, 1);
    }
  }
}

// ------------------------------------------------------------------- host
template <typename T, int KIND, int NSLS>
static int launch_wave_k(const StepArgs<T> &a, const FusedExtras<T> &xv, const FusedExtras<T> &xs,
                         const SplitMaps &mv, const SplitMaps &ms, const WaveSched &w, unsigned total,
                         int nsm, cudaStream_t st) {
  const int kp = w.nsteps - w.nfull * w.k;
  const int tab = wave_tab_len(w.nb, 2 * w.k, w.d) + (kp > 0 ? wave_tab_len(w.nb, 2 * kp, w.d) : 0);
  const size_t smem = (size_t)wave_tile_smem<T>() + (size_t)tab * sizeof(int);
  static std::atomic<unsigned long long> attr_set{0};  // one bit per device set up (any thread)
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && !(attr_set & (1ULL << dev))) {
    cudaError_t e = cudaFuncSetAttribute(k_wave<T, KIND, NSLS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         kWaveMaxSmem);
    if (e != cudaSuccess) return cuda_check(e, "wave smem attribute");
    attr_set |= 1ULL << dev;
  }
  if (smem > (size_t)kWaveMaxSmem) return set_error(VI_ERR_ARG, "wavefront schedule too long for shared memory");
  int per_sm = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_wave<T, KIND, NSLS>, kWaveThreads, smem);
  if (e != cudaSuccess) return cuda_check(e, "wave occupancy");
  if (per_sm < 1) return set_error(VI_ERR_CUDA, "wavefront kernel does not fit an SM");
  const long long grid = std::min<long long>(total, (long long)per_sm * nsm);
  k_wave<T, KIND, NSLS><<<(unsigned)grid, kWaveThreads, smem, st>>>(a, xv, xs, mv, ms, w, total);
  return cuda_check(cudaGetLastError(), "wave launch");
}

template <typename T>
static int launch_wave(int kind, const StepArgs<T> &a, const FusedExtras<T> &xv, const FusedExtras<T> &xs,
                       const SplitMaps &mv, const SplitMaps &ms, const WaveSched &w, unsigned total, int nsm,
                       cudaStream_t st) {
#define VB_CASE(K, N) \
  if (kind == K && a.nsls == N) return launch_wave_k<T, K, N>(a, xv, xs, mv, ms, w, total, nsm, st);
#define VB_KIND(K) VB_CASE(K, 0) VB_CASE(K, 1) VB_CASE(K, 2) VB_CASE(K, 3) VB_CASE(K, 4) VB_CASE(K, 5)
  VB_KIND(VI_MEDIUM_ISO)
  VB_KIND(VI_MEDIUM_VTI)
#undef VB_KIND
#undef VB_CASE
  return set_error(VI_ERR_ARG, "the wavefront step covers ISO and VTI media");
}

bool wave_eligible_cfg(const vi_config &c) {
  return c.medium != VI_MEDIUM_TTI && c.free_surface != kFsAfda && c.precision != VI_F32C && c.nsls <= 5;
}

template <typename T>
int wave_steps(vi_plan *p, StepArgs<T> a, const vi_shot *s, int it0, int nsteps, cudaStream_t st) {
  const vi_config &c = p->cfg;
  if (!split_eligible<T>(p, a))
    return set_error(VI_ERR_ARG, "wavefront step needs nx % 4 == 0 and 16-byte aligned planes");
  if (!wave_eligible_cfg(c))
    return set_error(VI_ERR_ARG, "the wavefront step covers ISO/VTI media without H-AFDA or VI_F32C");
  if (nsteps == 0) return VI_OK;
  const int k = p->wave_k > 0 ? p->wave_k : kWaveDefaultK, d = p->wave_d > 0 ? p->wave_d : kWaveDefaultD;
  if (d < 2) return set_error(VI_ERR_ARG, "wavefront band lag must be at least 2");
  using VG = WaveVelGeom<T>;
  using SG = WaveStressGeom<T>;
  int ntx, ntz, sntx, sntz;
  std::vector<int> off, soff;
  std::vector<int4> ent, sent;
  build_tile_lists(c.nx, c.nz, VG::TX, VG::TZ, 0, s, off, ent, ntx, ntz);
  build_tile_lists(c.nx, c.nz, SG::TX, SG::TZ, 0, s, soff, sent, sntx, sntz);
  const int nvoff = (int)off.size();
  for (int v : soff) off.push_back(v + (int)ent.size());
  ent.insert(ent.end(), sent.begin(), sent.end());
  int *d_off = nullptr;
  int4 *d_ent = nullptr;
  int rc = stage_tile_lists(p, off, ent, st, &d_off, &d_ent);
  if (rc) return rc;
  const int e = sizeof(T);
  SplitMaps ms, mv;
  if ((rc = encode_map(&ms.a, a.vx, e, c.nx, c.nz, 1, 0, SG::BW, SG::BH, 1))) return rc;
  if ((rc = encode_map(&ms.b, a.vz, e, c.nx, c.nz, 1, 0, SG::BW, SG::BH, 1))) return rc;
  ms.c = ms.b;
  if ((rc = encode_map(&mv.a, a.sxx, e, c.nx, c.nz, 1, 0, VG::WX, VG::TZ, 1))) return rc;
  if ((rc = encode_map(&mv.b, a.sxz, e, c.nx, c.nz, 1, 0, VG::WX, VG::HZ, 1))) return rc;
  if ((rc = encode_map(&mv.c, a.szz, e, c.nx, c.nz, 1, 0, VG::WZ, VG::HZ, 1))) return rc;
  FusedExtras<T> xv;
  xv.ntx = ntx;
  xv.fs = c.free_surface;
  xv.it = it0;
  xv.tile_off = d_off;
  xv.tile_ent = d_ent;
  xv.amp = (const T *)p->damp;
  xv.wavelet = (s && s->nsrc) ? (const T *)s->wavelet_dev : nullptr;
  xv.wnt = (s && s->nsrc) ? s->wavelet_nt : 0;
  xv.traces = (s && s->nrec) ? (T *)s->traces_dev : nullptr;
  xv.tnt = (s && s->nrec) ? s->traces_nt : 0;
  xv.nrec = s ? s->nrec : 0;
  xv.err = (int *)p->errflag;
  xv.l2hint = 0;
  FusedExtras<T> xs = xv;
  xs.ntx = sntx;
  xs.tile_off = d_off + nvoff;
  // in place on the current psi set
  if (a.psix) a.psix = a.psix_o = (T *)p->psix + p->psi_cur * kPsiPerSet * p->psix_plane;
  if (a.psiz) a.psiz = a.psiz_o = (T *)p->psiz + p->psi_cur * kPsiPerSet * p->psiz_plane;
  WaveSched w;
  w.nb = ntz;
  w.ntx_v = ntx;
  w.ntx_s = sntx;
  w.ntz_s = sntz;
  w.slots = std::max(ntx, 2 * sntx);
  w.d = d;
  const size_t ctl_bytes = (size_t)(kWaveCtlHead + 2 * w.nb * kWaveCtlPad) * sizeof(int);
  if ((rc = ensure_buffer(p, &p->wave_ctl, &p->wave_ctl_bytes, ctl_bytes))) return rc;
  w.ctl = (int *)p->wave_ctl;
  // tickets of one launch stay below 2^30: long runs on large grids take
  // several launches of whole sweeps
  const long long per_step = 2LL * w.nb * w.slots;
  const int kk = std::min(k, nsteps);
  const int chunk = (int)std::max<long long>(kk, (1LL << 30) / per_step / kk * kk);
  NvtxRange nr("vi_step: wavefront");
  for (int done = 0; done < nsteps; done += chunk) {
    const int n = std::min(chunk, nsteps - done);
    w.k = std::min(kk, n);
    w.it0 = it0 + done;
    w.nsteps = n;
    w.nfull = n / w.k;
    w.per_full = 2LL * w.k * w.nb;
    const int rem = n - w.nfull * w.k;
    const long long total = ((long long)w.nfull * w.per_full + 2LL * rem * w.nb) * w.slots;
    if (total >= (1LL << 31)) return set_error(VI_ERR_ARG, "wavefront schedule too large for one launch");
    if ((rc = cuda_check(cudaMemsetAsync(p->wave_ctl, 0, ctl_bytes, st), "zero wavefront counters"))) return rc;
    if ((rc = launch_wave<T>(c.medium, a, xv, xs, mv, ms, w, (unsigned)total, p->nsm, st))) return rc;
  }
  return VI_OK;
}

template int wave_steps<float>(vi_plan *, StepArgs<float>, const vi_shot *, int, int, cudaStream_t);
template int wave_steps<double>(vi_plan *, StepArgs<double>, const vi_shot *, int, int, cudaStream_t);

}  // namespace vb
