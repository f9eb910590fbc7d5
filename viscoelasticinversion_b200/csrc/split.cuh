// split.cuh — geometry and host interface of the two-kernel (velocity,
// stress) in-place step for ISO and VTI media.
#pragma once

#include <cuda.h>

#include "common.cuh"
#include "fused.cuh"
#include "fused_tma.cuh"

struct vi_plan;

namespace vb {

template <typename T>
struct SplitGeom {
  static constexpr int TX = 64, TZ = 8, NT = TX / 4 * TZ;  // one 4-cell group per thread
  static constexpr int BW = TX + 8, BH = TZ + 8;    // staged box: tile + 4-cell halo
  static constexpr int PB =
      (int)(((long long)BW * BH * (long long)sizeof(T) + 127) / 128 * 128 / (long long)sizeof(T));
  static constexpr int O0 = 128 / (int)sizeof(T);  // after the barrier slot
  static constexpr int BOX_BYTES = BW * BH * (int)sizeof(T);
  static constexpr int SMEM_STRESS = 128 + 2 * PB * (int)sizeof(T);
};

// Tiling of the stress kernel: TX_ x TZ_ cells, one 4-cell group per
// thread, the new velocities staged as a TMA box with a 4-cell halo.  The
// single-shot step uses 128 x 2 tiles (their rows are 512-byte runs of each
// of the ~30 planes the pass streams: 54.5 vs 55.9 us per 2048 x 1024 VTI
// step for 64 x 8, 54.8 for 128 x 4, 58.2 for 128 x 8); the merged batch
// kernels keep 64 x 8, the tiling of their shared tile lists.
template <typename T, int TX_, int TZ_>
struct SplitStressGeomT {
  static constexpr int TX = TX_, TZ = TZ_, NT = TX / 4 * TZ;
  static constexpr int BW = TX + 8, BH = TZ + 8;
  static constexpr int PB =
      (int)(((long long)BW * BH * (long long)sizeof(T) + 127) / 128 * 128 / (long long)sizeof(T));
  static constexpr int O0 = 128 / (int)sizeof(T);
  static constexpr int BOX_BYTES = BW * BH * (int)sizeof(T);
  static constexpr int SMEM = 128 + 2 * PB * (int)sizeof(T);
};
template <typename T>
using SplitStressGeom = SplitStressGeomT<T, 128, 2>;
template <typename T>
using SplitStressGeomBatch = SplitStressGeomT<T, 64, 8>;

// Tiling of the TTI stress kernel: TX_ x TZ_ cells; the effective rates are
// computed on the tile and a one-cell ring (4-aligned: EW x EH), from a TMA
// box of the new velocities with the ring's 4-cell stencil halo (BW x BH).
// Single shot 128 x 4 (73.8 vs 75.6 us per 2048 x 1024 TTI step for
// 64 x 8); the merged batch kernels keep 64 x 8.
template <typename T, int TX_, int TZ_>
struct SplitTtiGeomT {
  static constexpr int TX = TX_, TZ = TZ_, NT = TX / 4 * TZ;
  static constexpr int BW = TX + 16, BH = TZ + 10;
  static constexpr int EW = TX + 8, EH = TZ + 2;
  static constexpr int PB =
      (int)(((long long)BW * BH * (long long)sizeof(T) + 127) / 128 * 128 / (long long)sizeof(T));
  static constexpr int PE =
      (int)(((long long)EW * EH * (long long)sizeof(T) + 127) / 128 * 128 / (long long)sizeof(T));
  static constexpr int O0 = 128 / (int)sizeof(T);
  static constexpr int BOX_BYTES = BW * BH * (int)sizeof(T);
  static constexpr int SMEM = 128 + (2 * PB + 3 * PE) * (int)sizeof(T);
  static constexpr int NRING = 2 * (EW / 4) + 2 * TZ;  // ring groups: 2 rows + 2 columns
  static_assert(NRING <= NT, "one ring group per thread at most");
};
template <typename T>
using SplitTtiGeom = SplitTtiGeomT<T, 128, 4>;
template <typename T>
using SplitTtiGeomBatch = SplitTtiGeomT<T, 64, 8>;

// TMA maps of the staged planes: (sxx, szz, sxz) for the velocity kernel,
// (vx, vz) for the stress kernel.
struct SplitMaps {
  CUtensorMap a, b, c;
};

template <typename T>
int launch_split_vel(const StepArgs<T> &a, const FusedExtras<T> &x, int ntiles, cudaStream_t st,
                     bool pdl);
template <typename T>
int launch_split_stress(int kind, const StepArgs<T> &a, const FusedExtras<T> &x,
                        const SplitMaps &m, int ntiles, cudaStream_t st, bool pdl);
// The split pair over the tiles of many shots (BatchDev, per-shot v-box
// maps in smaps): item i of a launch is the tile batch_locate gives.
// afda: some shot of the batch has the H-AFDA free surface
template <typename T>
int launch_split_vel_batch(int kind, bool afda, const BatchDev<T> &b, int it, int nitems, cudaStream_t st,
                           bool pdl);
// comp: the shots are compensated FP32 (VI_F32C: stress residues in
// args.slo); afda: some shot has the H-AFDA free surface
template <typename T>
int launch_split_stress_batch(int kind, int nsls, bool comp, bool afda, const BatchDev<T> &b, int it, int nitems,
                              cudaStream_t st, bool pdl);
template <typename T>
int launch_split_stress_tti_batch(int nsls, bool comp, bool afda, const BatchDev<T> &b, int it, int nitems,
                                  cudaStream_t st, bool pdl);

// TTI stress pass: reads M (a.m) and psi (a.psix/psiz) of the tile and its
// ring, writes them to a.m_o and a.psix_o/psiz_o (must differ from the
// inputs); sigma in place.
template <typename T>
int launch_split_stress_tti(const StepArgs<T> &a, const FusedExtras<T> &x, const SplitMaps &m,
                            int ntiles, cudaStream_t st, bool pdl);

// TMA maps of the pipelined split kernels: velocity (sxx, szz, sxz boxes,
// vx, vz, rho tiles); stress (vx, vz boxes, sxx, szz, sxz tiles, M, then the
// coefficient slots and tau).
struct SplitPMaps {
  CUtensorMap m[11];
};
template <typename T>
int launch_split_vel_p(const StepArgs<T> &a, const FusedExtras<T> &x, const SplitPMaps &m,
                       int ntiles, int nsm, cudaStream_t st);
template <typename T>
int launch_split_stress_p(int kind, const StepArgs<T> &a, const FusedExtras<T> &x,
                          const SplitPMaps &m, int ntiles, int nsm, cudaStream_t st);
template <typename T>
int encode_split_p(const vi_config &c, const StepArgs<T> &a, SplitPMaps &mv, SplitPMaps &ms);
bool split_p_fits(int kind, int nsls, int esize);
void split_p_tiles(int &vtx, int &vtz, int &stx, int &stz);

// Runs nsteps split steps in place on the caller's fields, with the
// one-tile-per-CTA kernels or (pipelined) the persistent TMA-pipelined
// kernels.  Returns VI_ERR_ARG (without side effects) when the
// configuration is not eligible (TTI, nx % 4 != 0 or unaligned planes).
// Velocity pass of split_steps: TMA-staged stress taps (default), direct
// L1 loads, or the persistent TMA-pipelined pair (ISO/VTI).
enum SplitMode { kSplitVelTma = 0, kSplitLdg = 1, kSplitPipelined = 2 };
template <typename T>
int split_steps(vi_plan *p, StepArgs<T> a, const vi_shot *s, int it0, int nsteps, cudaStream_t st,
                int mode);

// The time-blocked form of the split pair (wave.cu): one persistent
// kernel runs sweeps of k steps as a wavefront over 8-row bands, with a
// lag of d bands between consecutive passes (plan's wave_k / wave_d, 0 =
// these defaults).  ISO/VTI, imaging or no free surface, FP32 or FP64 (not
// VI_F32C); same eligibility as split_steps otherwise.
constexpr int kWaveDefaultK = 4, kWaveDefaultD = 8;
bool wave_eligible_cfg(const vi_config &c);
template <typename T>
int wave_steps(vi_plan *p, StepArgs<T> a, const vi_shot *s, int it0, int nsteps, cudaStream_t st);

// true when split_steps can run this plan and these pointers
template <typename T>
bool split_eligible(const vi_plan *p, const StepArgs<T> &a);

}  // namespace vb
