// fused.cuh — host interface of the fused single-kernel step.
#pragma once
#include <vector>

#include "common.cuh"

struct vi_plan;

namespace vb {

// Tile geometry of the fused kernel (shared by the kernel and the host-side
// source/receiver tile lists).
template <int KIND>
struct FusedGeom {
  static constexpr int TX = 64, TZ = 32, NT = 256;
  static constexpr int HV = KIND == VI_MEDIUM_TTI ? 5 : 4;  // halo of the recomputed velocities
  static constexpr int HS = HV + 4;                          // halo of the staged stresses
  static constexpr int SW = TX + 2 * HS, SH = TZ + 2 * HS;
  static constexpr int VW = TX + 2 * HV, VH = TZ + 2 * HV;
  static constexpr int EW = TX + 2, EH = TZ + 2;
  static constexpr int smem_elems =
      3 * SW * SH + 2 * VW * VH + (KIND == VI_MEDIUM_TTI ? 3 * EW * EH : 0);
};

// tile-list entry kinds
// entry kinds of the per-tile lists; a tile's entries are sorted by kind
enum { TL_FORCE_X = 0, TL_FORCE_Z = 1, TL_EXPLOSIVE = 2, TL_RECEIVER = 3 };

template <typename T>
struct FusedExtras {
  int ntx;                 // tiles along x
  int fs;
  int it;
  const int *tile_off;     // ntiles + 1
  const int4 *tile_ent;    // i, j, index, kind
  const T *amp;
  const T *wavelet;
  int wnt;
  T *traces;
  int tnt, nrec;
  int *err;                // device error word (bounded waits that gave up)
  int l2hint;              // split kernels: L2 eviction priorities (see vec.cuh)
};

// Runs nsteps fused steps, ping-ponging between the caller's fields (in
// `a`) and the plan's second state copy; leaves the result in the caller's
// fields.  mode 0: TMA-staged kernel when the grid and every pointer are
// 16-byte aligned, else the non-TMA kernel; 2: non-TMA; 3: TMA (error when
// not eligible).
template <typename T>
int fused_steps(vi_plan *p, StepArgs<T> a, const vi_shot *s, int it0, int nsteps,
                cudaStream_t st, int mode);

// Per-tile CSR list of sources and receivers for a TX x TZ tiling whose
// recomputed-velocity halo is HV cells (0 for the split kernels).
void build_tile_lists(int nx, int nz, int TX, int TZ, int HV, const vi_shot *s,
                      std::vector<int> &off, std::vector<int4> &ent, int &ntx, int &ntz);
// Copies the lists into the plan's device buffer (synchronizes `st`).
int stage_tile_lists(vi_plan *p, const std::vector<int> &off, const std::vector<int4> &ent,
                     cudaStream_t st, int **d_off, int4 **d_ent);

}  // namespace vb
