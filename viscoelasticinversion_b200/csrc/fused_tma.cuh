// fused_tma.cuh — shared-memory layout and host interface of the TMA-staged
// fused step.
#pragma once

#include <cuda.h>

#include "common.cuh"
#include "fused.cuh"

namespace vb {

constexpr int kSmemLimit = 227 * 1024;  // per-CTA dynamic shared memory on sm_100

template <typename T>
constexpr int r128(int n) {  // round an element count up to 128 bytes
  return (int)((((long long)n * (long long)sizeof(T) + 127) / 128) * 128 / (long long)sizeof(T));
}

// Every operand of one TX x TZ tile, staged by TMA boxes (x extent padded to
// 4 elements so each box starts on a 16-byte boundary), in STAGES buffers.
// With two stages the kernel is persistent (one CTA per SM) and loads the
// next tile while computing the current one.
template <typename T, int KIND, int NSLS, int TZ_, int STAGES_>
struct TmaLayout {
  static constexpr int TX = 64, TZ = TZ_, STAGES = STAGES_;
  static constexpr int NT = STAGES == 2 ? 512 : 256;
  // cells per thread group in the stress stage: the persistent form has
  // twice the threads, so it splits the tile into 2-wide groups
  static constexpr int SWID = STAGES == 2 ? 2 : 4;
  static constexpr bool TTI = KIND == VI_MEDIUM_TTI;
  static constexpr int HV = TTI ? 5 : 4;        // halo of recomputed velocities
  static constexpr int HS = HV + 4;              // halo of staged stresses
  static constexpr int HVP = (HV + 3) / 4 * 4;   // x padding to 16-byte boxes
  static constexpr int HSP = (HS + 3) / 4 * 4;
  static constexpr int NM = 3 * NSLS;
  static constexpr int NC = KIND == VI_MEDIUM_ISO ? 2 : (KIND == VI_MEDIUM_VTI ? 4 : 6);
  // boxes (x extent, z extent)
  static constexpr int SWp = TX + 2 * HSP, SH = TZ + 2 * HS;        // sigma
  static constexpr int VWp = TX + 2 * HVP, VH = TZ + 2 * HV;        // velocity
  static constexpr int VW = TX + 2 * HV;                            // computed velocity width
  static constexpr int RWp = TX + 2 * HVP + 4, RH = TZ + 2 * HV + 1;  // rho
  static constexpr int MX0 = TTI ? -4 : 0, MZ0 = TTI ? -1 : 0;      // M / tau box origin
  static constexpr int MW = TTI ? TX + 8 : TX, MH = TTI ? TZ + 2 : TZ;
  static constexpr int CW = TX + 4, CH = TZ + 1;                    // coefficients (+1 ring)
  static constexpr int EW = TX + 8, EH = TZ + 2;  // TTI effective rates, origin (x0-4, z0-1)
  // plane sizes (elements, 128-byte aligned)
  static constexpr int PS = r128<T>(SWp * SH), PV = r128<T>(VWp * VH), PR = r128<T>(RWp * RH);
  static constexpr int PM = r128<T>(MW * MH * (NM > 0 ? NM : 1));
  static constexpr int PC = r128<T>(CW * CH);
  static constexpr int PT = TTI ? r128<T>(MW * MH) : PC;
  static constexpr int PE = r128<T>(EW * EH);
  // offsets inside one stage
  static constexpr int S_SXX = 0, S_SZZ = PS, S_SXZ = 2 * PS;
  static constexpr int S_VX = 3 * PS, S_VZ = S_VX + PV, S_RHO = S_VZ + PV;
  static constexpr int S_M = S_RHO + PR;
  static constexpr int S_C = S_M + (NSLS > 0 ? PM : 0);
  static constexpr int S_TAU = S_C + NC * PC;
  static constexpr int STAGE = S_TAU + (NSLS > 0 ? PT : 0);
  // whole buffer: 128-byte barrier slot, the stages, the TTI rate planes
  static constexpr int O_STAGE = 128 / (int)sizeof(T);
  static constexpr int O_E = O_STAGE + STAGES * STAGE;
  static constexpr int ELEMS = O_E + (TTI ? 3 * PE : 0);
  static constexpr int BYTES = ELEMS * (int)sizeof(T);
  // transaction bytes of all boxes of one tile
  static constexpr int TX_BYTES =
      (int)sizeof(T) * (3 * SWp * SH + 2 * VWp * VH + RWp * RH + (NSLS > 0 ? MW * MH * NM : 0) +
                        NC * CW * CH + (NSLS > 0 ? (TTI ? MW * MH : CW * CH) : 0));
  static constexpr bool FITS = BYTES <= kSmemLimit;
};

// Layout choice: (PERSIST) two stages of 16-row tiles, else two stages of
// 8-row tiles; else one stage of 16 or 8 rows (one tile per CTA).
template <typename T, int KIND, int NSLS, bool PERSIST = true>
struct TmaPick {
  static constexpr bool F16x2 = PERSIST && TmaLayout<T, KIND, NSLS, 16, 2>::FITS;
  static constexpr bool F8x2 = PERSIST && TmaLayout<T, KIND, NSLS, 8, 2>::FITS;
  static constexpr bool F16x1 = TmaLayout<T, KIND, NSLS, 16, 1>::FITS;
  static constexpr int TZ = F16x2 ? 16 : (F8x2 ? 8 : (F16x1 ? 16 : 8));
  static constexpr int STAGES = (F16x2 || F8x2) ? 2 : 1;
  using Lay = TmaLayout<T, KIND, NSLS, TZ, STAGES>;
  static constexpr bool OK = Lay::FITS;
};

// Tensor maps of one ping-pong parity.  Coefficient slot order per kind:
// ISO (c13, c55), VTI (c11, c13, c33, c55), TTI (c11, c13, c15, c33, c35, c55).
struct TmaMaps {
  CUtensorMap sxx, szz, sxz, vx, vz, rho, m, tau;
  CUtensorMap c[6];
};

// Tile and box geometry the host needs (tile lists, grid size, tensor-map
// boxes) for a medium kind, mechanism count and element size.
struct TmaBoxes {
  int TX, TZ, HV, HS, HVP, HSP, STAGES, NT;
  int SWp, SH, VWp, VH, RWp, RH, MX0, MZ0, MW, MH, NM, CW, CH, NC;
  bool ok;
};
TmaBoxes tma_boxes(int kind, int nsls, int esize, bool persist);

template <typename T>
int launch_fused_tma(int kind, const StepArgs<T> &a, const FusedExtras<T> &x,
                     const TmaMaps &maps, int ntiles, int nsm, bool persist, cudaStream_t st);

struct SplitMaps;

// Per-shot data of a batch in device memory (see k_fused_tma_batch and the
// batched split kernels).
template <typename T>
struct BatchDev {
  const StepArgs<T> *args;    // [2 * nshots]: index 2*s + parity of the step
  const FusedExtras<T> *ext;  // [nshots] (it is set per launch)
  const TmaMaps *maps;        // [2 * nshots] (fused kernel forms)
  const SplitMaps *smaps;     // [nshots] (split kernel form)
  const int *prefix;          // [nshots + 1] tile offsets in processing order
  const int *order;           // [nshots] shot at each processing position
  const int2 *items;          // [prefix[nshots]] (shot, tile) of every item
  int nshots;
  int *err;
};

#ifdef __CUDACC__
// The shot and tile of batch item `item` (items are the tiles of the shots
// in processing order): from the item table, else by binary search for the
// largest position p with prefix[p] <= item.
template <typename T>
__device__ __forceinline__ void batch_locate(const BatchDev<T> &b, int item, int &shot, int &tile) {
  if (b.items) {  // one load instead of a chain of dependent ones
    const int2 v = b.items[item];
    shot = v.x;
    tile = v.y;
    return;
  }
  int lo = 0, hi = b.nshots - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (b.prefix[mid] <= item)
      lo = mid;
    else
      hi = mid - 1;
  }
  shot = b.order[lo];
  tile = item - b.prefix[lo];
}
#endif

template <typename T>
int launch_fused_tma_batch(int kind, int nsls, const BatchDev<T> &b, int it, int nitems, int nsm,
                           bool persist, cudaStream_t st);

// Tensor maps of one ping-pong parity: the input state (in[0..4] = vx, vz,
// sxx, szz, sxz; M with its plane stride) and the medium of `a`.
template <typename T>
int encode_parity(TmaMaps &m, const TmaBoxes &b, const vi_config &c, T *const in[5], const T *min,
                  long long mstride, const StepArgs<T> &a);

// Encodes a 2D (depth = 1) or 3D tensor map over an x-fastest array.
int encode_map(CUtensorMap *map, const void *base, int esize, int nx, int nz, long long depth,
               long long plane_stride_elems, int box_x, int box_z, int box_d);

}  // namespace vb
