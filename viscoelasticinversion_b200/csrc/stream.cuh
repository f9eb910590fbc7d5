// stream.cuh — the streaming step kernel (stream.cu): host interface.
#pragma once

#include <cudaTypedefs.h>

#include "common.cuh"

struct vi_plan;

namespace vb {

// Per-launch extras: strips of 120 columns walked in chunks of 4 rows, the
// per-(strip, chunk) source/receiver lists (int4: i, j, index, kind;
// chunk_off has nstrips * (nchunks + 1) + 1 entries), wavelet, traces and
// the plan's device error word.
struct StreamExtras {
  int nstrips, nchunks, fs, it;
  const int *chunk_off;
  const int4 *chunk_ent;
  const float *amp;
  const float *wavelet;
  int wnt;
  float *traces;
  int tnt, nrec;
  int *err;
};

// Tensor maps: 0-2 old sxx, szz, sxz (ring boxes); 3-4 old vx, vz; 5 rho;
// 6 memory variables (3D); 7-10 per-cell stiffness planes (C13, [C11, C33],
// [tau]); 11 C55 (box with the +1 neighbours).
struct StreamMaps {
  CUtensorMap t[12];
};

bool stream_fits(int kind, int nsls);
bool stream_eligible(const vi_plan *p, const StepArgs<float> &a);
int stream_steps(vi_plan *p, StepArgs<float> a, const vi_shot *s, int it0, int nsteps, cudaStream_t st);

}  // namespace vb
