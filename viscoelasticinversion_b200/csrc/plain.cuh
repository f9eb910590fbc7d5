// plain.cuh — host-side launch interface of the plain multi-kernel step.
#pragma once
#include "common.cuh"

namespace vb {

template <typename T>
struct PlainExtras {
  T *scratch;         // 6 planes of nx*nz
  int fs;
  const int4 *src;    // device: i, j, kind, 0
  const T *amp;       // device
  int nsrc;
  const T *wavelet;   // device, nsrc rows of wnt
  int wnt;
  const int2 *rec;    // device
  int nrec;
  T *traces;          // device, 2*nrec rows of tnt
  int tnt;
};

template <typename T>
void plain_step(const StepArgs<T> &a, const PlainExtras<T> &x, int kind, int it,
                cudaStream_t st);

template <typename T>
void diff_launch(int op, const T *u, T *du, int nx, int nz, double h, cudaStream_t st);

}  // namespace vb
