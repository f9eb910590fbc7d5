// plan.cuh — the plan object behind the C ABI (host side).
#pragma once

#include <string>
#include <vector>

#include "common.cuh"

struct vi_plan {
  vi_config cfg;
  int device = 0;
  int nsm = 148;  // streaming multiprocessors of the device
  long long l2_bytes = 126ll << 20;  // L2 cache of the device
  int Lx = 0, Rx = 0, Tz = 0, Bz = 0, wx = 0, hz = 0;
  size_t esize = 4;  // bytes per real
  // device workspace
  void *psix = nullptr, *psiz = nullptr;  // kPsiPlanes planes each
  long long psix_plane = 0, psiz_plane = 0;
  int psi_cur = 0;  // which of the two psi sets holds the current state
  void *errflag = nullptr;     // device error word written by bounded waits
  bool last_used_tma = false;  // the last fused call ran the TMA-staged kernel
  int last_kernel = 0;         // 1 plain, 2 fused, 3 fused TMA-staged
  void *tabx = nullptr, *tabz = nullptr;  // 6*nx and 6*nz reals
  void *scratch = nullptr;                // plain path: 6 planes
  void *alt = nullptr;                    // fused path: second v/sigma copy (5 planes)
  // VI_F32C split step: the stresses' rounding residues (3 bfloat16
  // planes), part of the plan's state like the CPML memory; slo_valid is
  // false after a step that did not carry them (they restart from zero)
  void *slo = nullptr;
  bool slo_valid = false;
  // source / receiver lists (device, grown on demand)
  void *dsrc = nullptr, *damp = nullptr, *drec = nullptr;
  int src_cap = 0, rec_cap = 0;
  // fused path: per-tile source / receiver lists (device, grown on demand)
  void *tile_lists = nullptr;
  size_t tile_lists_bytes = 0;
  // wavefront step: ticket, abort flag and per-band completion counters;
  // sweep depth (steps) and band lag, 0 = the built-in defaults
  void *wave_ctl = nullptr;
  size_t wave_ctl_bytes = 0;
  int wave_k = 0, wave_d = 0;
  // forward_host buffers and the gradient's workspace (device, grown on demand)
  void *fwd = nullptr;
  size_t fwd_bytes = 0;
  // layout of the gradient's kept states whose never-written cells are
  // known zero (0: none)
  unsigned long long grad_zero_key = 0;
  // called by vi_gradient on its own thread after every step it enqueues
  // (units: 1 per forward or recompute step, 2 per adjoint step); a
  // server uses it to run a gradient in slices.  Nonzero: stop.
  int (*yield_fn)(void *ctx, int units) = nullptr;
  void *yield_ctx = nullptr;
  size_t bytes = 0;  // device bytes held
  // host copies of the CPML tables in double precision
  std::vector<double> htx, htz;
};

namespace vb {
int set_error(int code, const std::string &msg);
int cuda_check(cudaError_t e, const char *what);
// Grow-only device buffer.
int ensure_buffer(vi_plan *p, void **buf, size_t *have, size_t need);
// Step arguments of a plan for one medium and one set of fields (input side).
template <typename T>
StepArgs<T> make_args(const vi_plan *p, const vi_medium *m, const vi_fields *f);
int check_medium(const vi_plan *p, const vi_medium *m);
// Whether the split kernels' L2 eviction priorities pay off: the planes
// they keep (the new v and sigma, 5 per shot) fit in half the L2.
inline bool l2_hints_fit(long long kept_bytes, long long l2_bytes) { return 2 * kept_bytes <= l2_bytes; }
int check_fields(const vi_plan *p, const vi_fields *f);
// Sets the non-finite bit of the error word `err` when a stress value of
// the three planes (np cells each) is NaN or infinite (stream-ordered).
template <typename T>
int launch_finite_check(const void *sxx, const void *szz, const void *sxz, long long np, int *err, int nsm,
                        cudaStream_t st);
// Copies a shot's source / receiver lists to the plan's device buffers.
template <typename T>
int stage_shot(vi_plan *p, const vi_shot *s, cudaStream_t st);
}  // namespace vb
