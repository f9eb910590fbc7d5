// capi.cu — C ABI (include/visco_b200.h): plan, time stepping, forward solve.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "fused.cuh"
#include "nvtx.cuh"
#include "plain.cuh"
#include "plan.cuh"
#include "split.cuh"
#include "stream.cuh"

namespace vb {

static thread_local std::string g_err;

int set_error(int code, const std::string &msg) {
  g_err = msg;
  return code;
}

int cuda_check(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return VI_OK;
  cudaGetLastError();  // clear the sticky-free error state
  return set_error(VI_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

int ensure_buffer(vi_plan *p, void **buf, size_t *have, size_t need) {
  if (*have >= need && *buf) return VI_OK;
  if (*buf) {
    cudaFree(*buf);
    p->bytes -= *have;
    *buf = nullptr;
    *have = 0;
  }
  if (need == 0) return VI_OK;
  cudaError_t e = cudaMalloc(buf, need);
  if (e != cudaSuccess) {
    *buf = nullptr;
    cudaGetLastError();
    return set_error(VI_ERR_BUDGET, std::string("cudaMalloc of ") + std::to_string(need) +
                                        " bytes failed: " + cudaGetErrorString(e));
  }
  *have = need;
  p->bytes += need;
  return VI_OK;
}

// CPML profile of CPML.jl:91-189 evaluated at integer (half=0) or half
// (half=1) nodes of one axis; writes [1/kappa, a, b] tables of n values.
static void cpml_tables(const vi_config &c, int axis, int half, double *ik, double *a,
                        double *b) {
  const int n = axis == 0 ? c.nx : c.nz;
  const double h = axis == 0 ? c.dx : c.dz;
  const int lo = axis == 0 ? c.pml_left : c.pml_top;
  const int hi = axis == 0 ? c.pml_right : c.pml_bottom;
  const double Lp = c.pml_thickness;
  double d0 = c.pml_d0;
  if (d0 <= 0.0 && Lp > 0)
    d0 = -(c.pml_power + 1.0) * c.pml_vmax * std::log(c.pml_reflection) / (2.0 * Lp * h);
  for (int k = 0; k < n; ++k) {
    const double x = k + (half ? 0.5 : 0.0);
    double p = 0.0;
    if (Lp > 0) {
      if (lo) p = std::fmax(p, (Lp - 0.5 - x) / Lp);
      if (hi) p = std::fmax(p, (x - (n - Lp - 0.5)) / Lp);
    }
    double d = 0, al = 0, ka = 1;
    if (p > 0) {
      d = d0 * std::pow(p, c.pml_power);
      al = c.pml_alpha_max * (1.0 - p);
      ka = 1.0 + (c.pml_kappa_max - 1.0) * p;
    }
    double bb = 0, aa = 0;
    if (d > 0 || al > 0) {
      bb = std::exp(-(d / ka + al) * c.dt);
      if (std::fabs(d) > 2.220446049250313e-16) aa = d / (ka * (d + ka * al)) * (bb - 1.0);
    }
    ik[k] = 1.0 / ka;
    a[k] = aa;
    b[k] = bb;
  }
}

// Weights of the first derivative at x0 from the samples at x[0..n-1]
// (n <= 8): sum_k w_k (x_k - x0)^l / l! = [l == 1] for l < n — the
// Vandermonde system of Stencil.jl:_stencil (lines 9-14), solved by
// Gaussian elimination with partial pivoting.
static void fd_weights(const double *x, int n, double x0, double *w) {
  double A[8][9];
  for (int l = 0; l < n; ++l) {
    double fact = 1;
    for (int q = 2; q <= l; ++q) fact *= q;
    for (int k = 0; k < n; ++k) A[l][k] = std::pow(x[k] - x0, l) / fact;
    A[l][n] = l == 1 ? 1.0 : 0.0;
  }
  for (int c = 0; c < n; ++c) {
    int p = c;
    for (int r = c + 1; r < n; ++r)
      if (std::fabs(A[r][c]) > std::fabs(A[p][c])) p = r;
    for (int k = 0; k <= n; ++k) std::swap(A[c][k], A[p][k]);
    for (int r = 0; r < n; ++r)
      if (r != c && A[r][c] != 0) {
        const double f = A[r][c] / A[c][c];
        for (int k = c; k <= n; ++k) A[r][k] -= f * A[c][k];
      }
  }
  for (int k = 0; k < n; ++k) w[k] = A[k][n] / A[k][k];
}

// H-AFDA free surface (Kristek, Moczo & Archuleta 2002, the reference's
// FreeSurfaceStencil, Stencil.jl:52-105, and kernels,
// free-surface-kernels.jl:16-213): the surface z = 0 is the row of sxx,
// szz and vx; szz(0) = sxz(0) = 0 there and nothing lives above it.  A z
// derivative whose 8th-order staggered stencil would reach above the
// surface takes a one-sided approximation from kAfdaN samples at or below
// it (plus the zero boundary value of sxz or szz at z = 0) — unit-spacing
// weights w[op][q][m] in the layout of StepArgs::af.  The reference sizes
// these approximations like the interior stencil (8 samples); with 8 the
// semi-discrete operator has growing modes, with 5 it has none.
static void afda_unit_weights(double w[4][4][kAfdaN]) {
  double x[kAfdaN + 1], t[kAfdaN + 1];
  std::memset(w, 0, sizeof(double) * 4 * 4 * kAfdaN);
  for (int q = 0; q < 4; ++q) {  // d(sxz)/dz at z = q from sxz(0) = 0 and sxz at m + 1/2
    x[0] = 0;
    for (int m = 0; m < kAfdaN; ++m) x[m + 1] = m + 0.5;
    fd_weights(x, kAfdaN + 1, q, t);
    for (int m = 0; m < kAfdaN; ++m) w[0][q][m] = t[m + 1];
  }
  for (int q = 0; q < 3; ++q) {  // d(szz)/dz at z = q + 1/2 from szz(0) = 0 and szz at 1 + m
    for (int m = 0; m <= kAfdaN; ++m) x[m] = m;
    fd_weights(x, kAfdaN + 1, q + 0.5, t);
    for (int m = 0; m < kAfdaN; ++m) w[1][q][m] = t[m + 1];
  }
  for (int q = 1; q < 4; ++q) {  // d(vz)/dz at z = q from vz at m + 1/2
    for (int m = 0; m < kAfdaN; ++m) x[m] = m + 0.5;
    fd_weights(x, kAfdaN, q, t);
    for (int m = 0; m < kAfdaN; ++m) w[2][q][m] = t[m];
  }
  for (int q = 0; q < 3; ++q) {  // d(vx)/dz at z = q + 1/2 from vx at m
    for (int m = 0; m < kAfdaN; ++m) x[m] = m;
    fd_weights(x, kAfdaN, q + 0.5, t);
    for (int m = 0; m < kAfdaN; ++m) w[3][q][m] = t[m];
  }
}

static int validate(const vi_config *c) {
  if (!c) return set_error(VI_ERR_ARG, "config is NULL");
  if (c->nx < 2 * L + 2 || c->nz < 2 * L + 2)
    return set_error(VI_ERR_ARG, "grid must be at least 10 x 10 cells (8th-order stencil)");
  if ((long long)c->nx * c->nz > (1LL << 31))
    return set_error(VI_ERR_ARG, "grid larger than 2^31 cells");
  if (!(c->dx > 0 && c->dz > 0 && c->dt > 0))
    return set_error(VI_ERR_ARG, "dx, dz and dt must be positive");
  if (c->medium < VI_MEDIUM_ISO || c->medium > VI_MEDIUM_TTI)
    return set_error(VI_ERR_ARG, "unknown medium kind");
  if (c->precision != VI_F32 && c->precision != VI_F64 && c->precision != VI_F32C)
    return set_error(VI_ERR_ARG, "unknown precision");
  if (c->nsls < 0 || c->nsls > VI_MAX_SLS)
    return set_error(VI_ERR_ARG, "nsls must be in 0..5");
  for (int n = 0; n < c->nsls; ++n)
    if (!(c->tau_sls[n] > 0)) return set_error(VI_ERR_ARG, "tau_sls must be positive");
  if (c->pml_thickness < 0) return set_error(VI_ERR_ARG, "negative CPML thickness");
  if (c->pml_thickness > 0) {
    const int wx = (c->pml_left ? 1 : 0) + (c->pml_right ? 1 : 0);
    const int hz = (c->pml_top ? 1 : 0) + (c->pml_bottom ? 1 : 0);
    if (wx * c->pml_thickness > c->nx || hz * c->pml_thickness > c->nz)
      return set_error(VI_ERR_ARG, "CPML strips overlap");
    if (c->pml_d0 <= 0 && !(c->pml_vmax > 0 && c->pml_reflection > 0 && c->pml_reflection < 1))
      return set_error(VI_ERR_ARG, "CPML d0 needs vmax > 0 and 0 < R < 1");
    if (c->pml_kappa_max < 1) return set_error(VI_ERR_ARG, "CPML kappa_max must be >= 1");
  }
  if (c->free_surface < 0 || c->free_surface > kFsAfda)
    return set_error(VI_ERR_ARG, "free_surface must be 0 (none), 1 (stress imaging) or 2 (H-AFDA)");
  if (c->free_surface && c->pml_top && c->pml_thickness > 0)
    return set_error(VI_ERR_ARG, "free surface and a top CPML are exclusive");
  if (c->pml_vmax > 0) {
    double sum = 0;
    for (double d : kD8) sum += std::fabs(d);
    const double cfl = c->pml_vmax * c->dt * std::sqrt(1 / (c->dx * c->dx) + 1 / (c->dz * c->dz)) * sum;
    if (cfl > 1.0)
      return set_error(VI_ERR_CFL, "CFL violated: vmax*dt*sqrt(1/dx^2+1/dz^2)*sum|D| = " +
                                       std::to_string(cfl) + " > 1");
  }
  return VI_OK;
}

template <typename T>
static int upload_tables(vi_plan *p) {
  const int nx = p->cfg.nx, nz = p->cfg.nz;
  std::vector<T> tx(6 * (size_t)nx), tz(6 * (size_t)nz);
  for (size_t k = 0; k < tx.size(); ++k) tx[k] = (T)p->htx[k];
  for (size_t k = 0; k < tz.size(); ++k) tz[k] = (T)p->htz[k];
  int rc = cuda_check(cudaMemcpy(p->tabx, tx.data(), tx.size() * sizeof(T), cudaMemcpyHostToDevice),
                      "upload CPML x tables");
  if (rc) return rc;
  return cuda_check(cudaMemcpy(p->tabz, tz.data(), tz.size() * sizeof(T), cudaMemcpyHostToDevice),
                    "upload CPML z tables");
}

template <typename T>
StepArgs<T> make_args(const vi_plan *p, const vi_medium *m, const vi_fields *f) {
  const vi_config &c = p->cfg;
  StepArgs<T> a;
  std::memset(&a, 0, sizeof(a));
  a.nx = c.nx;
  a.nz = c.nz;
  a.nsls = c.nsls;
  a.Lx = p->Lx;
  a.Rx = p->Rx;
  a.Tz = p->Tz;
  a.Bz = p->Bz;
  a.wx = p->wx;
  a.hz = p->hz;
  a.dt = (T)c.dt;
  for (int k = 0; k < 4; ++k) {
    a.Dx[k] = (T)(kD8[k] / c.dx);
    a.Dz[k] = (T)(kD8[k] / c.dz);
  }
  for (int n = 0; n < c.nsls; ++n) {
    a.a1[n] = (T)(-1.0 / (c.nsls * c.tau_sls[n]));
    a.a2[n] = (T)(-1.0 / c.tau_sls[n]);
  }
  if (c.free_surface == kFsAfda) {
    double w[4][4][kAfdaN];
    afda_unit_weights(w);
    for (int op = 0; op < 4; ++op)
      for (int q = 0; q < 4; ++q)
        for (int k = 0; k < kAfdaN; ++k) a.af[op][q][k] = (T)(w[op][q][k] / c.dz);
  }
  a.rho = (const T *)m->rho;
  a.c11 = (const T *)m->c11;
  a.c13 = (const T *)m->c13;
  a.c15 = (const T *)m->c15;
  a.c33 = (const T *)m->c33;
  a.c35 = (const T *)m->c35;
  a.c55 = (const T *)m->c55;
  a.tau = (const T *)m->tau;
  a.vx = (T *)f->vx;
  a.vz = (T *)f->vz;
  a.sxx = (T *)f->sxx;
  a.szz = (T *)f->szz;
  a.sxz = (T *)f->sxz;
  a.m = (T *)f->m;
  a.mstride = f->m_plane_stride;
  a.psix = a.psix_o = (T *)p->psix;
  a.psiz = a.psiz_o = (T *)p->psiz;
  a.psix_plane = p->psix_plane;
  a.psiz_plane = p->psiz_plane;
  a.tx = (const T *)p->tabx;
  a.tz = (const T *)p->tabz;
  return a;
}

int check_medium(const vi_plan *p, const vi_medium *m) {
  if (!m) return set_error(VI_ERR_ARG, "medium is NULL");
  const int k = p->cfg.medium;
  if (!m->rho || !m->c13 || !m->c55) return set_error(VI_ERR_ARG, "medium: rho, c13, c55 required");
  if (k != VI_MEDIUM_ISO && (!m->c11 || !m->c33))
    return set_error(VI_ERR_ARG, "medium: c11, c33 required for VTI/TTI");
  if (k == VI_MEDIUM_TTI && (!m->c15 || !m->c35))
    return set_error(VI_ERR_ARG, "medium: c15, c35 required for TTI");
  if (p->cfg.nsls > 0 && !m->tau) return set_error(VI_ERR_ARG, "medium: tau required when nsls > 0");
  return VI_OK;
}

int check_fields(const vi_plan *p, const vi_fields *f) {
  if (!f) return set_error(VI_ERR_ARG, "fields is NULL");
  if (!f->vx || !f->vz || !f->sxx || !f->szz || !f->sxz)
    return set_error(VI_ERR_ARG, "fields: vx, vz, sxx, szz, sxz required");
  if (p->cfg.nsls > 0) {
    if (!f->m) return set_error(VI_ERR_ARG, "fields: m required when nsls > 0");
    if (f->m_plane_stride < (long long)p->cfg.nx * p->cfg.nz)
      return set_error(VI_ERR_ARG, "fields: m_plane_stride smaller than nx*nz");
  }
  return VI_OK;
}

static bool in_update_region(const vi_config &c, int i, int j) {
  return i >= L && i < c.nx - L && j >= L && j < c.nz - L;
}

// Copies the shot's source / receiver lists to the plan's device buffers.
template <typename T>
int stage_shot(vi_plan *p, const vi_shot *s, cudaStream_t st) {
  if (!s) return VI_OK;
  if (s->nsrc < 0 || s->nrec < 0) return set_error(VI_ERR_ARG, "negative source/receiver count");
  if (s->nsrc > 0) {
    if (!s->src_host || !s->wavelet_dev || s->wavelet_nt < 0)
      return set_error(VI_ERR_ARG, "sources need src_host and wavelet_dev");
    std::vector<int4> hs(s->nsrc);
    std::vector<T> ha(s->nsrc);
    for (int q = 0; q < s->nsrc; ++q) {
      const vi_source &v = s->src_host[q];
      if (!in_update_region(p->cfg, v.i, v.j))
        return set_error(VI_ERR_ARG, "source " + std::to_string(q) + " outside the update region");
      if (v.kind < VI_SRC_EXPLOSIVE || v.kind > VI_SRC_FORCE_Z)
        return set_error(VI_ERR_ARG, "unknown source kind");
      hs[q] = make_int4(v.i, v.j, v.kind, 0);
      ha[q] = (T)v.amp;
    }
    if (s->nsrc > p->src_cap) {
      size_t h1 = 0, h2 = 0;
      if (p->dsrc) { cudaFree(p->dsrc); p->bytes -= (size_t)p->src_cap * sizeof(int4); p->dsrc = nullptr; }
      if (p->damp) { cudaFree(p->damp); p->bytes -= (size_t)p->src_cap * sizeof(double); p->damp = nullptr; }
      int rc = ensure_buffer(p, &p->dsrc, &h1, (size_t)s->nsrc * sizeof(int4));
      if (rc) return rc;
      rc = ensure_buffer(p, &p->damp, &h2, (size_t)s->nsrc * sizeof(double));
      if (rc) return rc;
      p->src_cap = s->nsrc;
    }
    int rc = cuda_check(cudaMemcpyAsync(p->dsrc, hs.data(), hs.size() * sizeof(int4),
                                        cudaMemcpyHostToDevice, st), "copy sources");
    if (rc) return rc;
    rc = cuda_check(cudaMemcpyAsync(p->damp, ha.data(), ha.size() * sizeof(T),
                                    cudaMemcpyHostToDevice, st), "copy amplitudes");
    if (rc) return rc;
    // the staging vectors die at return: wait for the pageable copies
    rc = cuda_check(cudaStreamSynchronize(st), "stage sources");
    if (rc) return rc;
  }
  if (s->nrec > 0) {
    if (!s->rec_host) return set_error(VI_ERR_ARG, "receivers need rec_host");
    std::vector<int2> hr(s->nrec);
    for (int r = 0; r < s->nrec; ++r) {
      const vi_receiver &v = s->rec_host[r];
      if (!in_update_region(p->cfg, v.i, v.j))
        return set_error(VI_ERR_ARG, "receiver " + std::to_string(r) + " outside the update region");
      hr[r] = make_int2(v.i, v.j);
    }
    if (s->nrec > p->rec_cap) {
      size_t h1 = 0;
      if (p->drec) { cudaFree(p->drec); p->bytes -= (size_t)p->rec_cap * sizeof(int2); p->drec = nullptr; }
      int rc = ensure_buffer(p, &p->drec, &h1, (size_t)s->nrec * sizeof(int2));
      if (rc) return rc;
      p->rec_cap = s->nrec;
    }
    int rc = cuda_check(cudaMemcpyAsync(p->drec, hr.data(), hr.size() * sizeof(int2),
                                        cudaMemcpyHostToDevice, st), "copy receivers");
    if (rc) return rc;
    rc = cuda_check(cudaStreamSynchronize(st), "stage receivers");
    if (rc) return rc;
  }
  return VI_OK;
}

// Finite check of the stresses after a call of the step paths that do not
// fold it into their stress pass (the split pair does): one warp vote per
// 32 cells, the error word's non-finite bit on any NaN or infinity.
template <typename T>
__global__ void k_finite(const T *sxx, const T *szz, const T *sxz, long long np, int *err) {
  bool bad = false;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < np; c += (long long)gridDim.x * blockDim.x)
    bad |= !isfinite(sxx[c] + szz[c] + sxz[c]);
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(err, kErrNonFinite);
}

template <typename T>
int launch_finite_check(const void *sxx, const void *szz, const void *sxz, long long np, int *err, int nsm,
                        cudaStream_t st) {
  if (np <= 0) return VI_OK;
  k_finite<T><<<(unsigned)std::min<long long>(4LL * nsm, (np + 255) / 256), 256, 0, st>>>(
      (const T *)sxx, (const T *)szz, (const T *)sxz, np, err);
  return cuda_check(cudaGetLastError(), "finite check launch");
}
template int launch_finite_check<float>(const void *, const void *, const void *, long long, int *, int,
                                        cudaStream_t);
template int launch_finite_check<double>(const void *, const void *, const void *, long long, int *, int,
                                         cudaStream_t);

template <typename T>
static int step_impl(vi_plan *p, const vi_medium *m, vi_fields *f, const vi_shot *s, int it0,
                     int nsteps, int variant, cudaStream_t st) {
  int rc = check_medium(p, m);
  if (rc) return rc;
  rc = check_fields(p, f);
  if (rc) return rc;
  if (nsteps < 0) return set_error(VI_ERR_ARG, "nsteps must be >= 0");
  if (variant < 0 || variant > 9) return set_error(VI_ERR_ARG, "unknown kernel variant");
  if (s && s->nrec > 0 && s->traces_nt > 0 && !s->traces_dev)
    return set_error(VI_ERR_ARG, "receivers need traces_dev");
  rc = cuda_check(cudaSetDevice(p->device), "cudaSetDevice");
  if (rc) return rc;
  rc = stage_shot<T>(p, s, st);
  if (rc) return rc;
  StepArgs<T> a = make_args<T>(p, m, f);
  const int nsrc = s ? s->nsrc : 0;
  const int nrec = s ? s->nrec : 0;
  if (p->cfg.precision == VI_F32C && (variant == 1 || variant == 7))
    return set_error(VI_ERR_ARG, "compensated FP32 (VI_F32C) runs on the split pair only (kernel variant 0, 5 or 8)");
  if (p->cfg.free_surface == kFsAfda) {
    if (variant == 2 || variant == 3 || variant == 4 || variant == 6 || variant == 7)
      return set_error(VI_ERR_ARG, "the H-AFDA free surface runs on the split pair and the plain path "
                                   "(kernel variant 0, 1, 5 or 8)");
    if (variant == 0 && !split_eligible<T>(p, a) && p->cfg.precision != VI_F32C) variant = 1;
  }
  if (variant == 1) {
    if (!p->scratch) {
      // cells outside the update region are read by the neighbour averages
      // and never written: zero the planes once
      const size_t sb = 6 * (size_t)p->cfg.nx * p->cfg.nz * sizeof(T);
      size_t have = 0;
      rc = ensure_buffer(p, &p->scratch, &have, sb);
      if (rc) return rc;
      rc = cuda_check(cudaMemsetAsync(p->scratch, 0, sb, st), "zero scratch");
      if (rc) return rc;
    }
    PlainExtras<T> x;
    x.scratch = (T *)p->scratch;
    x.fs = p->cfg.free_surface;
    x.src = (const int4 *)p->dsrc;
    x.amp = (const T *)p->damp;
    x.nsrc = nsrc;
    x.wavelet = nsrc ? (const T *)s->wavelet_dev : nullptr;
    x.wnt = nsrc ? s->wavelet_nt : 0;
    x.rec = (const int2 *)p->drec;
    x.nrec = nrec;
    x.traces = nrec ? (T *)s->traces_dev : nullptr;
    x.tnt = nrec ? s->traces_nt : 0;
    // in place on the current psi set
    const int cur = p->psi_cur;
    if (a.psix) a.psix = a.psix_o = (T *)p->psix + cur * kPsiPerSet * p->psix_plane;
    if (a.psiz) a.psiz = a.psiz_o = (T *)p->psiz + cur * kPsiPerSet * p->psiz_plane;
    for (int k = 0; k < nsteps; ++k) plain_step<T>(a, x, p->cfg.medium, it0 + k, st);
  } else if (variant == 7) {
    if constexpr (sizeof(T) == 4) {
      rc = stream_steps(p, a, s, it0, nsteps, st);
      if (rc) return rc;
      p->last_kernel = 7;
    } else {
      return set_error(VI_ERR_ARG, "the streaming step is FP32 only");
    }
  } else if (variant == 9) {
    rc = wave_steps<T>(p, a, s, it0, nsteps, st);
    if (rc) return rc;
    p->last_kernel = 9;
  } else if (p->cfg.precision == VI_F32C &&
             !(variant == 5 || variant == 8 || (variant == 0 && split_eligible<T>(p, a)))) {
    return set_error(VI_ERR_ARG, "compensated FP32 (VI_F32C) runs on the split pair only (kernel variant 0, 5 or 8 "
                                 "with nx % 4 == 0 and 16-byte aligned planes)");
  } else if (variant == 5 || variant == 6 || variant == 8 || (variant == 0 && split_eligible<T>(p, a))) {
    // the one-tile-per-CTA pair measures faster than the pipelined pair on
    // B200 (2048 x 1024 VTI: 27.6 vs 24.4 Gpt/s), so it is the default
    const int mode = variant == 6 ? kSplitPipelined : variant == 8 ? kSplitLdg : kSplitVelTma;
    rc = split_steps<T>(p, a, s, it0, nsteps, st, mode);
    if (rc) return rc;
    p->last_kernel = variant == 0 ? 5 : variant;
  } else {
    rc = fused_steps<T>(p, a, s, it0, nsteps, st, variant);
    if (rc) return rc;
    p->last_kernel = p->last_used_tma ? (variant == 4 ? 4 : 3) : 2;
  }
  if (variant == 1) p->last_kernel = 1;
  // paths without the folded finite check get it once at the end of the call
  if (variant == 1 || variant == 7 || p->last_kernel == 2 || p->last_kernel == 3 || p->last_kernel == 4 ||
      p->last_kernel == 6) {
    if (nsteps > 0 &&
        (rc = launch_finite_check<T>(a.sxx, a.szz, a.sxz, (long long)p->cfg.nx * p->cfg.nz, (int *)p->errflag,
                                     p->nsm, st)))
      return rc;
  }
  return cuda_check(cudaGetLastError(), "step launch");
}

template StepArgs<float> make_args<float>(const vi_plan *, const vi_medium *, const vi_fields *);
template StepArgs<double> make_args<double>(const vi_plan *, const vi_medium *, const vi_fields *);
template int stage_shot<float>(vi_plan *, const vi_shot *, cudaStream_t);
template int stage_shot<double>(vi_plan *, const vi_shot *, cudaStream_t);

}  // namespace vb

using namespace vb;

extern "C" int vi_version(void) { return VI_ABI_VERSION; }

extern "C" const char *vi_last_error(void) { return g_err.c_str(); }

extern "C" int vi_plan_create(const vi_config *cfg, vi_plan **out) {
  if (!out) return set_error(VI_ERR_ARG, "out is NULL");
  *out = nullptr;
  int rc = validate(cfg);
  if (rc) return rc;
  vi_plan *p = new vi_plan();
  p->cfg = *cfg;
  cudaGetDevice(&p->device);
  int l2 = 0;
  if (cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, p->device) == cudaSuccess && l2 > 0)
    p->l2_bytes = l2;
  else
    cudaGetLastError();
  if (cudaDeviceGetAttribute(&p->nsm, cudaDevAttrMultiProcessorCount, p->device) != cudaSuccess ||
      p->nsm <= 0) {
    cudaGetLastError();
    p->nsm = 148;
  }
  p->esize = cfg->precision == VI_F64 ? 8 : 4;
  const int Lp = cfg->pml_thickness;
  p->Lx = (Lp > 0 && cfg->pml_left) ? Lp : 0;
  p->Rx = (Lp > 0 && cfg->pml_right) ? Lp : 0;
  p->Tz = (Lp > 0 && cfg->pml_top) ? Lp : 0;
  p->Bz = (Lp > 0 && cfg->pml_bottom) ? Lp : 0;
  p->wx = p->Lx + p->Rx;
  p->hz = p->Tz + p->Bz;
  const int nx = cfg->nx, nz = cfg->nz;
  p->htx.assign(6 * (size_t)nx, 0.0);
  p->htz.assign(6 * (size_t)nz, 0.0);
  for (int half = 0; half < 2; ++half) {
    double *tx = p->htx.data() + (half ? 3 : 0) * (size_t)nx;
    cpml_tables(*cfg, 0, half, tx, tx + nx, tx + 2 * (size_t)nx);
    double *tz = p->htz.data() + (half ? 3 : 0) * (size_t)nz;
    cpml_tables(*cfg, 1, half, tz, tz + nz, tz + 2 * (size_t)nz);
  }
  p->psix_plane = (long long)p->wx * nz;
  p->psiz_plane = (long long)nx * p->hz;
  size_t h = 0;
  if ((rc = ensure_buffer(p, &p->tabx, &h, 6 * (size_t)nx * p->esize))) goto fail;
  h = 0;
  if ((rc = ensure_buffer(p, &p->tabz, &h, 6 * (size_t)nz * p->esize))) goto fail;
  if (p->psix_plane > 0) {
    h = 0;
    if ((rc = ensure_buffer(p, &p->psix, &h, kPsiPlanes * (size_t)p->psix_plane * p->esize))) goto fail;
  }
  if (p->psiz_plane > 0) {
    h = 0;
    if ((rc = ensure_buffer(p, &p->psiz, &h, kPsiPlanes * (size_t)p->psiz_plane * p->esize))) goto fail;
  }
  h = 0;
  if ((rc = ensure_buffer(p, &p->errflag, &h, 16))) goto fail;
  if ((rc = cuda_check(cudaMemset(p->errflag, 0, 16), "zero error word"))) goto fail;
  rc = cfg->precision == VI_F64 ? upload_tables<double>(p) : upload_tables<float>(p);
  if (rc) goto fail;
  rc = vi_plan_reset(p, nullptr);
  if (rc) goto fail;
  rc = cuda_check(cudaDeviceSynchronize(), "plan create");
  if (rc) goto fail;
  *out = p;
  return VI_OK;
fail:
  vi_plan_destroy(p);
  return rc;
}

extern "C" int vi_plan_set_wave(vi_plan *p, int32_t depth, int32_t lag) {
  if (!p) return set_error(VI_ERR_ARG, "null plan");
  if (depth < 0 || depth > 64) return set_error(VI_ERR_ARG, "wavefront depth must be 0 (default) .. 64 steps");
  if (lag != 0 && (lag < 2 || lag > 64)) return set_error(VI_ERR_ARG, "wavefront band lag must be 0 (default) or 2 .. 64");
  p->wave_k = depth;
  p->wave_d = lag;
  return VI_OK;
}

extern "C" int vi_plan_destroy(vi_plan *p) {
  if (!p) return VI_OK;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(p->device);
  void *bufs[] = {p->psix, p->psiz, p->tabx, p->tabz, p->scratch, p->alt, p->slo,
                  p->dsrc, p->damp, p->drec, p->tile_lists, p->fwd, p->errflag, p->wave_ctl};
  for (void *b : bufs)
    if (b) cudaFree(b);
  cudaSetDevice(prev);
  delete p;
  return VI_OK;
}

extern "C" int vi_plan_reset(vi_plan *p, void *stream) {
  if (!p) return set_error(VI_ERR_ARG, "plan is NULL");
  cudaStream_t st = (cudaStream_t)stream;
  int rc;
  if (p->psix && (rc = cuda_check(cudaMemsetAsync(p->psix, 0, kPsiPlanes * (size_t)p->psix_plane * p->esize, st), "reset psi x")))
    return rc;
  if (p->psiz && (rc = cuda_check(cudaMemsetAsync(p->psiz, 0, kPsiPlanes * (size_t)p->psiz_plane * p->esize, st), "reset psi z")))
    return rc;
  if (p->slo && (rc = cuda_check(cudaMemsetAsync(p->slo, 0, 3 * (size_t)p->cfg.nx * p->cfg.nz * sizeof(uint16_t), st),
                                 "reset stress residues")))
    return rc;
  p->slo_valid = true;
  return VI_OK;
}

extern "C" int vi_plan_status(vi_plan *p, void *stream) {
  if (!p) return set_error(VI_ERR_ARG, "plan is NULL");
  int rc = cuda_check(cudaStreamSynchronize((cudaStream_t)stream), "plan status");
  if (rc) return rc;
  int flag = 0;
  rc = cuda_check(cudaMemcpy(&flag, p->errflag, sizeof(int), cudaMemcpyDeviceToHost), "read error word");
  if (rc) return rc;
  if (flag) {
    cudaMemset(p->errflag, 0, sizeof(int));
    if (flag & kErrTimeout)
      return set_error(VI_ERR_TIMEOUT, "a bounded device wait gave up (tile staging did not complete)");
    return set_error(VI_ERR_NONFINITE,
                     "a stress value came out NaN or infinite (non-finite medium or state, or an unstable run)");
  }
  return VI_OK;
}

extern "C" int vi_plan_last_kernel(const vi_plan *p, int32_t *kernel) {
  if (!p || !kernel) return set_error(VI_ERR_ARG, "NULL argument");
  *kernel = p->last_kernel;
  return VI_OK;
}

extern "C" int vi_plan_workspace_bytes(const vi_plan *p, int64_t *bytes) {
  if (!p || !bytes) return set_error(VI_ERR_ARG, "NULL argument");
  *bytes = (int64_t)p->bytes;
  return VI_OK;
}

extern "C" int vi_step(vi_plan *p, const vi_medium *med, vi_fields *f, const vi_shot *shot,
                       int32_t it0, int32_t nsteps, int32_t variant, void *stream) {
  if (!p) return set_error(VI_ERR_ARG, "plan is NULL");
  NvtxRange nr("vi_step");
  cudaStream_t st = (cudaStream_t)stream;
  return p->cfg.precision == VI_F64
             ? step_impl<double>(p, med, f, shot, it0, nsteps, variant, st)
             : step_impl<float>(p, med, f, shot, it0, nsteps, variant, st);
}

namespace vb {
template <typename T>
static int forward_host_impl(vi_plan *p, const vi_medium *mh, int nsrc, const vi_source *src,
                             const void *wavelet_host, int nrec, const vi_receiver *rec, int nt,
                             void *traces_host, vi_fields *final_host) {
  const vi_config &c = p->cfg;
  if (!mh) return set_error(VI_ERR_ARG, "medium is NULL");
  if (nt < 0 || nsrc < 0 || nrec < 0) return set_error(VI_ERR_ARG, "negative count");
  if (nsrc > 0 && (!src || !wavelet_host)) return set_error(VI_ERR_ARG, "sources need src and wavelet");
  if (nrec > 0 && (!rec || !traces_host)) return set_error(VI_ERR_ARG, "receivers need rec and traces");
  int rc = cuda_check(cudaSetDevice(p->device), "cudaSetDevice");
  if (rc) return rc;
  const size_t np = (size_t)c.nx * c.nz;
  const int nstate = 5 + 3 * c.nsls;
  const size_t bytes = (8 + nstate) * np * sizeof(T) + (size_t)nsrc * nt * sizeof(T) +
                       2 * (size_t)nrec * nt * sizeof(T) + 256 * 4;
  rc = ensure_buffer(p, &p->fwd, &p->fwd_bytes, bytes);
  if (rc) return rc;
  p->grad_zero_key = 0;  // the gradient's kept states are overwritten
  T *base = (T *)p->fwd;
  const void *hp[8] = {mh->rho, mh->c11, mh->c13, mh->c15, mh->c33, mh->c35, mh->c55, mh->tau};
  vi_medium md;
  const void **dp[8] = {&md.rho, &md.c11, &md.c13, &md.c15, &md.c33, &md.c35, &md.c55, &md.tau};
  for (int k = 0; k < 8; ++k) {
    *dp[k] = nullptr;
    if (hp[k]) {
      T *d = base + k * np;
      rc = cuda_check(cudaMemcpy(d, hp[k], np * sizeof(T), cudaMemcpyHostToDevice), "upload medium");
      if (rc) return rc;
      *dp[k] = d;
    }
  }
  rc = check_medium(p, &md);
  if (rc) return rc;
  T *state = base + 8 * np;
  rc = cuda_check(cudaMemset(state, 0, nstate * np * sizeof(T)), "zero state");
  if (rc) return rc;
  vi_fields fd;
  fd.vx = state;
  fd.vz = state + np;
  fd.sxx = state + 2 * np;
  fd.szz = state + 3 * np;
  fd.sxz = state + 4 * np;
  fd.m = c.nsls ? state + 5 * np : nullptr;
  fd.m_plane_stride = (long long)np;
  T *wav = state + nstate * np;
  T *tr = wav + (size_t)nsrc * nt;
  if (nsrc > 0) {
    rc = cuda_check(cudaMemcpy(wav, wavelet_host, (size_t)nsrc * nt * sizeof(T), cudaMemcpyHostToDevice),
                    "upload wavelets");
    if (rc) return rc;
  }
  if (nrec > 0) {
    rc = cuda_check(cudaMemset(tr, 0, 2 * (size_t)nrec * nt * sizeof(T)), "zero traces");
    if (rc) return rc;
  }
  rc = vi_plan_reset(p, nullptr);
  if (rc) return rc;
  vi_shot shot;
  shot.nsrc = nsrc;
  shot.src_host = src;
  shot.wavelet_dev = wav;
  shot.wavelet_nt = nt;
  shot.nrec = nrec;
  shot.rec_host = rec;
  shot.traces_dev = tr;
  shot.traces_nt = nt;
  rc = vi_step(p, &md, &fd, &shot, 0, nt, 0, nullptr);
  if (rc) return rc;
  if (nrec > 0) {
    rc = cuda_check(cudaMemcpy(traces_host, tr, 2 * (size_t)nrec * nt * sizeof(T), cudaMemcpyDeviceToHost),
                    "download traces");
    if (rc) return rc;
  }
  if (final_host) {
    void *dst[5] = {final_host->vx, final_host->vz, final_host->sxx, final_host->szz, final_host->sxz};
    for (int k = 0; k < 5; ++k)
      if (dst[k]) {
        rc = cuda_check(cudaMemcpy(dst[k], state + k * np, np * sizeof(T), cudaMemcpyDeviceToHost),
                        "download fields");
        if (rc) return rc;
      }
    if (final_host->m && c.nsls > 0)
      for (int k = 0; k < 3 * c.nsls; ++k) {
        rc = cuda_check(cudaMemcpy((char *)final_host->m + k * final_host->m_plane_stride * sizeof(T),
                                   state + (5 + k) * np, np * sizeof(T), cudaMemcpyDeviceToHost),
                        "download memory variables");
        if (rc) return rc;
      }
  }
  rc = cuda_check(cudaDeviceSynchronize(), "forward");
  if (rc) return rc;
  return vi_plan_status(p, nullptr);
}
}  // namespace vb

extern "C" int vi_forward_host(vi_plan *p, const vi_medium *med_host, int32_t nsrc,
                               const vi_source *src, const void *wavelet_host, int32_t nrec,
                               const vi_receiver *rec, int32_t nt, void *traces_host,
                               vi_fields *final_host) {
  if (!p) return set_error(VI_ERR_ARG, "plan is NULL");
  return p->cfg.precision == VI_F64
             ? forward_host_impl<double>(p, med_host, nsrc, src, wavelet_host, nrec, rec, nt,
                                         traces_host, final_host)
             : forward_host_impl<float>(p, med_host, nsrc, src, wavelet_host, nrec, rec, nt,
                                        traces_host, final_host);
}

extern "C" int vi_diff(int32_t precision, int32_t op, const void *u, void *du, int32_t nx,
                       int32_t nz, double h, void *stream) {
  if (!u || !du) return set_error(VI_ERR_ARG, "NULL array");
  if (op < 0 || op > 3) return set_error(VI_ERR_ARG, "op must be 0..3");
  if (nx < 2 * L + 1 || nz < 2 * L + 1) return set_error(VI_ERR_ARG, "grid too small");
  if (!(h > 0)) return set_error(VI_ERR_ARG, "h must be positive");
  cudaStream_t st = (cudaStream_t)stream;
  if (precision == VI_F64)
    diff_launch<double>(op, (const double *)u, (double *)du, nx, nz, h, st);
  else if (precision == VI_F32)
    diff_launch<float>(op, (const float *)u, (float *)du, nx, nz, h, st);
  else
    return set_error(VI_ERR_ARG, "unknown precision");
  return cuda_check(cudaGetLastError(), "diff launch");
}
