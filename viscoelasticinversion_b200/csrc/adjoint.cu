// adjoint.cu — discrete adjoint of the time step and the misfit gradient.
//
// J = 1/2 sum_n sum_r |d_n,r - obs_n,r|^2 over the vx and vz traces.  The
// gradient is the exact transpose of the forward step (plain in-place
// path, plain.cu), taken stage by stage in reverse:
//
//   forward step n:  V (velocity, CPML psi_sigma)  ->  receivers  ->
//                    S (SLS stress + memory variables, CPML psi_v, free
//                    surface)  ->  explosive sources  ->  stress images
//   reverse step n:  images^T -> S^T -> r^T (v += -D^T rbar) -> residual at
//                    the receivers -> V^T -> d^T (sigma += -D^T dbar)
//
// The transpose of ddxp is -ddxm (and of ddzp, -ddzm) over cells whose
// adjoint is zero outside the update region; each psi recursion
// psi' = b psi + a d, d~ = d/kappa + psi' transposes to
// dbar = dbar~/kappa + a (psibar' + dbar~), psibar = b (psibar' + dbar~).
//
// Memory: the state (v, sigma, M and the current psi set) is stored every
// K (default ceil(sqrt(nt))) steps; each segment is recomputed forward into
// K + 1 state slots and walked backwards.  Wavefields and the adjoint state
// are in the plan's precision; gradients and the misfit accumulate in FP64,
// each cell gathering its own terms (no atomics, deterministic).
//
// Gradients are with respect to the medium planes (rho, c11, c13, c33,
// c55, tau) — for ISO c13 = lambda and c55 = mu carry dJ/dlambda and
// dJ/dmu.  vi_gradient_velocity maps them to (vp, vs, rho, 1/Q) and, for
// VTI, vi_gradient_thomsen to the Thomsen (epsilon, delta).
#include <cmath>
#include <vector>

#include "fused.cuh"
#include "nvtx.cuh"
#include "fused_tma.cuh"
#include "pdl.cuh"
#include "plain.cuh"
#include "plan.cuh"
#include "split.cuh"
#include "vec.cuh"

namespace vb {

namespace {

template <typename T>
struct AdjArgs {
  int nx, nz, nsls, kind, fs;
  int Lx, Rx, Tz, Bz, wx, hz;
  T dt;
  T Dx[4], Dz[4];
  T a1[VI_MAX_SLS], a2[VI_MAX_SLS];
  const T *rho, *c11, *c13, *c33, *c55, *tau;
  const T *c15, *c35;  // TTI couplings
  const T *tx, *tz;
  long long np, psix_plane, psiz_plane;
};

// one state slot: [vx vz sxx szz sxz M(3N)] planes, then one psi set
// (4 x-strip planes, 4 z-strip planes)
template <typename T>
struct Slot {
  T *base;
  long long np, px, pz;  // plane sizes
  int nsls;
  __host__ __device__ T *vx() const { return base; }
  __host__ __device__ T *vz() const { return base + np; }
  __host__ __device__ T *sxx() const { return base + 2 * np; }
  __host__ __device__ T *szz() const { return base + 3 * np; }
  __host__ __device__ T *sxz() const { return base + 4 * np; }
  __host__ __device__ T *m() const { return base + 5 * np; }
  __host__ __device__ T *psix() const { return base + (5 + 3 * nsls) * np; }
  __host__ __device__ T *psiz() const { return psix() + 4 * px; }
  // rounded up to 64 elements, so every slot (and, with nx % 4 == 0, every
  // plane of it) starts on a 16-byte boundary, as the split kernels need
  __host__ __device__ static long long size(long long np, long long px, long long pz, int nsls) {
    return ((5 + 3 * nsls) * np + 4 * px + 4 * pz + 63) / 64 * 64;
  }
};

template <typename T>
__device__ __forceinline__ T tap_p(const T *u, long long c, long long s, const T *D) {  // ddxp/ddzp
  T v = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) v += D[k] * (u[c + (k + 1) * s] - u[c - k * s]);
  return v;
}
template <typename T>
__device__ __forceinline__ T tap_m(const T *u, long long c, long long s, const T *D) {  // ddxm/ddzm
  T v = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) v += D[k] * (u[c + k * s] - u[c - (k + 1) * s]);
  return v;
}
// bounds-checked forms for the transposes (u is zero outside its region)
template <typename T>
__device__ __forceinline__ T tap_p_b(const T *u, int i, int j, int nx, int nz, int ax, const T *D) {
  T v = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int a = k + 1, b = -k;
    const int ia = ax == 0 ? i + a : i, ja = ax == 0 ? j : j + a;
    const int ib = ax == 0 ? i + b : i, jb = ax == 0 ? j : j + b;
    const T ua = (ia >= 0 && ia < nx && ja >= 0 && ja < nz) ? u[(long long)ja * nx + ia] : T(0);
    const T ub = (ib >= 0 && ib < nx && jb >= 0 && jb < nz) ? u[(long long)jb * nx + ib] : T(0);
    v += D[k] * (ua - ub);
  }
  return v;
}
template <typename T>
__device__ __forceinline__ T tap_m_b(const T *u, int i, int j, int nx, int nz, int ax, const T *D) {
  T v = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int a = k, b = -(k + 1);
    const int ia = ax == 0 ? i + a : i, ja = ax == 0 ? j : j + a;
    const int ib = ax == 0 ? i + b : i, jb = ax == 0 ? j : j + b;
    const T ua = (ia >= 0 && ia < nx && ja >= 0 && ja < nz) ? u[(long long)ja * nx + ia] : T(0);
    const T ub = (ib >= 0 && ib < nx && jb >= 0 && jb < nz) ? u[(long long)jb * nx + ib] : T(0);
    v += D[k] * (ua - ub);
  }
  return v;
}

// CPML forward at one derivative: returns d~ (and the new psi in *pn)
template <typename T>
__device__ __forceinline__ T cpml_fwd(T d, T p0, T a, T b, T ik, T *pn) {
  const T p = b * p0 + a * d;
  *pn = p;
  return d * ik + p;
}

// ---- images^T: fold the ghost-row adjoints into the rows they mirror ----
// (all eight rows of a column are loaded before any store: the ghost and
// target rows are distinct, so the read-modify-writes need not serialise)
template <typename T>
__global__ void k_mirror_t(T *sb_zz, T *sb_xz, int nx) {
  pdl_wait();  // launched while the previous kernel drains
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nx) return;
  T gz[L], tz[L], gq[L], tq[L];
#pragma unroll
  for (int k = 1; k <= L; ++k) {
    gz[k - 1] = sb_zz[(long long)(L - k) * nx + i];
    tz[k - 1] = sb_zz[(long long)(L + k) * nx + i];
  }
#pragma unroll
  for (int k = 0; k < L; ++k) {
    gq[k] = sb_xz[(long long)(L - 1 - k) * nx + i];
    tq[k] = sb_xz[(long long)(L + k) * nx + i];
  }
#pragma unroll
  for (int k = 1; k <= L; ++k) {
    sb_zz[(long long)(L + k) * nx + i] = tz[k - 1] - gz[k - 1];
    sb_zz[(long long)(L - k) * nx + i] = T(0);
  }
#pragma unroll
  for (int k = 0; k < L; ++k) {
    sb_xz[(long long)(L + k) * nx + i] = tq[k] - gq[k];
    sb_xz[(long long)(L - 1 - k) * nx + i] = T(0);
  }
}

// ---- S^T: SLS stress stage transposed, per cell of the update region ----
// scratch planes: rbar[0..3] = (xx, zz, zx, xz) strain-rate adjoints, q = dt*sxzbar*exz.
// N (mechanisms) is a template parameter and every operand is loaded
// before the arithmetic, so the memory-variable and gradient
// read-modify-writes do not wait on one another.
template <typename T, int N>
__global__ void __launch_bounds__(256) k_stress_t(AdjArgs<T> A, Slot<T> x0, Slot<T> x1, Slot<T> ab,
                                                   T *rbar, T *q, double *gc11, double *gc13,
                                                   double *gc33, double *gtau) {
  pdl_wait();  // launched while the previous kernel drains
  constexpr int NM = N > 0 ? N : 1;
  const int i = blockIdx.x * blockDim.x + threadIdx.x + L;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + L;
  if (i >= A.nx - L || j >= A.nz - L) return;
  const int nx = A.nx;
  const long long c = (long long)j * nx + i, np = A.np;
  // ---- loads
  T mo[3 * NM], mbo[3 * NM];
#pragma unroll
  for (int k = 0; k < 3 * N; ++k) {
    mo[k] = x0.m()[k * np + c];
    mbo[k] = ab.m()[k * np + c];
  }
  T *sbx = ab.sxx(), *sbz = ab.szz(), *sbq = ab.sxz();
  const T bxx = sbx[c], bzz = sbz[c], bxz = sbq[c];
  const double g11o = gc11[c], g13o = gc13[c], g33o = gc33[c];
  const double gto = N > 0 ? gtau[c] : 0.0;
  const T tau = N > 0 ? A.tau[c] : T(0);
  const T c13 = A.c13[c], c55 = A.c55[c];
  const T c11 = A.kind == VI_MEDIUM_ISO ? T(0) : A.c11[c];
  const T c33 = A.kind == VI_MEDIUM_ISO ? T(0) : A.c33[c];
  const T c55r = A.c55[c + 1], c55b = A.c55[c + nx], c55br = A.c55[c + nx + 1];
  // forward strain rates from v(n+1) with the psi of step n
  T r[4];  // xx = ddxm vx, zz = ddzm vz, zx = ddzp vx, xz = ddxp vz
  r[0] = tap_m(x1.vx(), c, 1, A.Dx);
  r[1] = tap_m(x1.vz(), c, nx, A.Dz);
  r[2] = tap_p(x1.vx(), c, nx, A.Dz);
  r[3] = tap_p(x1.vz(), c, 1, A.Dx);
  T ik[4] = {1, 1, 1, 1}, ca[4] = {0, 0, 0, 0}, cb[4] = {0, 0, 0, 0};
  T *pb[4] = {nullptr, nullptr, nullptr, nullptr};
  T pbo[4] = {0, 0, 0, 0};
  const int xs = strip_x(i, nx, A.Lx, A.Rx), zs = strip_z(j, A.nz, A.Tz, A.Bz);
  if (xs >= 0) {
    const long long o = (long long)j * A.wx + xs;
    // x: xx at integer node (PX_VX), xz at half node (PX_VZ)
    ik[0] = A.tx[T_IK * nx + i]; ca[0] = A.tx[T_A * nx + i]; cb[0] = A.tx[T_B * nx + i];
    ik[3] = A.tx[T_IKH * nx + i]; ca[3] = A.tx[T_AH * nx + i]; cb[3] = A.tx[T_BH * nx + i];
    T pn;
    r[0] = cpml_fwd(r[0], x0.psix()[PX_VX * A.psix_plane + o], ca[0], cb[0], ik[0], &pn);
    r[3] = cpml_fwd(r[3], x0.psix()[PX_VZ * A.psix_plane + o], ca[3], cb[3], ik[3], &pn);
    pb[0] = ab.psix() + PX_VX * A.psix_plane + o;
    pb[3] = ab.psix() + PX_VZ * A.psix_plane + o;
    pbo[0] = *pb[0];
    pbo[3] = *pb[3];
  }
  if (zs >= 0) {
    const int nz = A.nz;
    const long long o = (long long)zs * nx + i;
    ik[1] = A.tz[T_IK * nz + j]; ca[1] = A.tz[T_A * nz + j]; cb[1] = A.tz[T_B * nz + j];
    ik[2] = A.tz[T_IKH * nz + j]; ca[2] = A.tz[T_AH * nz + j]; cb[2] = A.tz[T_BH * nz + j];
    T pn;
    r[1] = cpml_fwd(r[1], x0.psiz()[PZ_VZ * A.psiz_plane + o], ca[1], cb[1], ik[1], &pn);
    r[2] = cpml_fwd(r[2], x0.psiz()[PZ_VX * A.psiz_plane + o], ca[2], cb[2], ik[2], &pn);
    pb[1] = ab.psiz() + PZ_VZ * A.psiz_plane + o;
    pb[2] = ab.psiz() + PZ_VX * A.psiz_plane + o;
    pbo[1] = *pb[1];
    pbo[2] = *pb[2];
  }
  // ---- arithmetic
  const T rt[3] = {r[0], r[1], r[2] + r[3]};  // xx, zz, engineering xz
  T S[3] = {0, 0, 0};
#pragma unroll
  for (int n = 0; n < N; ++n)
#pragma unroll
    for (int k = 0; k < 3; ++k) S[k] += mo[k * N + n];
  T e[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) e[k] = N > 0 ? (T(1) + tau) * rt[k] + tau * S[k] : rt[k];
  const T C13 = c13;
  const T C11 = A.kind == VI_MEDIUM_ISO ? C13 + T(2) * c55 : c11;
  const T C33 = A.kind == VI_MEDIUM_ISO ? C11 : c33;
  const T C55h = T(0.25) * (c55 + c55r + c55b + c55br);
  const bool surf = A.fs && j == L;
  const T dt = A.dt;
  T eb[3];
  double g11 = g11o, g13 = g13o, g33 = g33o;
  if (!surf) {
    eb[0] = dt * (C11 * bxx + C13 * bzz);
    eb[1] = dt * (C13 * bxx + C33 * bzz);
    g11 += (double)dt * bxx * e[0];
    g13 += (double)dt * (bxx * e[1] + bzz * e[0]);
    g33 += (double)dt * bzz * e[1];
  } else {
    // sxx' = sxx + dt (C11 - C13^2/C33) exx; szz' = 0
    const T ceff = C11 - C13 * C13 / C33;
    eb[0] = dt * ceff * bxx;
    eb[1] = T(0);
    const double w = (double)dt * bxx * e[0];
    g11 += w;
    g13 += w * (-2.0 * (double)C13 / (double)C33);
    g33 += w * ((double)C13 * C13 / ((double)C33 * C33));
    sbz[c] = T(0);
  }
  gc11[c] = g11;
  gc13[c] = g13;
  gc33[c] = g33;
  eb[2] = dt * C55h * bxz;
  q[c] = dt * bxz * e[2];
  if (N > 0) {
    double gt = 0;
#pragma unroll
    for (int k = 0; k < 3; ++k) gt += (double)eb[k] * ((double)rt[k] + S[k]);
    gtau[c] = gto + gt;
  }
  // memory variables and the strain-rate adjoints
  T rtb[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) rtb[k] = (N > 0 ? (T(1) + tau) : T(1)) * eb[k];
#pragma unroll
  for (int n = 0; n < N; ++n) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const bool dead = surf && k == 1;  // Mzz' = 0 on the surface
      const T mb = dead ? T(0) : mbo[k * N + n];
      rtb[k] += dt * A.a1[n] * mb;
      ab.m()[(k * N + n) * np + c] = dead ? T(0) : tau * eb[k] + mb * (T(1) + dt * A.a2[n]);
    }
  }
  // psi transposes: rbar = rtbar/kappa + a (psibar' + rtbar), psibar = b (...)
  T rb[4] = {rtb[0], rtb[1], rtb[2], rtb[2]};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (pb[k]) {
      const T P = pbo[k] + rb[k];
      *pb[k] = cb[k] * P;
      rb[k] = rb[k] * ik[k] + ca[k] * P;
    }
    rbar[k * np + c] = rb[k];
  }
}


// ---- S^T for TTI media --------------------------------------------------
// The TTI stress law couples neighbouring cells (custom_solver/Model.jl:59-108
// on the staggered grid):
//   dsxx = C11 exx + C13 ezz + C15 ebxz,   dszz = C13 exx + C33 ezz + C35 ebxz,
//   dsxz = C55h exz + C15h ebxx + C35h ebzz,
// ebxz(i,j) the mean of exz over (i,j),(i-1,j),(i,j-1),(i-1,j-1), ebxx and
// ebzz the means of exx, ezz over (i,j),(i+1,j),(i,j+1),(i+1,j+1), C15h,
// C35h, C55h the means of the stiffness over the latter four cells, and on
// the free surface (row L) ezz = -(C13 exx + C35 ebxz) / C33.  Effective
// rates outside the update region U are zero.  The transpose runs in four
// kernels: the forward rates (k_tti_fwd_rates, k_tti_fwd_surface), the
// effective-rate adjoints gathered from the stress adjoints
// (k_tti_ebar_t), the surface relation transposed (k_tti_surface_t) and the
// per-cell rest — memory variables, tau, CPML psi (k_tti_stress_t).  Every
// cell gathers its own terms: no atomics.
template <typename T>
__device__ __forceinline__ bool in_u(int i, int j, int nx, int nz) {
  return i >= L && i < nx - L && j >= L && j < nz - L;
}

// Forward effective rates e (3 planes) and rt + S (3 planes: the CPML'd
// strain rates plus the memory-variable sums, de/dtau) of step it, from the
// new velocities (x1) and the CPML memory and memory variables before the
// step (x0).  fe is zero outside U.
template <typename T, int N>
__global__ void __launch_bounds__(256) k_tti_fwd_rates(AdjArgs<T> A, Slot<T> x0, Slot<T> x1, T *fe) {
  pdl_wait();  // launched while the previous kernel drains
  const int i = blockIdx.x * blockDim.x + threadIdx.x + L;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + L;
  if (i >= A.nx - L || j >= A.nz - L) return;
  const int nx = A.nx;
  const long long c = (long long)j * nx + i, np = A.np;
  T r[4];
  r[0] = tap_m(x1.vx(), c, 1, A.Dx);
  r[1] = tap_m(x1.vz(), c, nx, A.Dz);
  r[2] = tap_p(x1.vx(), c, nx, A.Dz);
  r[3] = tap_p(x1.vz(), c, 1, A.Dx);
  const int xs = strip_x(i, nx, A.Lx, A.Rx), zs = strip_z(j, A.nz, A.Tz, A.Bz);
  T pn;
  if (xs >= 0) {
    const long long o = (long long)j * A.wx + xs;
    r[0] = cpml_fwd(r[0], x0.psix()[PX_VX * A.psix_plane + o], A.tx[T_A * nx + i], A.tx[T_B * nx + i],
                    A.tx[T_IK * nx + i], &pn);
    r[3] = cpml_fwd(r[3], x0.psix()[PX_VZ * A.psix_plane + o], A.tx[T_AH * nx + i], A.tx[T_BH * nx + i],
                    A.tx[T_IKH * nx + i], &pn);
  }
  if (zs >= 0) {
    const int nz = A.nz;
    const long long o = (long long)zs * nx + i;
    r[1] = cpml_fwd(r[1], x0.psiz()[PZ_VZ * A.psiz_plane + o], A.tz[T_A * nz + j], A.tz[T_B * nz + j],
                    A.tz[T_IK * nz + j], &pn);
    r[2] = cpml_fwd(r[2], x0.psiz()[PZ_VX * A.psiz_plane + o], A.tz[T_AH * nz + j], A.tz[T_BH * nz + j],
                    A.tz[T_IKH * nz + j], &pn);
  }
  const T rt[3] = {r[0], r[1], r[2] + r[3]};
  T S[3] = {0, 0, 0};
#pragma unroll
  for (int n = 0; n < N; ++n)
#pragma unroll
    for (int k = 0; k < 3; ++k) S[k] += x0.m()[(k * N + n) * np + c];
  const T tau = N > 0 ? A.tau[c] : T(0);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    fe[k * np + c] = N > 0 ? (T(1) + tau) * rt[k] + tau * S[k] : rt[k];
    fe[(3 + k) * np + c] = rt[k] + S[k];
  }
}

// The free-surface relation of the forward step on row L:
// ezz = -(C13 exx + C35 ebxz) / C33 (row L - 1 lies outside U: zero there).
template <typename T>
__global__ void k_tti_fwd_surface(AdjArgs<T> A, T *fe) {
  pdl_wait();  // launched while the previous kernel drains
  const int i = blockIdx.x * blockDim.x + threadIdx.x + L;
  if (i >= A.nx - L) return;
  const int nx = A.nx;
  const long long np = A.np, c = (long long)L * nx + i;
  const T *exx = fe, *exz = fe + 2 * np;
  const T eb = T(0.25) * (exz[c] + exz[c - 1] + exz[c - nx] + exz[c - nx - 1]);
  fe[np + c] = -(A.c13[c] * exx[c] + A.c35[c] * eb) / A.c33[c];
}

// Adjoints of the effective rates (3 planes eb) gathered from the stress
// adjoints of the cells whose update reads them, and the direct stiffness
// gradient terms: C11, C13, C33, C15 and C35 at the cell, and the
// per-cell products q (C55h), q15 (C15h), q35 (C35h) that k_gather and
// k_tti_gather spread over the four cells of each half-node mean.  On the
// free surface the stress szz is reset after the update, so its adjoint
// there is zero.
template <typename T>
__global__ void __launch_bounds__(256) k_tti_ebar_t(AdjArgs<T> A, Slot<T> ab, const T *fe, T *eb, T *q,
                                                     T *q15, T *q35, double *g11, double *g13, double *g15,
                                                     double *g33, double *g35) {
  pdl_wait();  // launched while the previous kernel drains
  const int i = blockIdx.x * blockDim.x + threadIdx.x + L;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + L;
  const int nx = A.nx, nz = A.nz;
  if (i >= nx - L || j >= nz - L) return;
  const long long c = (long long)j * nx + i, np = A.np;
  const T *sbx = ab.sxx(), *sbz = ab.szz(), *sbq = ab.sxz();
  const T *exx = fe, *ezz = fe + np, *exz = fe + 2 * np;
  const T dt = A.dt;
  auto bzz = [&](int ii, int jj) -> T {  // szz adjoint of a cell of U (zero on the surface)
    return (A.fs && jj == L) ? T(0) : sbz[(long long)jj * nx + ii];
  };
  auto mean4p = [&](const T *u, long long cc) { return T(0.25) * (u[cc] + u[cc + 1] + u[cc + nx] + u[cc + nx + 1]); };
  const T bxx = sbx[c], bzc = bzz(i, j), bxz = sbq[c];
  const T C11 = A.c11[c], C13 = A.c13[c], C33 = A.c33[c], C15 = A.c15[c], C35 = A.c35[c];
  const T C55h = mean4p(A.c55, c);
  // exz feeds sxx, szz of the cells (i,j), (i+1,j), (i,j+1), (i+1,j+1)
  T sq = 0;
#pragma unroll
  for (int dj = 0; dj <= 1; ++dj)
#pragma unroll
    for (int di = 0; di <= 1; ++di) {
      const int ii = i + di, jj = j + dj;
      if (in_u<T>(ii, jj, nx, nz)) {
        const long long cc = (long long)jj * nx + ii;
        sq += A.c15[cc] * sbx[cc] + A.c35[cc] * bzz(ii, jj);
      }
    }
  // exx, ezz feed sxz of the cells (i,j), (i-1,j), (i,j-1), (i-1,j-1)
  T sx = 0, sz = 0;
#pragma unroll
  for (int dj = 0; dj <= 1; ++dj)
#pragma unroll
    for (int di = 0; di <= 1; ++di) {
      const int ii = i - di, jj = j - dj;
      if (in_u<T>(ii, jj, nx, nz)) {
        const long long cc = (long long)jj * nx + ii;
        sx += mean4p(A.c15, cc) * sbq[cc];
        sz += mean4p(A.c35, cc) * sbq[cc];
      }
    }
  eb[c] = dt * (C11 * bxx + C13 * bzc + T(0.25) * sx);
  eb[np + c] = dt * (C13 * bxx + C33 * bzc + T(0.25) * sz);
  eb[2 * np + c] = dt * (C55h * bxz + T(0.25) * sq);
  // forward rates at the cell and the neighbour means its update used
  const T ex = exx[c], ez = ezz[c], eq = exz[c];
  const T ebxz = T(0.25) * (exz[c] + exz[c - 1] + exz[c - nx] + exz[c - nx - 1]);
  const T ebxx = mean4p(exx, c), ebzz = mean4p(ezz, c);
  g11[c] += (double)dt * bxx * ex;
  g13[c] += (double)dt * ((double)bxx * ez + (double)bzc * ex);
  g33[c] += (double)dt * bzc * ez;
  g15[c] += (double)dt * bxx * ebxz;
  g35[c] += (double)dt * bzc * ebxz;
  q[c] = dt * bxz * eq;
  q15[c] = dt * bxz * ebxx;
  q35[c] = dt * bxz * ebzz;
}

// The surface relation transposed (row L): the adjoint of the surface ezz
// (as k_tti_ebar_t gathered it) moves to exx of the cell and to exz of the
// cell and its left neighbour, and adds its stiffness terms; the surface
// ezz adjoint itself is read as zero afterwards (k_tti_stress_t).
template <typename T>
__global__ void k_tti_surface_t(AdjArgs<T> A, const T *fe, T *eb, double *g13, double *g33, double *g35) {
  pdl_wait();  // launched while the previous kernel drains
  const int i = blockIdx.x * blockDim.x + threadIdx.x + L;
  const int nx = A.nx;
  if (i >= nx - L) return;
  const long long np = A.np, c = (long long)L * nx + i;
  const T *exx = fe, *ezz = fe + np, *exz = fe + 2 * np;
  const T zb = eb[np + c];
  const T C33 = A.c33[c];
  eb[c] += -A.c13[c] / C33 * zb;
  T xz = -T(0.25) * A.c35[c] / C33 * zb;
  if (i + 1 < nx - L) xz -= T(0.25) * A.c35[c + 1] / A.c33[c + 1] * eb[np + c + 1];
  eb[2 * np + c] += xz;
  const T ebs = T(0.25) * (exz[c] + exz[c - 1] + exz[c - nx] + exz[c - nx - 1]);
  g13[c] += -(double)zb * exx[c] / C33;
  g35[c] += -(double)zb * ebs / C33;
  g33[c] += -(double)zb * ezz[c] / C33;
}

// Memory variables, the tau gradient and the CPML psi transposes of a TTI
// cell, from the effective-rate adjoints: rbar (4 planes) as k_stress_t
// leaves it.
template <typename T, int N>
__global__ void __launch_bounds__(256) k_tti_stress_t(AdjArgs<T> A, Slot<T> ab, const T *fe, const T *eb,
                                                       T *rbar, double *gtau) {
  pdl_wait();  // launched while the previous kernel drains
  const int i = blockIdx.x * blockDim.x + threadIdx.x + L;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + L;
  const int nx = A.nx;
  if (i >= nx - L || j >= A.nz - L) return;
  const long long c = (long long)j * nx + i, np = A.np;
  const bool surf = A.fs && j == L;
  T e_b[3] = {eb[c], surf ? T(0) : eb[np + c], eb[2 * np + c]};
  if (surf) ab.szz()[c] = T(0);
  const T tau = N > 0 ? A.tau[c] : T(0);
  if (N > 0) {
    double gt = 0;
#pragma unroll
    for (int k = 0; k < 3; ++k) gt += (double)e_b[k] * fe[(3 + k) * np + c];
    gtau[c] += gt;
  }
  T rtb[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) rtb[k] = (N > 0 ? (T(1) + tau) : T(1)) * e_b[k];
#pragma unroll
  for (int n = 0; n < N; ++n) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const bool dead = surf && k == 1;  // Mzz' = 0 on the surface
      T *mp = ab.m() + (k * N + n) * np + c;
      const T mb = dead ? T(0) : *mp;
      rtb[k] += A.dt * A.a1[n] * mb;
      *mp = dead ? T(0) : tau * e_b[k] + mb * (T(1) + A.dt * A.a2[n]);
    }
  }
  T ik[4] = {1, 1, 1, 1}, ca[4] = {0, 0, 0, 0}, cb[4] = {0, 0, 0, 0};
  T *pb[4] = {nullptr, nullptr, nullptr, nullptr};
  const int xs = strip_x(i, nx, A.Lx, A.Rx), zs = strip_z(j, A.nz, A.Tz, A.Bz);
  if (xs >= 0) {
    const long long o = (long long)j * A.wx + xs;
    ik[0] = A.tx[T_IK * nx + i]; ca[0] = A.tx[T_A * nx + i]; cb[0] = A.tx[T_B * nx + i];
    ik[3] = A.tx[T_IKH * nx + i]; ca[3] = A.tx[T_AH * nx + i]; cb[3] = A.tx[T_BH * nx + i];
    pb[0] = ab.psix() + PX_VX * A.psix_plane + o;
    pb[3] = ab.psix() + PX_VZ * A.psix_plane + o;
  }
  if (zs >= 0) {
    const int nz = A.nz;
    const long long o = (long long)zs * nx + i;
    ik[1] = A.tz[T_IK * nz + j]; ca[1] = A.tz[T_A * nz + j]; cb[1] = A.tz[T_B * nz + j];
    ik[2] = A.tz[T_IKH * nz + j]; ca[2] = A.tz[T_AH * nz + j]; cb[2] = A.tz[T_BH * nz + j];
    pb[1] = ab.psiz() + PZ_VZ * A.psiz_plane + o;
    pb[2] = ab.psiz() + PZ_VX * A.psiz_plane + o;
  }
  T rb[4] = {rtb[0], rtb[1], rtb[2], rtb[2]};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (pb[k]) {
      const T P = *pb[k] + rb[k];
      *pb[k] = cb[k] * P;
      rb[k] = rb[k] * ik[k] + ca[k] * P;
    }
    rbar[k * np + c] = rb[k];
  }
}

// C15 and C35 gather the half-node products of the four means they enter
// (as k_gather does for C55)
template <typename T>
__global__ void k_tti_gather(const T *q15, const T *q35, double *g15, double *g35, int nx, int nz) {
  pdl_wait();  // launched while the previous kernel drains
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= nx || j >= nz) return;
  const long long c = (long long)j * nx + i;
  double t15 = 0, t35 = 0;
  for (int dj = 0; dj <= 1; ++dj)
    for (int di = 0; di <= 1; ++di) {
      const int ii = i - di, jj = j - dj;
      if (ii >= 0 && jj >= 0) {
        t15 += q15[(long long)jj * nx + ii];
        t35 += q35[(long long)jj * nx + ii];
      }
    }
  g15[c] += 0.25 * t15;
  g35[c] += 0.25 * t35;
}

// v += -D^T rbar over the update region (its taps reach at most L cells,
// so they stay inside the planes; rbar is zero outside the region)
template <typename T>
__global__ void k_rates_t(AdjArgs<T> A, Slot<T> ab, const T *rbar) {
  pdl_wait();  // launched while the previous kernel drains
  const int i = blockIdx.x * blockDim.x + threadIdx.x + L;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + L;
  if (i >= A.nx - L || j >= A.nz - L) return;
  const int nx = A.nx;
  const long long c = (long long)j * nx + i, np = A.np;
  const T vx = ab.vx()[c], vz = ab.vz()[c];
  ab.vx()[c] = vx - (tap_p(rbar, c, 1, A.Dx) + tap_m(rbar + 2 * np, c, nx, A.Dz));
  ab.vz()[c] = vz - (tap_p(rbar + np, c, nx, A.Dz) + tap_m(rbar + 3 * np, c, 1, A.Dx));
}

// residual at the receivers of step it: vbar += d - obs
template <typename T>
__global__ void k_residual(Slot<T> ab, Slot<T> x1, const int2 *rec, int nrec, const T *obs, int ont,
                           int it, int nx) {
  pdl_wait();  // launched while the previous kernel drains
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nrec) return;
  const long long c = (long long)rec[r].y * nx + rec[r].x;
  atomicAdd(ab.vx() + c, x1.vx()[c] - obs[(long long)r * ont + it]);
  atomicAdd(ab.vz() + c, x1.vz()[c] - obs[(long long)(nrec + r) * ont + it]);
}

// V^T per cell: dbar (4 planes: sxx-x, sxz-z, sxz-x, szz-z) and the
// buoyancy-gradient terms h (2 planes)
template <typename T>
__global__ void __launch_bounds__(256) k_vel_t(AdjArgs<T> A, Slot<T> x0, Slot<T> ab, T *dbar, T *h) {
  pdl_wait();  // launched while the previous kernel drains
  const int i = blockIdx.x * blockDim.x + threadIdx.x + L;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + L;
  if (i >= A.nx - L || j >= A.nz - L) return;
  const int nx = A.nx, nz = A.nz;
  const long long c = (long long)j * nx + i, np = A.np;
  T d[4];
  d[0] = tap_p(x0.sxx(), c, 1, A.Dx);   // ddxp sxx   (x, half)
  d[1] = tap_m(x0.sxz(), c, nx, A.Dz);  // ddzm sxz   (z, integer)
  d[2] = tap_m(x0.sxz(), c, 1, A.Dx);   // ddxm sxz   (x, integer)
  d[3] = tap_p(x0.szz(), c, nx, A.Dz);  // ddzp szz   (z, half)
  T ik[4] = {1, 1, 1, 1}, ca[4] = {0, 0, 0, 0}, cb[4] = {0, 0, 0, 0};
  T *pb[4] = {nullptr, nullptr, nullptr, nullptr};
  const int xs = strip_x(i, nx, A.Lx, A.Rx), zs = strip_z(j, nz, A.Tz, A.Bz);
  T pn;
  if (xs >= 0) {
    const long long o = (long long)j * A.wx + xs;
    ik[0] = A.tx[T_IKH * nx + i]; ca[0] = A.tx[T_AH * nx + i]; cb[0] = A.tx[T_BH * nx + i];
    ik[2] = A.tx[T_IK * nx + i]; ca[2] = A.tx[T_A * nx + i]; cb[2] = A.tx[T_B * nx + i];
    d[0] = cpml_fwd(d[0], x0.psix()[PX_SXX * A.psix_plane + o], ca[0], cb[0], ik[0], &pn);
    d[2] = cpml_fwd(d[2], x0.psix()[PX_SXZ * A.psix_plane + o], ca[2], cb[2], ik[2], &pn);
    pb[0] = ab.psix() + PX_SXX * A.psix_plane + o;
    pb[2] = ab.psix() + PX_SXZ * A.psix_plane + o;
  }
  if (zs >= 0) {
    const long long o = (long long)zs * nx + i;
    ik[1] = A.tz[T_IK * nz + j]; ca[1] = A.tz[T_A * nz + j]; cb[1] = A.tz[T_B * nz + j];
    ik[3] = A.tz[T_IKH * nz + j]; ca[3] = A.tz[T_AH * nz + j]; cb[3] = A.tz[T_BH * nz + j];
    d[1] = cpml_fwd(d[1], x0.psiz()[PZ_SXZ * A.psiz_plane + o], ca[1], cb[1], ik[1], &pn);
    d[3] = cpml_fwd(d[3], x0.psiz()[PZ_SZZ * A.psiz_plane + o], ca[3], cb[3], ik[3], &pn);
    pb[1] = ab.psiz() + PZ_SXZ * A.psiz_plane + o;
    pb[3] = ab.psiz() + PZ_SZZ * A.psiz_plane + o;
  }
  T pbo[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) pbo[k] = pb[k] ? *pb[k] : T(0);
  const T bx = T(2) / (A.rho[c] + A.rho[c + 1]);
  const T bz = T(2) / (A.rho[c] + A.rho[c + nx]);
  const T vbx = ab.vx()[c], vbz = ab.vz()[c];
  // d(vx')/d rho = dt * (-bx^2 / 2) * div
  h[c] = A.dt * T(-0.5) * bx * bx * (d[0] + d[1]) * vbx;
  h[np + c] = A.dt * T(-0.5) * bz * bz * (d[2] + d[3]) * vbz;
  T db[4] = {A.dt * bx * vbx, A.dt * bx * vbx, A.dt * bz * vbz, A.dt * bz * vbz};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (pb[k]) {
      const T P = pbo[k] + db[k];
      *pb[k] = cb[k] * P;
      db[k] = db[k] * ik[k] + ca[k] * P;
    }
    dbar[k * np + c] = db[k];
  }
}

// force sources: their buoyancy factor also depends on rho
template <typename T>
__global__ void k_force_rho_t(AdjArgs<T> A, Slot<T> ab, const int4 *src, const T *amp, int nsrc,
                              const T *wav, int wnt, int it, T *h) {
  pdl_wait();  // launched while the previous kernel drains
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nsrc) return;
  const int4 s = src[q];
  if (s.z == VI_SRC_EXPLOSIVE) return;
  const long long c = (long long)s.y * A.nx + s.x;
  const T f = it < wnt ? amp[q] * wav[(long long)q * wnt + it] : T(0);
  if (s.z == VI_SRC_FORCE_X) {
    const T bx = T(2) / (A.rho[c] + A.rho[c + 1]);
    atomicAdd(h + c, A.dt * T(-0.5) * bx * bx * f * ab.vx()[c]);
  } else {
    const T bz = T(2) / (A.rho[c] + A.rho[c + A.nx]);
    atomicAdd(h + A.np + c, A.dt * T(-0.5) * bz * bz * f * ab.vz()[c]);
  }
}

// grho gathers h of the two velocity nodes each density value feeds;
// gc55 gathers the 4 half-node terms q that average mu around each cell
template <typename T>
__global__ void k_gather(const T *h, double *grho, const T *q, double *gc55, int nx, int nz) {
  pdl_wait();  // launched while the previous kernel drains
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= nx || j >= nz) return;
  const long long c = (long long)j * nx + i, np = (long long)nx * nz;
  const double gr = grho[c], g55 = gc55[c];
  double s = (double)h[c] + (double)h[np + c];
  if (i > 0) s += h[c - 1];
  if (j > 0) s += h[np + c - nx];
  double t = 0;
  for (int dj = 0; dj <= 1; ++dj)
    for (int di = 0; di <= 1; ++di) {
      const int ii = i - di, jj = j - dj;
      if (ii >= 0 && jj >= 0) t += q[(long long)jj * nx + ii];
    }
  grho[c] = gr + s;
  gc55[c] = g55 + 0.25 * t;
}

// sigma += -D^T dbar over every cell the velocity stencil reads (ghost rows
// included; the images^T of the previous step folds them)
template <typename T>
__global__ void k_div_t(AdjArgs<T> A, Slot<T> ab, const T *dbar) {
  pdl_wait();  // launched while the previous kernel drains
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= A.nx || j >= A.nz) return;
  const int nx = A.nx, nz = A.nz;
  const long long c = (long long)j * nx + i, np = A.np;
  const T sxx = ab.sxx()[c], sxz = ab.sxz()[c], szz = ab.szz()[c];
  if (i >= L && i < nx - L && j >= L && j < nz - L) {  // taps inside the planes: unchecked
    ab.sxx()[c] = sxx - tap_m(dbar, c, 1, A.Dx);
    ab.sxz()[c] = sxz - (tap_p(dbar + np, c, nx, A.Dz) + tap_p(dbar + 2 * np, c, 1, A.Dx));
    ab.szz()[c] = szz - tap_m(dbar + 3 * np, c, nx, A.Dz);
  } else {
    ab.sxx()[c] = sxx - tap_m_b(dbar, i, j, nx, nz, 0, A.Dx);
    ab.sxz()[c] = sxz - (tap_p_b(dbar + np, i, j, nx, nz, 1, A.Dz) + tap_p_b(dbar + 2 * np, i, j, nx, nz, 0, A.Dx));
    ab.szz()[c] = szz - tap_m_b(dbar + 3 * np, i, j, nx, nz, 1, A.Dz);
  }
}

// ---- 4-cell forms of the transposed derivatives (nx % 4 == 0, 16-byte
// aligned planes): one thread per group of 4 x-adjacent cells, x taps from
// a 12-value row window of three 128-bit loads, z taps as one 128-bit load
// per row; per cell the same arithmetic as the scalar kernels.
template <typename T>
__device__ __forceinline__ void win12(const T *p, T (&o)[12]) {  // p[-4 .. +7]
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const Q4<T> v = ldc4(p - 4 + 4 * q);
#pragma unroll
    for (int k = 0; k < 4; ++k) o[4 * q + k] = v.v[k];
  }
}
template <typename T>
__device__ __forceinline__ Q4<T> zp4(const T *p, long long s, const T *D) {  // ddzp form
  Q4<T> acc = mul4(splat4<T>(D[0]), sub4(ldc4(p + s), ldc4(p)));
#pragma unroll
  for (int q = 1; q < 4; ++q) acc = fma4(splat4<T>(D[q]), sub4(ldc4(p + (q + 1) * s), ldc4(p - q * s)), acc);
  return acc;
}
template <typename T>
__device__ __forceinline__ Q4<T> zm4(const T *p, long long s, const T *D) {  // ddzm form
  Q4<T> acc = mul4(splat4<T>(D[0]), sub4(ldc4(p), ldc4(p - s)));
#pragma unroll
  for (int q = 1; q < 4; ++q) acc = fma4(splat4<T>(D[q]), sub4(ldc4(p + q * s), ldc4(p - (q + 1) * s)), acc);
  return acc;
}

// v += -D^T rbar, 4 cells per thread over the update region
template <typename T>
__global__ void __launch_bounds__(256) k_rates_t4(AdjArgs<T> A, Slot<T> ab, const T *rbar) {
  pdl_wait();  // launched while the previous kernel drains
  const int gi0 = L + 4 * (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int j = L + (int)(blockIdx.y * blockDim.y + threadIdx.y);
  if (gi0 >= A.nx - L || j >= A.nz - L) return;
  const int nx = A.nx;
  const long long g = (long long)j * nx + gi0, np = A.np;
  T w0[12], w3[12];
  win12(rbar + g, w0);
  win12(rbar + 3 * np + g, w3);
  const Q4<T> x0 = dps4(w0, A.Dx), x3 = dms4(w3, A.Dx);
  const Q4<T> z2 = zm4(rbar + 2 * np + g, nx, A.Dz), z1 = zp4(rbar + np + g, nx, A.Dz);
  const Q4<T> vx = ldc4(ab.vx() + g), vz = ldc4(ab.vz() + g);
  stg4(ab.vx() + g, sub4(vx, add4(x0, z2)));
  stg4(ab.vz() + g, sub4(vz, add4(z1, x3)));
}

// sigma += -D^T dbar, 4 cells per thread over every cell (groups whose taps
// leave the planes take the checked scalar form)
template <typename T>
__global__ void __launch_bounds__(256) k_div_t4(AdjArgs<T> A, Slot<T> ab, const T *dbar) {
  pdl_wait();  // launched while the previous kernel drains
  const int gi0 = 4 * (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int j = (int)(blockIdx.y * blockDim.y + threadIdx.y);
  const int nx = A.nx, nz = A.nz;
  if (gi0 >= nx || j >= nz) return;
  const long long g = (long long)j * nx + gi0, np = A.np;
  if (gi0 >= L && gi0 + 3 < nx - L && j >= L && j < nz - L) {
    T w0[12], w2[12];
    win12(dbar + g, w0);
    win12(dbar + 2 * np + g, w2);
    const Q4<T> sxx = ldc4(ab.sxx() + g), sxz = ldc4(ab.sxz() + g), szz = ldc4(ab.szz() + g);
    stg4(ab.sxx() + g, sub4(sxx, dms4(w0, A.Dx)));
    stg4(ab.sxz() + g, sub4(sxz, add4(zp4(dbar + np + g, nx, A.Dz), dps4(w2, A.Dx))));
    stg4(ab.szz() + g, sub4(szz, zm4(dbar + 3 * np + g, nx, A.Dz)));
  } else {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int i = gi0 + k;
      const long long c = g + k;
      const T sxx = ab.sxx()[c], sxz = ab.sxz()[c], szz = ab.szz()[c];
      ab.sxx()[c] = sxx - tap_m_b(dbar, i, j, nx, nz, 0, A.Dx);
      ab.sxz()[c] = sxz - (tap_p_b(dbar + np, i, j, nx, nz, 1, A.Dz) + tap_p_b(dbar + 2 * np, i, j, nx, nz, 0, A.Dx));
      ab.szz()[c] = szz - tap_m_b(dbar + 3 * np, i, j, nx, nz, 1, A.Dz);
    }
  }
}

// FP64 misfit: 1/2 sum (d - obs)^2 (one block, deterministic order)
template <typename T>
__global__ void k_misfit(const T *tr, const T *obs, long long n, double *out) {
  __shared__ double red[256];
  double s = 0;
  for (long long k = threadIdx.x; k < n; k += blockDim.x) {
    const double d = (double)tr[k] - (double)obs[k];
    s += d * d;
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = 0.5 * red[0];
}

// ISO fold and the (vp, vs, rho, 1/Q) chain rule
__global__ void k_velocity_grad(int kind, long long np, const double *g, const double *vp,
                                const double *vs, const double *rho, const double *eps,
                                const double *delta, double tau_scale, double *out) {
  const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= np) return;
  const double grho = g[0 * np + c], g11 = g[1 * np + c], g13 = g[2 * np + c];
  const double g33 = g[4 * np + c], g55 = g[6 * np + c], gtau = g[7 * np + c];
  const double p = vp[c], s = vs[c], r = rho[c];
  double gC33, gC55;
  if (kind == VI_MEDIUM_ISO) {
    // g13 slot carries dJ/dlambda, g55 slot dJ/dmu (already folded)
    const double gl = g13, gm = g55;
    gC33 = gl;          // lambda = rho (vp^2 - 2 vs^2): d/dvp via vp^2
    gC55 = gm - 2 * gl; // mu = rho vs^2
  } else {
    const double e = eps ? eps[c] : 0.0, d = delta ? delta[c] : 0.0;
    const double C33 = r * p * p, C55 = r * s * s;
    const double A = C33 - C55, B = C33 * (1 + 2 * d) - C55;
    const double sq = sqrt(fmax(A * B, 1e-300));
    const double dC13_dC33 = (B + A * (1 + 2 * d)) / (2 * sq);
    const double dC13_dC55 = (-B - A) / (2 * sq) - 1.0;
    gC33 = g33 + g11 * (1 + 2 * e) + g13 * dC13_dC33;
    gC55 = g55 + g13 * dC13_dC55;
  }
  out[0 * np + c] = gC33 * 2 * r * p;                 // dJ/dvp
  out[1 * np + c] = gC55 * 2 * r * s;                 // dJ/dvs
  out[2 * np + c] = grho + gC33 * p * p + gC55 * s * s;  // dJ/drho at fixed vp, vs
  out[3 * np + c] = gtau * tau_scale;                 // dJ/d(1/Q)
}

// VTI Thomsen parameters at fixed (vp, vs, rho): C11 = C33 (1 + 2 eps)
// gives dC11/deps = 2 C33; C13 = sqrt(A B) - C55 with A = C33 - C55,
// B = C33 (1 + 2 delta) - C55 gives dC13/ddelta = A C33 / sqrt(A B)
// (media.thomsen_vti; custom_solver/Model.jl:12-16).  gamma enters only SH
// motion: no 2D P-SV stiffness depends on it.
__global__ void k_thomsen_grad(long long np, const double *g, const double *vp, const double *vs,
                               const double *rho, const double *delta, double *out) {
  const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= np) return;
  const double g11 = g[1 * np + c], g13 = g[2 * np + c];
  const double r = rho[c], C33 = r * vp[c] * vp[c], C55 = r * vs[c] * vs[c];
  const double d = delta ? delta[c] : 0.0;
  const double A = C33 - C55, B = C33 * (1 + 2 * d) - C55;
  const double sq = sqrt(fmax(A * B, 1e-300));
  out[0 * np + c] = g11 * 2 * C33;     // dJ/deps
  out[1 * np + c] = g13 * A * C33 / sq;  // dJ/ddelta
}

// Forward-mode derivative pairs (value, d/dp) for the TTI chain rule.
struct Dual {
  double v, d;
};
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ Dual operator*(double s, Dual a) { return {s * a.v, s * a.d}; }
__device__ __forceinline__ Dual dsqrt(Dual a) {
  const double r = sqrt(fmax(a.v, 1e-300));
  return {r, a.d / (2.0 * r)};
}

// The TTI stiffness of one cell from (vp, vs, rho, epsilon, delta, theta):
// Thomsen's VTI law (Models.jl:27-52, custom_solver/Model.jl:12-16) tilted
// by the 2D Bond rotation (the map of vi_medium_from_velocity), carried on
// derivative pairs.  out = (C11, C13, C15, C33, C35, C55).
__device__ __forceinline__ void tti_stiffness(Dual p, Dual s, Dual r, Dual e, Dual d, Dual th, Dual (&out)[6]) {
  const Dual C33 = r * p * p, C55 = r * s * s;
  const Dual C11 = C33 * Dual{1.0 + 2.0 * e.v, 2.0 * e.d};
  const Dual C13 = dsqrt((C33 - C55) * (C33 * Dual{1.0 + 2.0 * d.v, 2.0 * d.d} - C55)) - C55;
  const Dual co{cos(th.v), -sin(th.v) * th.d}, si{sin(th.v), cos(th.v) * th.d};
  const Dual c2 = co * co, s2 = si * si, cs = co * si, A = C13 + 2.0 * C55, dcs = c2 - s2;
  out[0] = c2 * c2 * C11 + 2.0 * (c2 * s2 * A) + s2 * s2 * C33;
  out[1] = c2 * s2 * (C11 + C33 - 4.0 * C55) + (c2 * c2 + s2 * s2) * C13;
  out[2] = -1.0 * (cs * (c2 * C11 - s2 * C33 - dcs * A));
  out[3] = s2 * s2 * C11 + 2.0 * (c2 * s2 * A) + c2 * c2 * C33;
  out[4] = -1.0 * (cs * (s2 * C11 - c2 * C33 + dcs * A));
  out[5] = c2 * s2 * (C11 + C33 - 2.0 * C13) + dcs * dcs * C55;
}

// dJ/d(vp, vs, rho, 1/Q, epsilon, delta, theta) of a TTI medium from the
// stiffness gradient g (vi_gradient's eight planes): the chain rule through
// tti_stiffness, one derivative direction per parameter.
__global__ void k_tti_param_grad(long long np, const double *g, const double *vp, const double *vs,
                                 const double *rho, const double *eps, const double *delta,
                                 const double *theta, double tau_scale, double *out) {
  const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= np) return;
  const double gk[6] = {g[1 * np + c], g[2 * np + c], g[3 * np + c], g[4 * np + c], g[5 * np + c], g[6 * np + c]};
  const double val[6] = {vp[c], vs[c], rho[c], eps ? eps[c] : 0.0, delta ? delta[c] : 0.0, theta ? theta[c] : 0.0};
  const int slot[6] = {0, 1, 2, 4, 5, 6};  // output plane of each parameter (3 is 1/Q)
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    Dual x[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) x[k] = {val[k], k == q ? 1.0 : 0.0};
    Dual C[6];
    tti_stiffness(x[0], x[1], x[2], x[3], x[4], x[5], C);
    double s = 0;
#pragma unroll
    for (int k = 0; k < 6; ++k) s += gk[k] * C[k].d;
    if (q == 2) s += g[c];  // rho also enters the buoyancy directly
    out[slot[q] * np + c] = s;
  }
  out[3 * np + c] = g[7 * np + c] * tau_scale;  // dJ/d(1/Q)
}

__global__ void k_fold_iso(long long np, double *g) {
  const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= np) return;
  // C11 = C33 = lambda + 2 mu, C13 = lambda, C55 = mu
  const double g11 = g[1 * np + c], g13 = g[2 * np + c], g33 = g[4 * np + c], g55 = g[6 * np + c];
  g[2 * np + c] = g11 + g13 + g33;
  g[6 * np + c] = 2 * (g11 + g33) + g55;
  g[1 * np + c] = 0;
  g[4 * np + c] = 0;
}

}  // namespace

template <typename T>
static int gradient_impl(vi_plan *p, const vi_medium *m, const vi_shot *shot, int nt, const T *obs,
                         int K, int accumulate, double *grad, double *misfit, cudaStream_t st) {
  const vi_config &c = p->cfg;
  const bool tti = c.medium == VI_MEDIUM_TTI;
  if (c.free_surface == kFsAfda)
    return set_error(VI_ERR_ARG, "gradient: the adjoint covers the stress-imaging free surface, not H-AFDA");
  int rc = check_medium(p, m);
  if (rc) return rc;
  if (!shot || shot->nrec <= 0 || !obs) return set_error(VI_ERR_ARG, "gradient: needs receivers and observed traces");
  if (!grad) return set_error(VI_ERR_ARG, "gradient: grad buffer is NULL");
  if (nt <= 0) return set_error(VI_ERR_ARG, "gradient: nt must be positive");
  if ((rc = cuda_check(cudaSetDevice(p->device), "cudaSetDevice"))) return rc;
  const long long np = (long long)c.nx * c.nz;
  const int N = c.nsls;
  const long long slot = Slot<T>::size(np, p->psix_plane, p->psiz_plane, N);
  const int nrec = shot->nrec;
  const long long ntr = 2LL * nrec * nt;
  const long long scratch = 4 * np + np + 2 * np + 6 * np + (tti ? 5 * np : 0);
  // K = 0: every state of the forward sweep kept in HBM when the sweep fits
  // in 60 % of the device's memory and in what is free (1024 x 512 x 3000
  // VTI FP32: 88 GB), so the adjoint reads each step's states and nothing
  // is recomputed; else checkpoints every ceil(sqrt(nt)) steps
  bool keep_all = false;
  if (K <= 0) {
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) == cudaSuccess) {
      const size_t all = sizeof(T) * ((size_t)(nt + 2) * slot + scratch + ntr) + 64;
      const size_t avail = fr + p->fwd_bytes;
      keep_all = all <= (size_t)(0.6 * (double)tot) && all + (2ull << 30) <= avail;
    }
    cudaGetLastError();
    K = (int)std::ceil(std::sqrt((double)nt));
  }
  if (K > nt) K = nt;
  const int nck = keep_all ? nt + 1 : (nt + K - 1) / K;
  // workspace: checkpoints (keep_all: every state) | segment (K + 1 slots; none when keep_all) |
  // adjoint slot | scratch (4 rbar/dbar, q, 2 h, 6 plain (TTI: also the forward effective rates of
  // the adjoint sweep), TTI: 3 effective-rate adjoints, q15, q35) | traces
  const size_t need = sizeof(T) * ((size_t)(nck + (keep_all ? 0 : K + 1) + 1) * slot + scratch + ntr) + 64;
  size_t have = p->fwd_bytes;
  if ((rc = ensure_buffer(p, &p->fwd, &have, need))) return rc;
  p->fwd_bytes = have;
  T *ck = (T *)p->fwd;
  T *seg = keep_all ? ck : ck + (size_t)nck * slot;
  T *adj = keep_all ? ck + (size_t)nck * slot : seg + (size_t)(K + 1) * slot;
  T *rbar = adj + slot;   // also dbar
  T *q = rbar + 4 * np;
  T *h = q + np;
  T *pscr = h + 2 * np;   // plain-path scratch (6 planes)
  T *teb = pscr + 6 * np;  // TTI: effective-rate adjoints (3 planes), q15, q35
  T *tq15 = teb + 3 * np, *tq35 = tq15 + np;
  T *tr = pscr + 6 * np + (tti ? 5 * np : 0);
  auto mk = [&](T *b) { return Slot<T>{b, np, p->psix_plane, p->psiz_plane, N}; };
  if ((rc = stage_shot<T>(p, shot, st))) return rc;
  // plain forward step on a slot, in place (bind() points it at the slot)
  vi_fields fdummy{};
  fdummy.vx = fdummy.vz = fdummy.sxx = fdummy.szz = fdummy.sxz = (void *)ck;
  fdummy.m = ck;
  fdummy.m_plane_stride = np;
  StepArgs<T> a = make_args<T>(p, m, &fdummy);
  PlainExtras<T> x;
  x.scratch = pscr;
  x.fs = c.free_surface;
  x.src = (const int4 *)p->dsrc;
  x.amp = (const T *)p->damp;
  x.nsrc = shot->nsrc;
  x.wavelet = shot->nsrc ? (const T *)shot->wavelet_dev : nullptr;
  x.wnt = shot->nsrc ? shot->wavelet_nt : 0;
  x.rec = (const int2 *)p->drec;
  x.nrec = nrec;
  x.traces = nullptr;
  x.tnt = nt;
  auto bind = [&](StepArgs<T> &s, const Slot<T> &sl) {
    s.vx = sl.vx(); s.vz = sl.vz(); s.sxx = sl.sxx(); s.szz = sl.szz(); s.sxz = sl.sxz();
    s.m = sl.m(); s.mstride = np;
    s.psix = s.psix_o = p->wx ? sl.psix() : nullptr;
    s.psiz = s.psiz_o = p->hz ? sl.psiz() : nullptr;
  };
  const size_t sbytes = (size_t)slot * sizeof(T);
  // plain-path scratch: cells outside the update region are read, never written
  if ((rc = cuda_check(cudaMemsetAsync(pscr, 0, 6 * np * sizeof(T), st), "zero scratch"))) return rc;
  // The two forward sweeps (traces + checkpoints, then the segment
  // recompute) run on the split pair when the grid allows it (the same
  // discrete step as the plain path the adjoint transposes, faster), else
  // on the plain path.
  using SG = SplitGeom<T>;
  StepArgs<T> probe = a;
  bind(probe, mk(seg));
  // TTI sweeps step out of place only (the TTI stress pass reads M and psi
  // on a ring of neighbouring cells, so it writes them to the other slot);
  // the 4-cell transposed derivatives only need aligned planes
  const bool split_ok = split_eligible<T>(p, probe);
  const bool use_split = split_ok;
  using STG = SplitTtiGeom<T>;
  using SS = SplitStressGeom<T>;
  FusedExtras<T> fx{}, fxs{};
  SplitMaps ms{};
  int ntiles = 0, sntiles = 0;
  if (use_split) {
    // velocity tiling and stress tiling, one buffer of lists
    int ntx = 0, ntz = 0, sntx = 0, sntz = 0;
    std::vector<int> off, soff;
    std::vector<int4> ent, sent;
    build_tile_lists(c.nx, c.nz, SG::TX, SG::TZ, 0, shot, off, ent, ntx, ntz);
    build_tile_lists(c.nx, c.nz, tti ? STG::TX : SS::TX, tti ? STG::TZ : SS::TZ, 0, shot, soff, sent, sntx, sntz);
    const int nvoff = (int)off.size();
    for (int v : soff) off.push_back(v + (int)ent.size());
    ent.insert(ent.end(), sent.begin(), sent.end());
    int *d_off = nullptr;
    int4 *d_ent = nullptr;
    if ((rc = stage_tile_lists(p, off, ent, st, &d_off, &d_ent))) return rc;
    ntiles = ntx * ntz;
    sntiles = sntx * sntz;
    fxs.ntx = sntx;
    fxs.tile_off = d_off + nvoff;
    fx.ntx = ntx;
    fx.fs = c.free_surface;
    fx.tile_off = d_off;
    fx.tile_ent = d_ent;
    fx.amp = (const T *)p->damp;
    fx.wavelet = shot->nsrc ? (const T *)shot->wavelet_dev : nullptr;
    fx.wnt = shot->nsrc ? shot->wavelet_nt : 0;
    fx.nrec = nrec;
    fx.tnt = nt;
    fx.err = (int *)p->errflag;
    fx.l2hint = l2_hints_fit(5LL * c.nx * c.nz * (long long)sizeof(T), p->l2_bytes);
    const int sntx_keep = fxs.ntx;
    const int *soff_keep = fxs.tile_off;
    fxs = fx;
    fxs.ntx = sntx_keep;
    fxs.tile_off = soff_keep;
  }
  // One forward step of slot sl, in place, or (split pair, out != nullptr)
  // from slot sl into slot *out, which then holds the next state.
  auto fwd_step = [&](const Slot<T> &sl, int it, T *traces, bool pdl, const Slot<T> *out = nullptr) -> int {
    if (!use_split) {
      bind(a, sl);
      x.traces = traces;
      plain_step<T>(a, x, c.medium, it, st);
      return VI_OK;
    }
    StepArgs<T> b = a;
    if (tti) {
      // v and sigma copied into the output slot and stepped there in place;
      // M and psi from the input slot to the output one
      if (!out) return set_error(VI_ERR_ARG, "gradient: the TTI split step runs out of place");
      int r2 = cuda_check(cudaMemcpyAsync(out->vx(), sl.vx(), 5 * (size_t)np * sizeof(T), cudaMemcpyDeviceToDevice, st),
                          "state copy");
      bind(b, *out);
      b.m = sl.m();
      b.mstride = np;
      b.m_o = out->m();
      b.mstride_o = np;
      b.psix = p->wx ? sl.psix() : nullptr;
      b.psiz = p->hz ? sl.psiz() : nullptr;
      b.psix_o = p->wx ? out->psix() : nullptr;
      b.psiz_o = p->hz ? out->psiz() : nullptr;
      fx.it = fxs.it = it;
      fx.traces = fxs.traces = traces;
      if (!r2) r2 = encode_map(&ms.a, out->vx(), (int)sizeof(T), c.nx, c.nz, 1, 0, STG::BW, STG::BH, 1);
      if (!r2) r2 = encode_map(&ms.b, out->vz(), (int)sizeof(T), c.nx, c.nz, 1, 0, STG::BW, STG::BH, 1);
      if (!r2) r2 = launch_split_vel<T>(b, fx, ntiles, st, false);
      if (!r2) r2 = launch_split_stress_tti<T>(b, fxs, ms, sntiles, st, true);
      return r2;
    }
    bind(b, sl);
    if (out) {
      b.vx_o = out->vx(); b.vz_o = out->vz();
      b.sxx_o = out->sxx(); b.szz_o = out->szz(); b.sxz_o = out->sxz();
      b.m_o = out->m(); b.mstride_o = np;
      b.psix_o = p->wx ? out->psix() : nullptr;
      b.psiz_o = p->hz ? out->psiz() : nullptr;
    }
    fx.it = fxs.it = it;
    fx.traces = fxs.traces = traces;
    // the stress pass stages the new velocities: those of the output state
    T *nvx = out ? out->vx() : b.vx, *nvz = out ? out->vz() : b.vz;
    int r2 = encode_map(&ms.a, nvx, (int)sizeof(T), c.nx, c.nz, 1, 0, SS::BW, SS::BH, 1);
    if (!r2) r2 = encode_map(&ms.b, nvz, (int)sizeof(T), c.nx, c.nz, 1, 0, SS::BW, SS::BH, 1);
    if (!r2) r2 = launch_split_vel<T>(b, fx, ntiles, st, pdl);
    if (!r2) r2 = launch_split_stress<T>(c.medium, b, fxs, ms, sntiles, st, true);
    return r2;
  };
  // the caller's hook after every enqueued step (a server's slicing)
  auto yield = [&](int units) -> int {
    if (p->yield_fn && p->yield_fn(p->yield_ctx, units)) return set_error(VI_ERR_STATE, "gradient: stopped");
    return VI_OK;
  };
  // ---- forward sweep with checkpoints and traces ----
  Slot<T> cur = mk(seg);
  // every state slot starts at zero: cells the kernels never write (outside
  // the update region, off the CPML strips) stay zero in all of them.  The
  // kept states are zeroed once per layout of the plan's buffer (the key
  // is cleared by any other user of the buffer), so slot 0, never written,
  // stays the state at rest
  const unsigned long long zkey = keep_all ? ((unsigned long long)nt << 32) ^ (unsigned long long)slot ^
                                                 ((unsigned long long)sizeof(T) << 60) ^ (uintptr_t)p->fwd
                                           : 0;
  if (keep_all && p->grad_zero_key != zkey) {
    if ((rc = cuda_check(cudaMemsetAsync(ck, 0, (size_t)nck * sbytes, st), "zero kept states"))) return rc;
    p->grad_zero_key = zkey;
  } else if (!keep_all) {
    p->grad_zero_key = 0;
    if ((rc = cuda_check(cudaMemsetAsync(seg, 0, (size_t)(K + 1) * sbytes, st), "zero segment"))) return rc;
  }
  if (keep_all) {
    NvtxRange nr("vi_gradient: forward sweep, every state kept");
    for (int it = 0; it < nt; ++it) {
      T *nxt = ck + (size_t)(it + 1) * slot;
      if (use_split) {
        const Slot<T> out = mk(nxt);
        if ((rc = fwd_step(mk(ck + (size_t)it * slot), it, tr, it > 0, &out))) return rc;
      } else {
        if ((rc = cuda_check(cudaMemcpyAsync(nxt, ck + (size_t)it * slot, sbytes, cudaMemcpyDeviceToDevice, st),
                             "state copy")))
          return rc;
        if ((rc = fwd_step(mk(nxt), it, tr, false))) return rc;
      }
      if ((rc = yield(1))) return rc;
    }
  } else {
    NvtxRange nr("vi_gradient: forward sweep");
    for (int it = 0; it < nt; ++it) {
      if (it % K == 0)
        if ((rc = cuda_check(cudaMemcpyAsync(ck + (size_t)(it / K) * slot, cur.base, sbytes,
                                             cudaMemcpyDeviceToDevice, st),
                             "checkpoint")))
          return rc;
      if (tti && use_split) {  // out of place: between the segment's first two slots
        const Slot<T> nxt = mk(cur.base == seg ? seg + slot : seg);
        if ((rc = fwd_step(cur, it, tr, false, &nxt))) return rc;
        cur = nxt;
      } else if ((rc = fwd_step(cur, it, tr, it % K != 0))) {
        return rc;
      }
      if ((rc = yield(1))) return rc;
    }
  }
  if (shot->traces_dev && shot->traces_nt >= nt) {
    for (int k = 0; k < 2 * nrec; ++k)
      cudaMemcpyAsync((T *)shot->traces_dev + (size_t)k * shot->traces_nt, tr + (size_t)k * nt,
                      nt * sizeof(T), cudaMemcpyDeviceToDevice, st);
  }
  double *dmis = (double *)(tr + ntr);
  dmis = (double *)(((uintptr_t)dmis + 15) / 16 * 16);
  k_misfit<T><<<1, 256, 0, st>>>(tr, obs, ntr, dmis);
  // ---- adjoint sweep ----
  AdjArgs<T> A;
  A.nx = c.nx; A.nz = c.nz; A.nsls = N; A.kind = c.medium; A.fs = c.free_surface;
  A.Lx = p->Lx; A.Rx = p->Rx; A.Tz = p->Tz; A.Bz = p->Bz; A.wx = p->wx; A.hz = p->hz;
  A.dt = (T)c.dt;
  for (int k = 0; k < 4; ++k) {
    A.Dx[k] = (T)(kD8[k] / c.dx);
    A.Dz[k] = (T)(kD8[k] / c.dz);
  }
  for (int n = 0; n < N; ++n) {  // the forward step's memory-variable coefficients
    A.a1[n] = a.a1[n];
    A.a2[n] = a.a2[n];
  }
  A.rho = (const T *)m->rho; A.c11 = (const T *)m->c11; A.c13 = (const T *)m->c13;
  A.c33 = (const T *)m->c33; A.c55 = (const T *)m->c55; A.tau = (const T *)m->tau;
  A.c15 = (const T *)m->c15; A.c35 = (const T *)m->c35;
  A.tx = (const T *)p->tabx; A.tz = (const T *)p->tabz;
  A.np = np; A.psix_plane = p->psix_plane; A.psiz_plane = p->psiz_plane;
  Slot<T> ab = mk(adj);
  if ((rc = cuda_check(cudaMemsetAsync(adj, 0, sbytes, st), "zero adjoint"))) return rc;
  if ((rc = cuda_check(cudaMemsetAsync(rbar, 0, 7 * np * sizeof(T), st), "zero scratch"))) return rc;
  if (tti && (rc = cuda_check(cudaMemsetAsync(teb, 0, 5 * np * sizeof(T), st), "zero TTI scratch"))) return rc;
  if (!accumulate)
    if ((rc = cuda_check(cudaMemsetAsync(grad, 0, 8 * np * sizeof(double), st), "zero gradient"))) return rc;
  double *gr = grad, *g11 = grad + np, *g13 = grad + 2 * np, *g33 = grad + 4 * np;
  double *g55 = grad + 6 * np, *gt = grad + 7 * np, *g15 = grad + 3 * np, *g35 = grad + 5 * np;
  const dim3 blk(32, 8);
  const dim3 gU((c.nx - 2 * L + 31) / 32, (c.nz - 2 * L + 7) / 8);
  const dim3 gA((c.nx + 31) / 32, (c.nz + 7) / 8);
  // 4-cell forms of the transposed derivatives where the planes allow
  // 128-bit access (the same condition as the split pair)
  const bool vec4 = split_ok;
  const dim3 gU4(((c.nx - 2 * L) / 4 + 31) / 32, (c.nz - 2 * L + 7) / 8);
  const dim3 gA4((c.nx / 4 + 31) / 32, (c.nz + 7) / 8);
  int lrc = VI_OK;  // first launch error of the adjoint sweep
  auto lc = [&](auto kernel, dim3 g, dim3 b, auto... args) {
    const cudaError_t e = launch_pdl(kernel, g, b, 0, st, true, args...);
    if (e != cudaSuccess && !lrc) lrc = cuda_check(e, "adjoint launch");
  };
  // keep_all: one segment of nt steps whose states are all kept
  for (int qseg = keep_all ? 0 : nck - 1; qseg >= 0; --qseg) {
    const int s0 = keep_all ? 0 : qseg * K, s1 = keep_all ? nt : std::min(nt, s0 + K);
    // recompute the segment: seg[k] = state before step s0 + k
    if (!keep_all &&
        (rc = cuda_check(cudaMemcpyAsync(seg, ck + (size_t)qseg * slot, sbytes, cudaMemcpyDeviceToDevice, st),
                         "restore checkpoint")))
      return rc;
    NvtxRange nr_seg("vi_gradient: segment recompute and adjoint");
    for (int k = 0; !keep_all && k < s1 - s0; ++k) {
      T *nxt = seg + (size_t)(k + 1) * slot;
      if (use_split) {
        // straight from slot k into slot k + 1 (no copy of the state)
        const Slot<T> out = mk(nxt);
        if ((rc = fwd_step(mk(seg + (size_t)k * slot), s0 + k, nullptr, k > 0, &out))) return rc;
      } else {
        if ((rc = cuda_check(cudaMemcpyAsync(nxt, seg + (size_t)k * slot, sbytes, cudaMemcpyDeviceToDevice, st),
                             "segment copy")))
          return rc;
        if ((rc = fwd_step(mk(nxt), s0 + k, nullptr, false))) return rc;
      }
      if ((rc = yield(1))) return rc;
    }
    for (int it = s1 - 1; it >= s0; --it) {
      const Slot<T> x0 = mk(seg + (size_t)(it - s0) * slot), x1 = mk(seg + (size_t)(it - s0 + 1) * slot);
      // every kernel of the step overlaps its predecessor's tail and waits
      // for it at entry (programmatic dependent launch)
      if (c.free_surface) lc(k_mirror_t<T>, dim3((c.nx + 127) / 128), dim3(128), ab.szz(), ab.sxz(), c.nx);
      if (tti) {
        const dim3 gS((c.nx - 2 * L + 127) / 128);
        switch (N) {
          case 0: lc(k_tti_fwd_rates<T, 0>, gU, blk, A, x0, x1, pscr); break;
          case 1: lc(k_tti_fwd_rates<T, 1>, gU, blk, A, x0, x1, pscr); break;
          case 2: lc(k_tti_fwd_rates<T, 2>, gU, blk, A, x0, x1, pscr); break;
          case 3: lc(k_tti_fwd_rates<T, 3>, gU, blk, A, x0, x1, pscr); break;
          case 4: lc(k_tti_fwd_rates<T, 4>, gU, blk, A, x0, x1, pscr); break;
          default: lc(k_tti_fwd_rates<T, 5>, gU, blk, A, x0, x1, pscr); break;
        }
        if (c.free_surface) lc(k_tti_fwd_surface<T>, gS, dim3(128), A, pscr);
        lc(k_tti_ebar_t<T>, gU, blk, A, ab, (const T *)pscr, teb, q, tq15, tq35, g11, g13, g15, g33, g35);
        if (c.free_surface) lc(k_tti_surface_t<T>, gS, dim3(128), A, (const T *)pscr, teb, g13, g33, g35);
        switch (N) {
          case 0: lc(k_tti_stress_t<T, 0>, gU, blk, A, ab, (const T *)pscr, (const T *)teb, rbar, gt); break;
          case 1: lc(k_tti_stress_t<T, 1>, gU, blk, A, ab, (const T *)pscr, (const T *)teb, rbar, gt); break;
          case 2: lc(k_tti_stress_t<T, 2>, gU, blk, A, ab, (const T *)pscr, (const T *)teb, rbar, gt); break;
          case 3: lc(k_tti_stress_t<T, 3>, gU, blk, A, ab, (const T *)pscr, (const T *)teb, rbar, gt); break;
          case 4: lc(k_tti_stress_t<T, 4>, gU, blk, A, ab, (const T *)pscr, (const T *)teb, rbar, gt); break;
          default: lc(k_tti_stress_t<T, 5>, gU, blk, A, ab, (const T *)pscr, (const T *)teb, rbar, gt); break;
        }
      } else switch (N) {
        case 0: lc(k_stress_t<T, 0>, gU, blk, A, x0, x1, ab, rbar, q, g11, g13, g33, gt); break;
        case 1: lc(k_stress_t<T, 1>, gU, blk, A, x0, x1, ab, rbar, q, g11, g13, g33, gt); break;
        case 2: lc(k_stress_t<T, 2>, gU, blk, A, x0, x1, ab, rbar, q, g11, g13, g33, gt); break;
        case 3: lc(k_stress_t<T, 3>, gU, blk, A, x0, x1, ab, rbar, q, g11, g13, g33, gt); break;
        case 4: lc(k_stress_t<T, 4>, gU, blk, A, x0, x1, ab, rbar, q, g11, g13, g33, gt); break;
        default: lc(k_stress_t<T, 5>, gU, blk, A, x0, x1, ab, rbar, q, g11, g13, g33, gt); break;
      }
      if (vec4)
        lc(k_rates_t4<T>, gU4, blk, A, ab, (const T *)rbar);
      else
        lc(k_rates_t<T>, gU, blk, A, ab, (const T *)rbar);
      lc(k_residual<T>, dim3((nrec + 127) / 128), dim3(128), ab, x1, (const int2 *)p->drec, nrec, obs, nt, it, c.nx);
      lc(k_vel_t<T>, gU, blk, A, x0, ab, rbar, h);  // the 4-cell form measured slower
      if (shot->nsrc > 0)
        lc(k_force_rho_t<T>, dim3((shot->nsrc + 127) / 128), dim3(128), A, ab, (const int4 *)p->dsrc,
           (const T *)p->damp, shot->nsrc, (const T *)shot->wavelet_dev, shot->wavelet_nt, it, h);
      lc(k_gather<T>, gA, blk, (const T *)h, gr, (const T *)q, g55, c.nx, c.nz);
      if (tti) lc(k_tti_gather<T>, gA, blk, (const T *)tq15, (const T *)tq35, g15, g35, c.nx, c.nz);
      if (vec4)
        lc(k_div_t4<T>, gA4, blk, A, ab, (const T *)rbar);
      else
        lc(k_div_t<T>, gA, blk, A, ab, (const T *)rbar);
      if (lrc) return lrc;
      if ((rc = yield(2))) return rc;
    }
  }
  if (lrc) return lrc;
  if (c.medium == VI_MEDIUM_ISO) k_fold_iso<<<(unsigned)((np + 255) / 256), 256, 0, st>>>(np, grad);
  p->last_kernel = 1;
  if ((rc = cuda_check(cudaGetLastError(), "gradient launch"))) return rc;
  if ((rc = cuda_check(cudaMemcpyAsync(misfit, dmis, sizeof(double), cudaMemcpyDeviceToHost, st), "misfit")))
    return rc;
  return cuda_check(cudaStreamSynchronize(st), "gradient");
}

}  // namespace vb

using namespace vb;

extern "C" int vi_gradient(vi_plan *p, const vi_medium *med_dev, const vi_shot *shot, int32_t nt,
                           const void *obs_dev, int32_t checkpoint_every, int32_t accumulate,
                           double *grad_dev, double *misfit_host, void *stream) {
  if (!p || !misfit_host) return set_error(VI_ERR_ARG, "gradient: NULL argument");
  cudaStream_t st = (cudaStream_t)stream;
  return p->cfg.precision == VI_F64
             ? gradient_impl<double>(p, med_dev, shot, nt, (const double *)obs_dev, checkpoint_every,
                                     accumulate, grad_dev, misfit_host, st)
             : gradient_impl<float>(p, med_dev, shot, nt, (const float *)obs_dev, checkpoint_every,
                                    accumulate, grad_dev, misfit_host, st);
}

extern "C" int vi_gradient_velocity(int32_t medium, int64_t np, const double *grad8, const double *vp,
                                    const double *vs, const double *rho, const double *eps,
                                    const double *delta, double tau_scale, double *out4, void *stream) {
  if (!grad8 || !vp || !vs || !rho || !out4 || np <= 0)
    return set_error(VI_ERR_ARG, "gradient_velocity: NULL argument");
  if (medium != VI_MEDIUM_ISO && medium != VI_MEDIUM_VTI)
    return set_error(VI_ERR_ARG, "gradient_velocity: ISO or VTI only");
  k_velocity_grad<<<(unsigned)((np + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
      medium, np, grad8, vp, vs, rho, eps, delta, tau_scale, out4);
  return cuda_check(cudaGetLastError(), "gradient_velocity launch");
}

extern "C" int vi_gradient_tti(int64_t np, const double *grad8, const double *vp, const double *vs,
                               const double *rho, const double *eps, const double *delta, const double *theta,
                               double tau_scale, double *out7, void *stream) {
  if (!grad8 || !vp || !vs || !rho || !out7 || np <= 0)
    return set_error(VI_ERR_ARG, "gradient_tti: NULL argument");
  k_tti_param_grad<<<(unsigned)((np + 255) / 256), 256, 0, (cudaStream_t)stream>>>(np, grad8, vp, vs, rho, eps,
                                                                                   delta, theta, tau_scale, out7);
  return cuda_check(cudaGetLastError(), "gradient_tti launch");
}

extern "C" int vi_gradient_thomsen(int64_t np, const double *grad8, const double *vp, const double *vs,
                                   const double *rho, const double *delta, double *out2, void *stream) {
  if (!grad8 || !vp || !vs || !rho || !out2 || np <= 0)
    return set_error(VI_ERR_ARG, "gradient_thomsen: NULL argument");
  k_thomsen_grad<<<(unsigned)((np + 255) / 256), 256, 0, (cudaStream_t)stream>>>(np, grad8, vp, vs, rho,
                                                                                 delta, out2);
  return cuda_check(cudaGetLastError(), "gradient_thomsen launch");
}
