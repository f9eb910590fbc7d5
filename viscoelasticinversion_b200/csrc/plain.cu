// plain.cu — the plain multi-kernel step: one thread per cell, one kernel
// per physical stage, global-memory operands.  It is the straightforward
// CUDA form of the step (the shape of the reference's per-stage
// KernelAbstractions launches, visco-kernels.jl:87-100) and serves as the
// in-place path of vi_step(kernel_variant = 1).  The strain pass writes six
// scratch planes (raw CPML-corrected rates and effective SLS rates) that
// the update pass reads back; the fused path never materialises them.
#include "plain.cuh"

namespace vb {

// fs: free-surface kind; under the H-AFDA surface the z derivatives of the
// four rows below it take the one-sided weights a.af
template <typename T>
__global__ void __launch_bounds__(256) k_vel_plain(const __grid_constant__ StepArgs<T> a, int fs) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + L;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + L;
  if (i >= a.nx - L || j >= a.nz - L) return;
  const int nx = a.nx;
  const long long c = (long long)j * nx + i;
  T dxx = 0, dzxz = 0, dxxz = 0, dzz = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int l = k + 1;
    dxx += a.Dx[k] * (a.sxx[c + l] - a.sxx[c - l + 1]);
    dzxz += a.Dz[k] * (a.sxz[c + (long long)(l - 1) * nx] - a.sxz[c - (long long)l * nx]);
    dxxz += a.Dx[k] * (a.sxz[c + l - 1] - a.sxz[c - l]);
    dzz += a.Dz[k] * (a.szz[c + (long long)l * nx] - a.szz[c - (long long)(l - 1) * nx]);
  }
  if (fs == kFsAfda && j < L + 4) {
    const int q = j - L;
    dzxz = 0;
#pragma unroll
    for (int m = 0; m < kAfdaN; ++m) dzxz += a.af[0][q][m] * a.sxz[(long long)(L + m) * nx + i];
    if (q < 3) {
      dzz = 0;
#pragma unroll
      for (int m = 0; m < kAfdaN; ++m) dzz += a.af[1][q][m] * a.szz[(long long)(L + 1 + m) * nx + i];
    }
  }
  const int xs = strip_x(i, nx, a.Lx, a.Rx);
  if (xs >= 0) {
    const T *t = a.tx;
    T *p0 = a.psix_o + PX_SXX * a.psix_plane + (long long)j * a.wx + xs;
    T *p1 = a.psix_o + PX_SXZ * a.psix_plane + (long long)j * a.wx + xs;
    *p0 = t[T_BH * nx + i] * *p0 + t[T_AH * nx + i] * dxx;
    dxx = dxx * t[T_IKH * nx + i] + *p0;
    *p1 = t[T_B * nx + i] * *p1 + t[T_A * nx + i] * dxxz;
    dxxz = dxxz * t[T_IK * nx + i] + *p1;
  }
  const int zs = strip_z(j, a.nz, a.Tz, a.Bz);
  if (zs >= 0) {
    const int nz = a.nz;
    const T *t = a.tz;
    T *p0 = a.psiz_o + PZ_SXZ * a.psiz_plane + (long long)zs * nx + i;
    T *p1 = a.psiz_o + PZ_SZZ * a.psiz_plane + (long long)zs * nx + i;
    *p0 = t[T_B * nz + j] * *p0 + t[T_A * nz + j] * dzxz;
    dzxz = dzxz * t[T_IK * nz + j] + *p0;
    *p1 = t[T_BH * nz + j] * *p1 + t[T_AH * nz + j] * dzz;
    dzz = dzz * t[T_IKH * nz + j] + *p1;
  }
  const T bx = T(2) / (a.rho[c] + a.rho[c + 1]);
  const T bz = T(2) / (a.rho[c] + a.rho[c + nx]);
  a.vx[c] += a.dt * bx * (dxx + dzxz);
  a.vz[c] += a.dt * bz * (dxxz + dzz);
}

// Pass 1 of the stress stage: CPML-corrected rates r and effective SLS rates
// e into scratch (6 planes of nx*nz: rxx, rzz, rxz, exx, ezz, exz).
template <typename T, int NSLS>
__global__ void __launch_bounds__(256) k_strain_plain(const __grid_constant__ StepArgs<T> a, T *scratch, int fs) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + L;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + L;
  if (i >= a.nx - L || j >= a.nz - L) return;
  const int nx = a.nx;
  const long long np = (long long)nx * a.nz;
  const long long c = (long long)j * nx + i;
  T dxvx = 0, dzvz = 0, dzvx = 0, dxvz = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int l = k + 1;
    dxvx += a.Dx[k] * (a.vx[c + l - 1] - a.vx[c - l]);
    dzvz += a.Dz[k] * (a.vz[c + (long long)(l - 1) * nx] - a.vz[c - (long long)l * nx]);
    dzvx += a.Dz[k] * (a.vx[c + (long long)l * nx] - a.vx[c - (long long)(l - 1) * nx]);
    dxvz += a.Dx[k] * (a.vz[c + l] - a.vz[c - l + 1]);
  }
  if (fs == kFsAfda && j < L + 4) {  // on the surface row the tau_zz = 0 relation sets e_zz
    const int q = j - L;
    if (q >= 1) {
      dzvz = 0;
#pragma unroll
      for (int m = 0; m < kAfdaN; ++m) dzvz += a.af[2][q][m] * a.vz[(long long)(L + m) * nx + i];
    }
    if (q < 3) {
      dzvx = 0;
#pragma unroll
      for (int m = 0; m < kAfdaN; ++m) dzvx += a.af[3][q][m] * a.vx[(long long)(L + m) * nx + i];
    }
  }
  const int xs = strip_x(i, nx, a.Lx, a.Rx);
  if (xs >= 0) {
    const T *t = a.tx;
    T *p0 = a.psix_o + PX_VX * a.psix_plane + (long long)j * a.wx + xs;
    T *p1 = a.psix_o + PX_VZ * a.psix_plane + (long long)j * a.wx + xs;
    *p0 = t[T_B * nx + i] * *p0 + t[T_A * nx + i] * dxvx;
    dxvx = dxvx * t[T_IK * nx + i] + *p0;
    *p1 = t[T_BH * nx + i] * *p1 + t[T_AH * nx + i] * dxvz;
    dxvz = dxvz * t[T_IKH * nx + i] + *p1;
  }
  const int zs = strip_z(j, a.nz, a.Tz, a.Bz);
  if (zs >= 0) {
    const int nz = a.nz;
    const T *t = a.tz;
    T *p0 = a.psiz_o + PZ_VZ * a.psiz_plane + (long long)zs * nx + i;
    T *p1 = a.psiz_o + PZ_VX * a.psiz_plane + (long long)zs * nx + i;
    *p0 = t[T_B * nz + j] * *p0 + t[T_A * nz + j] * dzvz;
    dzvz = dzvz * t[T_IK * nz + j] + *p0;
    *p1 = t[T_BH * nz + j] * *p1 + t[T_AH * nz + j] * dzvx;
    dzvx = dzvx * t[T_IKH * nz + j] + *p1;
  }
  const T g = dzvx + dxvz;
  scratch[c] = dxvx;
  scratch[np + c] = dzvz;
  scratch[2 * np + c] = g;
  if (NSLS > 0) {
    T Sxx = 0, Szz = 0, Sxz = 0;
#pragma unroll
    for (int n = 0; n < NSLS; ++n) {
      Sxx += a.m[(0 * NSLS + n) * a.mstride + c];
      Szz += a.m[(1 * NSLS + n) * a.mstride + c];
      Sxz += a.m[(2 * NSLS + n) * a.mstride + c];
    }
    const T t = a.tau[c];
    const T t1 = T(1) + t;
    scratch[3 * np + c] = t1 * dxvx + t * Sxx;
    scratch[4 * np + c] = t1 * dzvz + t * Szz;
    scratch[5 * np + c] = t1 * g + t * Sxz;
  } else {
    scratch[3 * np + c] = dxvx;
    scratch[4 * np + c] = dzvz;
    scratch[5 * np + c] = g;
  }
}

template <typename T, int KIND>
__device__ __forceinline__ T c11_at(const StepArgs<T> &a, long long c) {
  return KIND == VI_MEDIUM_ISO ? a.c13[c] + T(2) * a.c55[c] : a.c11[c];
}
template <typename T, int KIND>
__device__ __forceinline__ T c33_at(const StepArgs<T> &a, long long c) {
  return KIND == VI_MEDIUM_ISO ? a.c13[c] + T(2) * a.c55[c] : a.c33[c];
}

// Pass 2 (free surface only): ezz on the surface row from tau_zz = 0.
template <typename T, int KIND>
__global__ void k_surface_rate_plain(StepArgs<T> a, T *scratch) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + L;
  if (i >= a.nx - L) return;
  const int nx = a.nx;
  const long long np = (long long)nx * a.nz;
  const long long c = (long long)L * nx + i;
  const T *exx = scratch + 3 * np, *exz = scratch + 5 * np;
  T num = a.c13[c] * exx[c];
  if (KIND == VI_MEDIUM_TTI) {
    const T eb = T(0.25) * (exz[c] + exz[c - 1] + exz[c - nx] + exz[c - nx - 1]);
    num += a.c35[c] * eb;
  }
  scratch[4 * np + c] = -num / c33_at<T, KIND>(a, c);
}

// Pass 3: stress and memory-variable update.
template <typename T, int KIND, int NSLS>
__global__ void __launch_bounds__(256) k_update_plain(StepArgs<T> a, const T *scratch, int fs) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + L;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + L;
  if (i >= a.nx - L || j >= a.nz - L) return;
  const int nx = a.nx;
  const long long np = (long long)nx * a.nz;
  const long long c = (long long)j * nx + i;
  const T *rxx = scratch, *rzz = scratch + np, *rxz = scratch + 2 * np;
  const T *exx = scratch + 3 * np, *ezz = scratch + 4 * np, *exz = scratch + 5 * np;
  const T C11 = c11_at<T, KIND>(a, c), C13 = a.c13[c], C33 = c33_at<T, KIND>(a, c);
  const T C55h = T(0.25) * (a.c55[c] + a.c55[c + 1] + a.c55[c + nx] + a.c55[c + nx + 1]);
  T dsxx = C11 * exx[c] + C13 * ezz[c];
  T dszz = C13 * exx[c] + C33 * ezz[c];
  T dsxz = C55h * exz[c];
  if (KIND == VI_MEDIUM_TTI) {
    const T ebxz = T(0.25) * (exz[c] + exz[c - 1] + exz[c - nx] + exz[c - nx - 1]);
    const T ebxx = T(0.25) * (exx[c] + exx[c + 1] + exx[c + nx] + exx[c + nx + 1]);
    const T ebzz = T(0.25) * (ezz[c] + ezz[c + 1] + ezz[c + nx] + ezz[c + nx + 1]);
    const T C15h = T(0.25) * (a.c15[c] + a.c15[c + 1] + a.c15[c + nx] + a.c15[c + nx + 1]);
    const T C35h = T(0.25) * (a.c35[c] + a.c35[c + 1] + a.c35[c + nx] + a.c35[c + nx + 1]);
    dsxx += a.c15[c] * ebxz;
    dszz += a.c35[c] * ebxz;
    dsxz += C15h * ebxx + C35h * ebzz;
  }
  a.sxx[c] += a.dt * dsxx;
  a.szz[c] += a.dt * dszz;
  a.sxz[c] += a.dt * dsxz;
  const bool surf = fs && j == L;
#pragma unroll
  for (int n = 0; n < NSLS; ++n) {
    T *mxx = a.m + (0 * NSLS + n) * a.mstride + c;
    T *mzz = a.m + (1 * NSLS + n) * a.mstride + c;
    T *mxz = a.m + (2 * NSLS + n) * a.mstride + c;
    *mxx += a.dt * (a.a1[n] * rxx[c] + a.a2[n] * *mxx);
    *mzz = surf ? T(0) : *mzz + a.dt * (a.a1[n] * rzz[c] + a.a2[n] * *mzz);
    *mxz += a.dt * (a.a1[n] * rxz[c] + a.a2[n] * *mxz);
  }
}

// Sources.  stage 0: force sources (after the velocity update);
// stage 1: explosive sources (after the stress update).
template <typename T>
__global__ void k_sources(StepArgs<T> a, const int4 *src, const T *amp, int nsrc,
                          const T *wavelet, int wnt, int it, int stage) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nsrc) return;
  const int4 s = src[q];  // i, j, kind
  const bool explosive = s.z == VI_SRC_EXPLOSIVE;
  if (explosive != (stage == 1)) return;
  const long long c = (long long)s.y * a.nx + s.x;
  const T w = it < wnt ? wavelet[(long long)q * wnt + it] : T(0);
  const T f = amp[q] * w;
  if (s.z == VI_SRC_EXPLOSIVE) {
    a.sxx[c] += a.dt * f;
    a.szz[c] += a.dt * f;
  } else if (s.z == VI_SRC_FORCE_X) {
    a.vx[c] += a.dt * (T(2) / (a.rho[c] + a.rho[c + 1])) * f;
  } else {
    a.vz[c] += a.dt * (T(2) / (a.rho[c] + a.rho[c + a.nx])) * f;
  }
}

template <typename T>
__global__ void k_receivers(const T *vx, const T *vz, int nx, const int2 *rec, int nrec,
                            T *traces, int tnt, int it) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nrec || it >= tnt) return;
  const long long c = (long long)rec[r].y * nx + rec[r].x;
  traces[(long long)r * tnt + it] = vx[c];
  traces[(long long)(nrec + r) * tnt + it] = vz[c];
}

// Free surface: szz = 0 on row L, and (stress imaging) the images above it.
template <typename T>
__global__ void k_mirror(T *szz, T *sxz, int nx, int fs) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nx) return;
  szz[(long long)L * nx + i] = T(0);
  if (fs != kFsImaging) return;
#pragma unroll
  for (int k = 1; k <= L; ++k) szz[(long long)(L - k) * nx + i] = -szz[(long long)(L + k) * nx + i];
#pragma unroll
  for (int k = 0; k < L; ++k) sxz[(long long)(L - 1 - k) * nx + i] = -sxz[(long long)(L + k) * nx + i];
}

template <typename T, int KIND, int NSLS>
static void plain_step_impl(const StepArgs<T> &a, const PlainExtras<T> &x, int it,
                            cudaStream_t st) {
  const dim3 blk(32, 8);
  const dim3 grd((a.nx - 2 * L + 31) / 32, (a.nz - 2 * L + 7) / 8);
  k_vel_plain<T><<<grd, blk, 0, st>>>(a, x.fs);
  if (x.nsrc > 0)
    k_sources<T><<<(x.nsrc + 127) / 128, 128, 0, st>>>(a, x.src, x.amp, x.nsrc, x.wavelet,
                                                        x.wnt, it, 0);
  if (x.nrec > 0 && x.traces)
    k_receivers<T><<<(x.nrec + 127) / 128, 128, 0, st>>>(a.vx, a.vz, a.nx, x.rec, x.nrec,
                                                          x.traces, x.tnt, it);
  k_strain_plain<T, NSLS><<<grd, blk, 0, st>>>(a, x.scratch, x.fs);
  if (x.fs)
    k_surface_rate_plain<T, KIND><<<(a.nx + 127) / 128, 128, 0, st>>>(a, x.scratch);
  k_update_plain<T, KIND, NSLS><<<grd, blk, 0, st>>>(a, x.scratch, x.fs);
  if (x.nsrc > 0)
    k_sources<T><<<(x.nsrc + 127) / 128, 128, 0, st>>>(a, x.src, x.amp, x.nsrc, x.wavelet,
                                                        x.wnt, it, 1);
  if (x.fs) k_mirror<T><<<(a.nx + 127) / 128, 128, 0, st>>>(a.szz, a.sxz, a.nx, x.fs);
}

template <typename T>
void plain_step(const StepArgs<T> &a, const PlainExtras<T> &x, int kind, int it,
                cudaStream_t st) {
#define VB_CASE(K, N)                                  \
  if (kind == K && a.nsls == N) {                      \
    plain_step_impl<T, K, N>(a, x, it, st);            \
    return;                                            \
  }
#define VB_KIND(K) VB_CASE(K, 0) VB_CASE(K, 1) VB_CASE(K, 2) VB_CASE(K, 3) VB_CASE(K, 4) VB_CASE(K, 5)
  VB_KIND(VI_MEDIUM_ISO)
  VB_KIND(VI_MEDIUM_VTI)
  VB_KIND(VI_MEDIUM_TTI)
#undef VB_KIND
#undef VB_CASE
}

template void plain_step<float>(const StepArgs<float> &, const PlainExtras<float> &, int, int,
                                cudaStream_t);
template void plain_step<double>(const StepArgs<double> &, const PlainExtras<double> &, int,
                                 int, cudaStream_t);

// Staggered derivative of one plane over the update region (diff-funcs.jl:3-32).
template <typename T>
__global__ void k_diff(int op, const T *u, T *du, int nx, int nz, T D0, T D1, T D2, T D3) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + L;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + L;
  if (i >= nx - L || j >= nz - L) return;
  const long long c = (long long)j * nx + i;
  const T D[4] = {D0, D1, D2, D3};
  const long long s = op < 2 ? 1 : nx;  // stride along the operator axis
  const bool plus = (op == 0 || op == 2);
  T v = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int l = k + 1;
    v += plus ? D[k] * (u[c + l * s] - u[c - (l - 1) * s])
              : D[k] * (u[c + (l - 1) * s] - u[c - l * s]);
  }
  du[c] = v;
}

template <typename T>
void diff_launch(int op, const T *u, T *du, int nx, int nz, double h, cudaStream_t st) {
  const dim3 blk(32, 8);
  const dim3 grd((nx - 2 * L + 31) / 32, (nz - 2 * L + 7) / 8);
  k_diff<T><<<grd, blk, 0, st>>>(op, u, du, nx, nz, T(kD8[0] / h), T(kD8[1] / h),
                                 T(kD8[2] / h), T(kD8[3] / h));
}
template void diff_launch<float>(int, const float *, float *, int, int, double, cudaStream_t);
template void diff_launch<double>(int, const double *, double *, int, int, double,
                                  cudaStream_t);

}  // namespace vb
