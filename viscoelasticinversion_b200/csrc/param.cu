// param.cu — medium planes from velocity-domain parameters, on the device.
//
// The reference builds its stiffness on the host: ISO Lame from (vp, vs,
// rho), VTI from Thomsen (epsilon, delta) (sciml_solver/Models.jl:27-52,
// custom_solver/Model.jl:12-16), tau = N / (Kbar Q) from the Q fit
// (Models.jl:67).  Here one elementwise pass writes the planes the step
// reads, in the plan's precision, straight from FP64 parameter planes on
// the device, so an inversion that updates (vp, vs, rho, 1/Q, epsilon,
// delta) never moves its medium through the host.  TTI tilts the VTI
// stiffness by theta (symmetry axis turned from z towards x) with the 2D
// Bond rotation of the Voigt matrix.  Arithmetic in FP64, one rounding at
// the store.
#include <cmath>
#include <cstdint>

#include "plan.cuh"

namespace vb {

namespace {

template <typename T>
__device__ __forceinline__ void put(const void *plane, long long c, double v) {
  // the caller's medium planes: written by this call only
  reinterpret_cast<T *>(const_cast<void *>(plane))[c] = static_cast<T>(v);
}

template <typename T>
__global__ void k_medium_from_velocity(int kind, long long np, const double *vp, const double *vs,
                                       const double *rho, const double *eps, const double *delta,
                                       const double *theta, const double *q, double tau_scale,
                                       vi_medium out) {
  const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= np) return;
  const double r = rho[c], p = vp[c], s = vs[c];
  const double C33 = r * p * p, C55 = r * s * s;
  put<T>(out.rho, c, r);
  if (q && out.tau) put<T>(out.tau, c, tau_scale / q[c]);
  if (kind == VI_MEDIUM_ISO) {
    put<T>(out.c13, c, C33 - 2.0 * C55);  // lambda
    put<T>(out.c55, c, C55);              // mu
    return;
  }
  const double e = eps ? eps[c] : 0.0, d = delta ? delta[c] : 0.0;
  const double C11 = C33 * (1.0 + 2.0 * e);
  const double C13 = sqrt(fmax((C33 - C55) * (C33 * (1.0 + 2.0 * d) - C55), 0.0)) - C55;
  if (kind == VI_MEDIUM_VTI) {
    put<T>(out.c11, c, C11);
    put<T>(out.c13, c, C13);
    put<T>(out.c33, c, C33);
    put<T>(out.c55, c, C55);
    return;
  }
  // TTI: C' = R C R^T in Voigt form for the rotation by theta in the x-z plane
  const double th = theta ? theta[c] : 0.0;
  const double co = cos(th), si = sin(th);
  const double c2 = co * co, s2 = si * si, cs = co * si;
  const double A = C13 + 2.0 * C55;
  put<T>(out.c11, c, c2 * c2 * C11 + 2.0 * c2 * s2 * A + s2 * s2 * C33);
  put<T>(out.c33, c, s2 * s2 * C11 + 2.0 * c2 * s2 * A + c2 * c2 * C33);
  put<T>(out.c13, c, c2 * s2 * (C11 + C33 - 4.0 * C55) + (c2 * c2 + s2 * s2) * C13);
  put<T>(out.c55, c, c2 * s2 * (C11 + C33 - 2.0 * C13) + (c2 - s2) * (c2 - s2) * C55);
  put<T>(out.c15, c, -cs * (c2 * C11 - s2 * C33 - (c2 - s2) * A));
  put<T>(out.c35, c, -cs * (s2 * C11 - c2 * C33 + (c2 - s2) * A));
}

}  // namespace

}  // namespace vb

extern "C" int vi_medium_from_velocity(int32_t medium, int32_t precision, int64_t np,
                                       const double *vp, const double *vs, const double *rho,
                                       const double *eps, const double *delta, const double *theta,
                                       const double *q, double tau_scale, const vi_medium *out,
                                       void *stream) {
  using namespace vb;
  if (!vp || !vs || !rho || !out || np <= 0)
    return set_error(VI_ERR_ARG, "medium_from_velocity: NULL argument");
  if (precision != VI_F32 && precision != VI_F64)
    return set_error(VI_ERR_ARG, "medium_from_velocity: precision must be VI_F32 or VI_F64");
  if (medium != VI_MEDIUM_ISO && medium != VI_MEDIUM_VTI && medium != VI_MEDIUM_TTI)
    return set_error(VI_ERR_ARG, "medium_from_velocity: unknown medium kind");
  const vi_medium &o = *out;
  bool ok = o.rho && o.c13 && o.c55;
  if (medium != VI_MEDIUM_ISO) ok = ok && o.c11 && o.c33;
  if (medium == VI_MEDIUM_TTI) ok = ok && o.c15 && o.c35;
  if (q) ok = ok && o.tau;
  if (!ok) return set_error(VI_ERR_ARG, "medium_from_velocity: an output plane the medium needs is NULL");
  const unsigned grid = (unsigned)((np + 255) / 256);
  cudaStream_t st = (cudaStream_t)stream;
  if (precision == VI_F64)
    k_medium_from_velocity<double><<<grid, 256, 0, st>>>(medium, np, vp, vs, rho, eps, delta, theta, q,
                                                         tau_scale, o);
  else
    k_medium_from_velocity<float><<<grid, 256, 0, st>>>(medium, np, vp, vs, rho, eps, delta, theta, q,
                                                        tau_scale, o);
  return cuda_check(cudaGetLastError(), "medium_from_velocity launch");
}
