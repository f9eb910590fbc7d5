// common.cuh — device-side definitions shared by the step kernels.
//
// Physics of one step (both the plain and the fused kernels implement it):
//   velocity:  vx += dt*bx*(ddxp(sxx) + ddzm(sxz) [+ f]),  bx = 2/(rho_i + rho_i+1)
//              vz += dt*bz*(ddxm(sxz) + ddzp(szz) [+ f]),  bz = 2/(rho_j + rho_j+1)
//              (visco-kernels.jl:3-20 with the Virieux staggering fixed;
//               free-surface-kernels.jl:24 uses the same ddxp(sxx))
//   strain:    exx = ddxm(vx), ezz = ddzm(vz), gxz = ddzp(vx) + ddxp(vz)
//              (engineering shear; visco-kernels.jl:65-67 halves it and calls
//               an undefined _ddz — the custom/SciML paths use the full sum,
//               custom_solver/Model.jl:100, ViscoelasticProblem.jl:49)
//   SLS:       e = (1+tau)*rate + tau*sum_n M_n   per Voigt component
//              sigma += dt * C : e                (visco-kernels.jl:22-46)
//              M_n += dt*(-rate/(N tau_n) - M_n/tau_n)   (visco-kernels.jl:49-57)
//   CPML:      psi = b*psi + a*d;  d~ = d/kappa + psi  (CPML.jl:291-308,
//              Komatitsch–Martin recursion), strip storage only.
//   surface:   szz = 0 and Mzz = 0 on row 4; the vertical rate there follows
//              from tau_zz = 0 (free-surface-kernels.jl:84-95); stress images
//              szz(4-k) = -szz(4+k), sxz(3-k) = -sxz(4+k) (CPML.jl:372-380).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/visco_b200.h"

namespace vb {

constexpr int L = VI_HALF;

// Staggered 8th-order half-stencil at unit spacing (Stencil.jl:_stencil on
// the points -7/2..7/2): 1225/1024, -245/3072, 49/5120, -5/7168.
constexpr double kD8[4] = {1225.0 / 1024.0, -245.0 / 3072.0, 49.0 / 5120.0,
                           -5.0 / 7168.0};

// Arguments of one time step, passed by value to every step kernel.
template <typename T>
struct StepArgs {
  int nx, nz, nsls;
  int Lx, Rx, Tz, Bz;   // CPML strip widths (cells) per side
  int wx, hz;           // wx = Lx + Rx, hz = Tz + Bz
  T dt;
  T Dx[4], Dz[4];       // D_k / dx, D_k / dz
  T a1[VI_MAX_SLS], a2[VI_MAX_SLS];
  // medium
  const T *rho, *c11, *c13, *c15, *c33, *c35, *c55, *tau;
  // state: input side (the plain path updates it in place)
  T *vx, *vz, *sxx, *szz, *sxz;
  T *m;
  long long mstride;
  // state: output side of the ping-pong (fused) kernels
  T *vx_o, *vz_o, *sxx_o, *szz_o, *sxz_o;
  T *m_o;
  long long mstride_o;
  // CPML: x strips are planes of wx*nz (x fastest), z strips nx*hz.
  // psix/psiz point at the input set of 4 planes, psix_o/psiz_o at the
  // output set (equal for the in-place plain path).
  T *psix, *psiz, *psix_o, *psiz_o;
  long long psix_plane, psiz_plane;
  // coefficient tables: [ik, a, b, ikh, ah, bh] x n
  const T *tx, *tz;
  // compensated stress accumulation (FP32 split step; nullptr: off): the
  // rounding residue of sxx, szz, sxz per cell as bfloat16 bits, 3 planes
  // of slo_plane elements.  The stress update adds each increment to
  // sigma + residue with an error-free two-sum and keeps the new residue.
  uint16_t *slo;
  long long slo_plane;
  // H-AFDA free surface (free_surface == 2): weights / dz of the adjusted
  // one-sided z derivatives near the surface, af[op][q][m] (kAfdaN samples):
  // op 0 d(sxz)/dz at the vx row VI_HALF + q (samples sxz rows VI_HALF + m),
  // op 1 d(szz)/dz at the vz row VI_HALF + q (szz rows VI_HALF + 1 + m),
  // op 2 d(vz)/dz at the szz row VI_HALF + q (vz rows VI_HALF + m, q >= 1),
  // op 3 d(vx)/dz at the sxz row VI_HALF + q (vx rows VI_HALF + m);
  // ops 0, 2 for q < 4, ops 1, 3 for q < 3
  T af[4][4][5];
};
constexpr int kAfdaN = 5;  // samples of each adjusted one-sided derivative
constexpr int kFsImaging = 1, kFsAfda = 2;  // vi_config.free_surface values

// Bits of the device error word (plan or batch): a bounded wait gave up;
// a stress value came out non-finite (NaN or Inf in the medium or the
// state, or an unstable run).
enum { kErrTimeout = 1, kErrNonFinite = 2 };

__device__ __forceinline__ int strip_x(int i, int nx, int Lx, int Rx) {
  return i < Lx ? i : (i >= nx - Rx ? i - (nx - Rx) + Lx : -1);
}
__device__ __forceinline__ int strip_z(int j, int nz, int Tz, int Bz) {
  return j < Tz ? j : (j >= nz - Bz ? j - (nz - Bz) + Tz : -1);
}

// x-strip psi planes of one set: d(sxx)/dx at i+1/2, d(sxz)/dx at i,
// d(vx)/dx at i, d(vz)/dx at i+1/2
enum { PX_SXX = 0, PX_SXZ = 1, PX_VX = 2, PX_VZ = 3 };
// z-strip psi planes of one set: d(sxz)/dz at j, d(szz)/dz at j+1/2,
// d(vz)/dz at j, d(vx)/dz at j+1/2
enum { PZ_SXZ = 0, PZ_SZZ = 1, PZ_VZ = 2, PZ_VX = 3 };
constexpr int kPsiPerSet = 4;
constexpr int kPsiPlanes = 2 * kPsiPerSet;  // two sets for the ping-pong

// coefficient-table offsets
enum { T_IK = 0, T_A = 1, T_B = 2, T_IKH = 3, T_AH = 4, T_BH = 5 };

}  // namespace vb
