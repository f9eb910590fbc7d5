/*
 * visco_oracle.c — CPU oracle (test infrastructure; see visco_oracle.h).
 *
 * Straightforward loops, one pass per physical stage, OpenMP over rows.
 * The step body lives in oracle_step.inc, included once per precision.
 *
 * Reference restated (haralddd/ViscoelasticInversion, Julia):
 *   staggered operators ddxp/ddxm/ddzp/ddzm ........ src/diff-funcs.jl:3-32
 *   8th-order coefficients (rational Vandermonde) ... src/common/Stencil.jl:9-14,280-328
 *   velocity update, buoyancy 2/(rho_i+rho_i+1) ..... src/visco-kernels.jl:3-20
 *   SLS stress law and memory variables ............. src/visco-kernels.jl:22-85
 *   mu 4-point average at (i+1/2,j+1/2) ............. src/visco-kernels.jl:25
 *   Voigt C11..C55 stress law (TTI) .................. src/custom_solver/Model.jl:59-66,98-100
 *   CPML profiles and a/b coefficients ............... src/sciml_solver/CPML.jl:55-61,91-102,109-189
 *   CPML derivative correction du/kappa + psi ........ src/sciml_solver/CPML.jl:291-308
 *   stress imaging free surface ...................... src/sciml_solver/CPML.jl:366-393
 *   tau_zz = 0 relation at the surface ............... src/free-surface-kernels.jl:84-95,106,116
 *   Ricker wavelet ................................... src/sciml_solver/Source.jl:3-5
 *   source added before buoyancy scaling ............. src/sciml_solver/ViscoelasticProblem.jl:162-171
 * The fixes applied to the reference's inconsistencies (engineering shear
 * strain, the dszz pairing, the velocity operator staggering) are the
 * physics choices documented with the step in the package; both this
 * oracle and the CUDA kernels implement them.
 */
#include "visco_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define L VI_HALF

/* Stencil.jl:_stencil on the half-integer points -7/2..7/2, derivative of
 * order 1 at 0: the staggered 8th-order weights are
 * +-1225/1024, -+245/3072, +-49/5120, -+5/7168. */
static const double D8[4] = {1225.0 / 1024.0, -245.0 / 3072.0, 49.0 / 5120.0,
                             -5.0 / 7168.0};

void or_stencil8(double *D) {
  for (int k = 0; k < 4; ++k) D[k] = D8[k];
}

double or_ricker(double f, double t) {
  const double x = M_PI * f * t;
  return (1.0 - 2.0 * x * x) * exp(-x * x);
}

int or_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* Damping profile of CPML.jl:91-102 at normalised depth p in (0,1]. */
static void pml_point(double p, double d0, double power, double amax,
                      double kmax, double dt, double *d, double *al,
                      double *ka, double *a, double *b) {
  if (p > 0.0) {
    *d = d0 * pow(p, power);
    *al = amax * (1.0 - p);
    *ka = 1.0 + (kmax - 1.0) * p;
  } else {
    *d = 0.0;
    *al = 0.0;
    *ka = 1.0;
  }
  /* CPML.jl:171-179 */
  if (*d > 0.0 || *al > 0.0) {
    *b = exp(-(*d / *ka + *al) * dt);
    *a = (fabs(*d) > DBL_EPSILON) ? *d / (*ka * (*d + *ka * *al)) * (*b - 1.0)
                                  : 0.0;
  } else {
    *b = 0.0;
    *a = 0.0;
  }
}

int or_cpml_profile(const vi_config *cfg, int axis, int half, double *d,
                    double *alpha, double *kappa, double *a, double *b) {
  const int n = axis == 0 ? cfg->nx : cfg->nz;
  const double h = axis == 0 ? cfg->dx : cfg->dz;
  const int lo = axis == 0 ? cfg->pml_left : cfg->pml_top;
  const int hi = axis == 0 ? cfg->pml_right : cfg->pml_bottom;
  const double Lp = (double)cfg->pml_thickness;
  double d0 = cfg->pml_d0;
  if (d0 <= 0.0) /* Collino & Tsogka, CPML.jl:60 */
    d0 = -(cfg->pml_power + 1.0) * cfg->pml_vmax * log(cfg->pml_reflection) /
         (2.0 * Lp * h);
  for (int k = 0; k < n; ++k) {
    const double x = k + (half ? 0.5 : 0.0);
    double p = 0.0;
    if (cfg->pml_thickness > 0) {
      /* left strip: interface at Lp-1/2 (CPML.jl:123-124 in 0-based form) */
      if (lo) {
        const double pl = (Lp - 0.5 - x) / Lp;
        if (pl > p) p = pl;
      }
      /* right strip: interface at n-Lp-1/2 (CPML.jl:133-134) */
      if (hi) {
        const double pr = (x - ((double)n - Lp - 0.5)) / Lp;
        if (pr > p) p = pr;
      }
    }
    double dd, al, ka, aa, bb;
    pml_point(p, d0, cfg->pml_power, cfg->pml_alpha_max, cfg->pml_kappa_max,
              cfg->dt, &dd, &al, &ka, &aa, &bb);
    if (d) d[k] = dd;
    if (alpha) alpha[k] = al;
    if (kappa) kappa[k] = ka;
    if (a) a[k] = aa;
    if (b) b[k] = bb;
  }
  return 0;
}

/* ---- per-precision step body ---- */
#define REAL double
#define SFX(name) name##_f64
#include "oracle_step.inc"
#undef REAL
#undef SFX

#define REAL float
#define SFX(name) name##_f32
#include "oracle_step.inc"
#undef REAL
#undef SFX
