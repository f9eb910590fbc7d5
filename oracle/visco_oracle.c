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
 *   H-AFDA free surface (one-sided z derivatives) ..... src/free-surface-kernels.jl:16-213,
 *                                                       src/common/Stencil.jl:52-105
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

/* Weights w[0..n-1] of the first derivative at x0 from samples at x[0..n-1]
 * (n <= 8): the conditions sum_k w_k (x_k - x0)^l / l! = [l == 1], l < n,
 * the Vandermonde system Stencil.jl:_stencil solves in rationals (its
 * lines 9-14), here by Gaussian elimination with partial pivoting. */
static void fd_weights(const double *x, int n, double x0, double *w) {
  double A[8][9];
  for (int l = 0; l < n; ++l) {
    double fact = 1.0;
    for (int q = 2; q <= l; ++q) fact *= q;
    for (int k = 0; k < n; ++k) A[l][k] = pow(x[k] - x0, l) / fact;
    A[l][n] = l == 1 ? 1.0 : 0.0;
  }
  for (int c = 0; c < n; ++c) {
    int p = c;
    for (int r = c + 1; r < n; ++r)
      if (fabs(A[r][c]) > fabs(A[p][c])) p = r;
    for (int k = 0; k <= n; ++k) {
      const double t = A[c][k];
      A[c][k] = A[p][k];
      A[p][k] = t;
    }
    for (int r = 0; r < n; ++r)
      if (r != c && A[r][c] != 0.0) {
        const double f = A[r][c] / A[c][c];
        for (int k = c; k <= n; ++k) A[r][k] -= f * A[c][k];
      }
  }
  for (int k = 0; k < n; ++k) w[k] = A[k][n] / A[k][k];
}

/* H-AFDA free surface (Kristek, Moczo & Archuleta 2002; the reference's
 * FreeSurfaceStencil, Stencil.jl:52-105, and its kernels,
 * free-surface-kernels.jl:16-213): the surface z = 0 lies on the row of
 * sxx, szz and vx (row VI_HALF); szz(0) = 0 and sxz(0) = 0 there; nothing
 * lives above it.  The z derivatives whose 8th-order staggered stencil
 * would reach above the surface use adjusted one-sided approximations of
 * AFDA_N = 5 samples (plus the zero boundary value where there is one):
 *   0  d(sxz)/dz at vx rows z = q h (q = 0..3): samples sxz at (m + 1/2) h,
 *      m = 0..4, and sxz(0) = 0;
 *   1  d(szz)/dz at vz rows z = (q + 1/2) h (q = 0..2): samples szz at
 *      m h, m = 1..5, and szz(0) = 0;
 *   2  d(vz)/dz at szz rows z = q h (q = 1..3): samples vz at (m + 1/2) h,
 *      m = 0..4 (on the surface row the tau_zz = 0 relation gives it);
 *   3  d(vx)/dz at sxz rows z = (q + 1/2) h (q = 0..2): samples vx at m h,
 *      m = 0..4.
 * w[op][q][m] (unit spacing) multiplies the sample of row VI_HALF + m
 * (op 1: row VI_HALF + 1 + m).  The reference builds these one-sided
 * approximations with as many samples as the interior stencil (8); with 8
 * the semi-discrete operator has growing modes (eigenvalues with real
 * part 0.4 c/h in a 1D half-space), with 5 it has none, so 5 are used. */
void or_afda_weights(double w[4][4][AFDA_N]) {
  double x[AFDA_N + 1], t[AFDA_N + 1];
  memset(w, 0, sizeof(double) * 4 * 4 * AFDA_N);
  for (int q = 0; q < 4; ++q) { /* op 0 */
    x[0] = 0.0;
    for (int m = 0; m < AFDA_N; ++m) x[m + 1] = m + 0.5;
    fd_weights(x, AFDA_N + 1, (double)q, t);
    for (int m = 0; m < AFDA_N; ++m) w[0][q][m] = t[m + 1];
  }
  for (int q = 0; q < 3; ++q) { /* op 1 */
    for (int m = 0; m <= AFDA_N; ++m) x[m] = m;
    fd_weights(x, AFDA_N + 1, q + 0.5, t);
    for (int m = 0; m < AFDA_N; ++m) w[1][q][m] = t[m + 1];
  }
  for (int q = 1; q < 4; ++q) { /* op 2 */
    for (int m = 0; m < AFDA_N; ++m) x[m] = m + 0.5;
    fd_weights(x, AFDA_N, (double)q, t);
    for (int m = 0; m < AFDA_N; ++m) w[2][q][m] = t[m];
  }
  for (int q = 0; q < 3; ++q) { /* op 3 */
    for (int m = 0; m < AFDA_N; ++m) x[m] = m;
    fd_weights(x, AFDA_N, q + 0.5, t);
    for (int m = 0; m < AFDA_N; ++m) w[3][q][m] = t[m];
  }
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
