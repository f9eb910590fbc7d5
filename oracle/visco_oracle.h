/*
 * visco_oracle.h — CPU oracle for the 2D viscoelastic staggered-grid step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-loop C restatement of the
 * reference's hot path (haralddd/ViscoelasticInversion, Julia) used by the
 * tests, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg as
 * the checker.  The product (libvisco_b200.so) never links or calls it.
 *
 * Parity status: the reference's step kernels cannot run (undefined `D`,
 * `_ddz`, wrong arities; no Julia on this machine), and no reference test
 * touches them, so the step itself is "parity unpinned".  The pieces the
 * reference's tests do pin (Ricker wavelet, CPML profile, source injection,
 * stencil coefficients) are checked against those tests' facts in
 * tests/test_oracle_golden.py.
 */
#ifndef VISCO_ORACLE_H
#define VISCO_ORACLE_H

#include "../include/visco_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Oracle state: full nx*nz planes.  psi holds 8 full CPML planes:
 *  0 psi(d sxx/dx) at (i+1/2,j)   1 psi(d sxz/dz) at (i+1/2,j)
 *  2 psi(d sxz/dx) at (i,j+1/2)   3 psi(d szz/dz) at (i,j+1/2)
 *  4 psi(d vx/dx)  at (i,j)       5 psi(d vz/dz)  at (i,j)
 *  6 psi(d vx/dz)  at (i+1/2,j+1/2)  7 psi(d vz/dx) at (i+1/2,j+1/2) */
typedef struct or_state {
  void *vx, *vz, *sxx, *szz, *sxz, *m, *psi;
} or_state;

/* Runs nsteps steps from step index it0 (same step definition as vi_step).
 * All arrays are host arrays of double (f64) or float (f32). */
int or_run_f64(const vi_config *cfg, const vi_medium *med, or_state *st,
               int it0, int nsteps, int nsrc, const vi_source *src,
               const double *wavelet, int wavelet_nt, int nrec,
               const vi_receiver *rec, double *traces, int traces_nt);
int or_run_f32(const vi_config *cfg, const vi_medium *med, or_state *st,
               int it0, int nsteps, int nsrc, const vi_source *src,
               const float *wavelet, int wavelet_nt, int nrec,
               const vi_receiver *rec, float *traces, int traces_nt);

/* CPML profile along one axis (0 = x, 1 = z) at integer (half = 0) or
 * half (half = 1) nodes.  Outputs n = nx or nz values each. */
int or_cpml_profile(const vi_config *cfg, int axis, int half, double *d,
                    double *alpha, double *kappa, double *a, double *b);

/* Ricker wavelet (1 - 2 (pi f t)^2) exp(-(pi f t)^2), Source.jl:3-5. */
double or_ricker(double f, double t);

/* The 8th-order staggered half-stencil D[0..3] (unit spacing). */
void or_stencil8(double *D);

/* H-AFDA free surface (vi_config.free_surface = 2): unit-spacing weights of
 * the adjusted one-sided z derivatives near the surface, w[op][q][m]
 * (see visco_oracle.c for the operators, rows and samples). */
#define AFDA_N 5
void or_afda_weights(double w[4][4][AFDA_N]);

/* Discrete adjoint of the FP64 step (oracle_adjoint.c): the transposed
 * stress half and velocity half of one step on an adjoint state a, with
 * the medium gradient (8 planes) accumulated when g != NULL (x0 / x1: the
 * forward states before / after the step); the whole transposed step
 * without sources (dot-product tests); and the misfit gradient of an
 * nt-step run (every forward state kept: small grids).  Stress-imaging
 * surface only. */
int or_adjoint_stress_f64(const vi_config *cfg, const vi_medium *m, const or_state *x0, const or_state *x1,
                          or_state *a, double *g);
int or_adjoint_velocity_f64(const vi_config *cfg, const vi_medium *m, const or_state *x0, or_state *a, double *g,
                            int nsrc, const vi_source *src, const double *wavelet, int wavelet_nt, int it);
int or_adjoint_step_f64(const vi_config *cfg, const vi_medium *m, or_state *a);
int or_gradient_f64(const vi_config *cfg, const vi_medium *m, int nsrc, const vi_source *src,
                    const double *wavelet, int wavelet_nt, int nrec, const vi_receiver *rec, const double *obs,
                    int nt, double *grad, double *misfit);

/* Number of OpenMP threads the oracle uses. */
int or_num_threads(void);

#ifdef __cplusplus
}
#endif
#endif
