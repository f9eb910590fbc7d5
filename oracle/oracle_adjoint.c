/*
 * oracle_adjoint.c — discrete adjoint of the oracle's time step, FP64
 * (TEST INFRASTRUCTURE, like the rest of oracle/).
 *
 * The step of oracle_step.inc is linear in the state (v, sigma, memory
 * variables M, CPML psi) for a fixed medium; or_adjoint_step_f64 applies
 * its transpose, stage by stage in reverse, written here as scatters of
 * each forward statement's partial derivatives (serial loops: the clearest
 * form, and the sizes it serves are small):
 *   forward:  V (velocity, psi 0..3)  -> receivers -> S1 (rates, psi 4..7,
 *             effective SLS rates) -> S2 (tau_zz = 0 on the surface) -> S3
 *             (stress, memory variables) -> explosive sources -> surface
 *             (szz = 0, stress images)
 *   reverse:  surface^T -> S3^T -> S2^T -> S1^T -> [receiver residuals,
 *             by the caller] -> V^T
 * With the forward states before and after the step it also accumulates
 * the misfit gradient with respect to the medium planes (rho, c11, c13,
 * c15, c33, c35, c55, tau).  or_gradient_f64 runs the whole misfit
 * gradient: a forward run that keeps every state, then the reverse sweep.
 *
 * The reference has no adjoint or gradient (no Enzyme call exists; its
 * optimizer, EnergyNaturalGradient.jl:239-321, takes a grad_fn); this is
 * the transpose of the oracle's own restatement of the step
 * (visco-kernels.jl:3-85, diff-funcs.jl:3-32, CPML.jl:291-308,
 * free-surface-kernels.jl:84-95, CPML.jl:372-380, custom_solver/Model.jl:
 * 59-108).  The stress-imaging surface only (free_surface 0 or 1).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "visco_oracle.h"

#define L VI_HALF

typedef struct {
  int nx, nz, N, kind, fs;
  size_t np;
  double dt, Dx[4], Dz[4], a1[VI_MAX_SLS], a2[VI_MAX_SLS];
  /* CPML tables: integer (i) and half (h) nodes per axis */
  double *ikx, *ax, *bx, *ikxh, *axh, *bxh, *ikz, *az, *bz, *ikzh, *azh, *bzh;
  double *tab;
} adj_ctx;

static int ctx_init(adj_ctx *c, const vi_config *cfg) {
  c->nx = cfg->nx;
  c->nz = cfg->nz;
  c->N = cfg->nsls;
  c->kind = cfg->medium;
  c->fs = cfg->free_surface;
  c->np = (size_t)cfg->nx * cfg->nz;
  c->dt = cfg->dt;
  double D[4];
  or_stencil8(D);
  for (int k = 0; k < 4; ++k) {
    c->Dx[k] = D[k] / cfg->dx;
    c->Dz[k] = D[k] / cfg->dz;
  }
  for (int n = 0; n < c->N; ++n) {
    c->a1[n] = -1.0 / (c->N * cfg->tau_sls[n]);
    c->a2[n] = -1.0 / cfg->tau_sls[n];
  }
  const int nx = c->nx, nz = c->nz;
  c->tab = (double *)malloc(sizeof(double) * 6 * ((size_t)nx + nz));
  if (!c->tab) return VI_ERR_BUDGET;
  double *t = c->tab;
  c->ikx = t; c->ax = t + nx; c->bx = t + 2 * nx;
  c->ikxh = t + 3 * nx; c->axh = t + 4 * nx; c->bxh = t + 5 * nx;
  t += 6 * (size_t)nx;
  c->ikz = t; c->az = t + nz; c->bz = t + 2 * nz;
  c->ikzh = t + 3 * nz; c->azh = t + 4 * nz; c->bzh = t + 5 * nz;
  /* or_cpml_profile gives kappa, a, b; the step uses 1/kappa */
  or_cpml_profile(cfg, 0, 0, NULL, NULL, c->ikx, c->ax, c->bx);
  or_cpml_profile(cfg, 0, 1, NULL, NULL, c->ikxh, c->axh, c->bxh);
  or_cpml_profile(cfg, 1, 0, NULL, NULL, c->ikz, c->az, c->bz);
  or_cpml_profile(cfg, 1, 1, NULL, NULL, c->ikzh, c->azh, c->bzh);
  for (int k = 0; k < nx; ++k) {
    c->ikx[k] = 1.0 / c->ikx[k];
    c->ikxh[k] = 1.0 / c->ikxh[k];
  }
  for (int k = 0; k < nz; ++k) {
    c->ikz[k] = 1.0 / c->ikz[k];
    c->ikzh[k] = 1.0 / c->ikzh[k];
  }
  return VI_OK;
}

static int in_u(const adj_ctx *c, int i, int j) {
  return i >= L && i < c->nx - L && j >= L && j < c->nz - L;
}

/* p' = b p + a d, d~ = d ik + p' transposed: given the adjoint db of d~
 * and the adjoint *pb of p' (from the later steps), leaves the adjoint of
 * the old p in *pb and returns the adjoint of the raw d. */
static double cpml_t(double db, double *pb, double a, double b, double ik) {
  const double P = *pb + db;
  *pb = b * P;
  return db * ik + a * P;
}

/* Scatter the adjoint of d = sum_k D_k (u[c + (k+1) s] - u[c - k s])
 * (the ddxp / ddzp form) into u_b, and of the ddxm / ddzm form
 * d = sum_k D_k (u[c + k s] - u[c - (k+1) s]). */
static void tp(double *ub, size_t c, long s, const double *D, double db) {
  for (int k = 0; k < 4; ++k) {
    ub[c + (k + 1) * s] += D[k] * db;
    ub[c - k * s] -= D[k] * db;
  }
}
static void tm(double *ub, size_t c, long s, const double *D, double db) {
  for (int k = 0; k < 4; ++k) {
    ub[c + k * s] += D[k] * db;
    ub[c - (k + 1) * s] -= D[k] * db;
  }
}
static double dp(const double *u, size_t c, long s, const double *D) {
  double v = 0;
  for (int k = 0; k < 4; ++k) v += D[k] * (u[c + (k + 1) * s] - u[c - k * s]);
  return v;
}
static double dm(const double *u, size_t c, long s, const double *D) {
  double v = 0;
  for (int k = 0; k < 4; ++k) v += D[k] * (u[c + k * s] - u[c - (k + 1) * s]);
  return v;
}

/* C11, C33 of a cell (ISO: lambda + 2 mu). */
static double c11_at(const adj_ctx *c, const vi_medium *m, size_t q) {
  return c->kind == VI_MEDIUM_ISO ? ((const double *)m->c13)[q] + 2 * ((const double *)m->c55)[q]
                                  : ((const double *)m->c11)[q];
}
static double c33_at(const adj_ctx *c, const vi_medium *m, size_t q) {
  return c->kind == VI_MEDIUM_ISO ? ((const double *)m->c13)[q] + 2 * ((const double *)m->c55)[q]
                                  : ((const double *)m->c33)[q];
}

/* Forward rates of a step: rt (CPML'd strain rates xx, zz, xz), S (sums of
 * the old memory variables) and the effective rates e, on U (zero
 * elsewhere), from the new velocities v1 and the old psi and M of x0,
 * with the tau_zz = 0 relation on the surface row. */
static void fwd_rates(const adj_ctx *c, const vi_medium *m, const or_state *x0, const double *vx1,
                      const double *vz1, double *rt, double *S, double *e) {
  const int nx = c->nx, N = c->N;
  const size_t np = c->np;
  const double *psi = (const double *)x0->psi, *M = (const double *)x0->m;
  const double *tau = (const double *)m->tau;
  memset(rt, 0, 3 * np * sizeof(double));
  memset(S, 0, 3 * np * sizeof(double));
  memset(e, 0, 3 * np * sizeof(double));
  for (int j = L; j < c->nz - L; ++j)
    for (int i = L; i < nx - L; ++i) {
      const size_t q = (size_t)j * nx + i;
      double r0 = dm(vx1, q, 1, c->Dx), r1 = dm(vz1, q, nx, c->Dz);
      double r2 = dp(vx1, q, nx, c->Dz), r3 = dp(vz1, q, 1, c->Dx);
      r0 = r0 * c->ikx[i] + (c->bx[i] * psi[4 * np + q] + c->ax[i] * r0);
      r1 = r1 * c->ikz[j] + (c->bz[j] * psi[5 * np + q] + c->az[j] * r1);
      r2 = r2 * c->ikzh[j] + (c->bzh[j] * psi[6 * np + q] + c->azh[j] * r2);
      r3 = r3 * c->ikxh[i] + (c->bxh[i] * psi[7 * np + q] + c->axh[i] * r3);
      const double r[3] = {r0, r1, r2 + r3};
      for (int k = 0; k < 3; ++k) {
        double s = 0;
        for (int n = 0; n < N; ++n) s += M[(size_t)(k * N + n) * np + q];
        rt[k * np + q] = r[k];
        S[k * np + q] = s;
        e[k * np + q] = N > 0 ? (1 + tau[q]) * r[k] + tau[q] * s : r[k];
      }
    }
  if (c->fs)
    for (int i = L; i < nx - L; ++i) {
      const size_t q = (size_t)L * nx + i;
      const double *exx = e, *exz = e + 2 * np;
      double num = ((const double *)m->c13)[q] * exx[q];
      if (c->kind == VI_MEDIUM_TTI)
        num += ((const double *)m->c35)[q] * 0.25 * (exz[q] + exz[q - 1] + exz[q - nx] + exz[q - nx - 1]);
      e[np + q] = -num / c33_at(c, m, q);
    }
}

/* Transpose of the stress half of one step (surface, stress update,
 * surface relation, rates; sources excluded: they add constants), in
 * place on the adjoint state a (same layout as or_state).  With g != NULL
 * also accumulates the medium gradient (8 planes, vi_medium order; ISO
 * writes its stiffness terms into the c11/c13/c33/c55 planes as for VTI,
 * folded by the caller), which needs x0 (the state before the step) and x1
 * (after). */
int or_adjoint_stress_f64(const vi_config *cfg, const vi_medium *m, const or_state *x0, const or_state *x1,
                          or_state *a, double *g) {
  if (cfg->free_surface == 2) return VI_ERR_ARG;
  adj_ctx c;
  int rc = ctx_init(&c, cfg);
  if (rc) return rc;
  const int nx = c.nx, nz = c.nz, N = c.N, tti = c.kind == VI_MEDIUM_TTI;
  const size_t np = c.np;
  const double dt = c.dt;
  double *avx = (double *)a->vx, *avz = (double *)a->vz;
  double *asxx = (double *)a->sxx, *aszz = (double *)a->szz, *asxz = (double *)a->sxz;
  double *aM = (double *)a->m, *ap = (double *)a->psi;
  const double *c13 = (const double *)m->c13, *c55 = (const double *)m->c55;
  const double *c15 = (const double *)m->c15, *c35 = (const double *)m->c35, *tau = (const double *)m->tau;
  double *g11 = g ? g + np : NULL, *g13 = g ? g + 2 * np : NULL, *g15 = g ? g + 3 * np : NULL;
  double *g33 = g ? g + 4 * np : NULL, *g35 = g ? g + 5 * np : NULL, *g55 = g ? g + 6 * np : NULL;
  double *gt = g ? g + 7 * np : NULL;
  double *w = (double *)calloc(12 * np, sizeof(double));
  if (!w) {
    free(c.tab);
    return VI_ERR_BUDGET;
  }
  double *rt = w, *S = w + 3 * np, *e = w + 6 * np, *eb = w + 9 * np;
  if (g) fwd_rates(&c, m, x0, (const double *)x1->vx, (const double *)x1->vz, rt, S, e);

  /* ---- surface^T: images, then szz = 0 on the surface row ---- */
  if (c.fs) {
    for (int i = 0; i < nx; ++i) {
      for (int k = 1; k <= L; ++k) {
        aszz[(size_t)(L + k) * nx + i] -= aszz[(size_t)(L - k) * nx + i];
        aszz[(size_t)(L - k) * nx + i] = 0;
      }
      for (int k = 0; k < L; ++k) {
        asxz[(size_t)(L + k) * nx + i] -= asxz[(size_t)(L - 1 - k) * nx + i];
        asxz[(size_t)(L - 1 - k) * nx + i] = 0;
      }
      aszz[(size_t)L * nx + i] = 0;
    }
  }
  /* ---- S3^T: sigma' = sigma + dt ds(e): the stress adjoints pass through
   * and scatter into the effective-rate adjoints eb ---- */
  for (int j = L; j < nz - L; ++j)
    for (int i = L; i < nx - L; ++i) {
      const size_t q = (size_t)j * nx + i;
      const double bxx = asxx[q], bzz = aszz[q], bxz = asxz[q];
      const double C11 = c11_at(&c, m, q), C13 = c13[q], C33 = c33_at(&c, m, q);
      const double C55h = 0.25 * (c55[q] + c55[q + 1] + c55[q + nx] + c55[q + nx + 1]);
      eb[q] += dt * (C11 * bxx + C13 * bzz);
      eb[np + q] += dt * (C13 * bxx + C33 * bzz);
      eb[2 * np + q] += dt * C55h * bxz;
      if (tti) {
        /* ebxz(q): exz at q, q-1, q-nx, q-nx-1; ebxx, ebzz(q): exx, ezz at
         * q, q+1, q+nx, q+nx+1 (zero outside U: only U cells receive) */
        const size_t dm4[4] = {q, q - 1, q - nx, q - nx - 1}, pm4[4] = {q, q + 1, q + nx, q + nx + 1};
        const int im4[4] = {i, i - 1, i, i - 1}, jm4[4] = {j, j, j - 1, j - 1};
        const int ip4[4] = {i, i + 1, i, i + 1}, jp4[4] = {j, j, j + 1, j + 1};
        const double C15h = 0.25 * (c15[q] + c15[q + 1] + c15[q + nx] + c15[q + nx + 1]);
        const double C35h = 0.25 * (c35[q] + c35[q + 1] + c35[q + nx] + c35[q + nx + 1]);
        for (int k = 0; k < 4; ++k) {
          if (in_u(&c, im4[k], jm4[k])) eb[2 * np + dm4[k]] += 0.25 * dt * (c15[q] * bxx + c35[q] * bzz);
          if (in_u(&c, ip4[k], jp4[k])) {
            eb[pm4[k]] += 0.25 * dt * C15h * bxz;
            eb[np + pm4[k]] += 0.25 * dt * C35h * bxz;
          }
        }
      }
      if (g) {
        const double ex = e[q], ez = e[np + q], eq = e[2 * np + q];
        g11[q] += dt * bxx * ex;
        g13[q] += dt * (bxx * ez + bzz * ex);
        g33[q] += dt * bzz * ez;
        for (int k = 0; k < 4; ++k) { /* C55h: the mean over q, q+1, q+nx, q+nx+1 */
          const size_t pq = k == 0 ? q : k == 1 ? q + 1 : k == 2 ? q + nx : q + nx + 1;
          g55[pq] += 0.25 * dt * bxz * eq;
        }
        if (tti) {
          const double ebxz = 0.25 * (e[2 * np + q] + e[2 * np + q - 1] + e[2 * np + q - nx] + e[2 * np + q - nx - 1]);
          const double ebxx = 0.25 * (e[q] + e[q + 1] + e[q + nx] + e[q + nx + 1]);
          const double ebzz = 0.25 * (e[np + q] + e[np + q + 1] + e[np + q + nx] + e[np + q + nx + 1]);
          g15[q] += dt * bxx * ebxz;
          g35[q] += dt * bzz * ebxz;
          for (int k = 0; k < 4; ++k) {
            const size_t pq = k == 0 ? q : k == 1 ? q + 1 : k == 2 ? q + nx : q + nx + 1;
            g15[pq] += 0.25 * dt * bxz * ebxx;
            g35[pq] += 0.25 * dt * bxz * ebzz;
          }
        }
      }
    }

  /* ---- S2^T: the surface ezz = -(C13 exx + C35 ebxz) / C33 replaced the
   * raw rate there: move its adjoint onto exx (and exz, TTI), then drop
   * it ---- */
  if (c.fs)
    for (int i = L; i < nx - L; ++i) {
      const size_t q = (size_t)L * nx + i;
      const double zb = eb[np + q], C33 = c33_at(&c, m, q);
      eb[q] += -c13[q] / C33 * zb;
      if (tti) {
        eb[2 * np + q] += -0.25 * c35[q] / C33 * zb;
        if (in_u(&c, i - 1, L)) eb[2 * np + q - 1] += -0.25 * c35[q] / C33 * zb;
      }
      if (g) {
        const double ebs =
            tti ? 0.25 * (e[2 * np + q] + e[2 * np + q - 1] + e[2 * np + q - nx] + e[2 * np + q - nx - 1]) : 0.0;
        g13[q] += -zb * e[q] / C33;
        if (tti) g35[q] += -zb * ebs / C33;
        g33[q] += -zb * e[np + q] / C33;
      }
      eb[np + q] = 0;
    }
  /* ---- S1^T: effective rates -> strain rates, memory variables, tau;
   * CPML psi 4..7; the staggered derivatives of the new velocities ---- */
  for (int j = L; j < nz - L; ++j)
    for (int i = L; i < nx - L; ++i) {
      const size_t q = (size_t)j * nx + i;
      const int surf = c.fs && j == L;
      const double t = N > 0 ? tau[q] : 0.0;
      double rb[3];
      for (int k = 0; k < 3; ++k) rb[k] = (N > 0 ? 1 + t : 1.0) * eb[k * np + q];
      if (g && N > 0)
        for (int k = 0; k < 3; ++k) gt[q] += eb[k * np + q] * (rt[k * np + q] + S[k * np + q]);
      for (int n = 0; n < N; ++n)
        for (int k = 0; k < 3; ++k) {
          double *mb = &aM[(size_t)(k * N + n) * np + q];
          const double mprime = (surf && k == 1) ? 0.0 : *mb; /* Mzz' = 0 on the surface */
          rb[k] += dt * c.a1[n] * mprime;
          *mb = t * eb[k * np + q] + (1 + dt * c.a2[n]) * mprime;
        }
      const double d0 = cpml_t(rb[0], &ap[4 * np + q], c.ax[i], c.bx[i], c.ikx[i]);
      const double d1 = cpml_t(rb[1], &ap[5 * np + q], c.az[j], c.bz[j], c.ikz[j]);
      const double d2 = cpml_t(rb[2], &ap[6 * np + q], c.azh[j], c.bzh[j], c.ikzh[j]);
      const double d3 = cpml_t(rb[2], &ap[7 * np + q], c.axh[i], c.bxh[i], c.ikxh[i]);
      tm(avx, q, 1, c.Dx, d0);
      tm(avz, q, nx, c.Dz, d1);
      tp(avx, q, nx, c.Dz, d2);
      tp(avz, q, 1, c.Dx, d3);
    }
  free(w);
  free(c.tab);
  return VI_OK;
}

/* V^T of step it: the adjoint of the new velocities (a->vx, a->vz, after
 * the caller added the receiver residuals) into the stress adjoints and
 * CPML psi 0..3, and with g the rho gradient (buoyancy of the velocity
 * update and of the force sources).  x0: the state before the step. */
int or_adjoint_velocity_f64(const vi_config *cfg, const vi_medium *m, const or_state *x0, or_state *a, double *g,
                            int nsrc, const vi_source *src, const double *wavelet, int wavelet_nt, int it) {
  adj_ctx c;
  int rc = ctx_init(&c, cfg);
  if (rc) return rc;
  const int nx = c.nx, nz = c.nz;
  const size_t np = c.np;
  const double dt = c.dt;
  const double *rho = (const double *)m->rho;
  double *avx = (double *)a->vx, *avz = (double *)a->vz;
  double *asxx = (double *)a->sxx, *aszz = (double *)a->szz, *asxz = (double *)a->sxz, *ap = (double *)a->psi;
  if (g) /* force sources: v += dt b f, b = 2 / (rho_q + rho_neighbour) */
    for (int s = 0; s < nsrc; ++s) {
      if (src[s].kind == VI_SRC_EXPLOSIVE) continue;
      const size_t q = (size_t)src[s].j * nx + src[s].i;
      const double f = src[s].amp * (it < wavelet_nt ? wavelet[(size_t)s * wavelet_nt + it] : 0.0);
      const size_t qn = src[s].kind == VI_SRC_FORCE_X ? q + 1 : q + nx;
      const double b = 2.0 / (rho[q] + rho[qn]);
      const double w = dt * f * (-0.5 * b * b) * (src[s].kind == VI_SRC_FORCE_X ? avx[q] : avz[q]);
      g[q] += w;
      g[qn] += w;
    }
  /* the forward state is read only for the gradient */
  const double *sxx = g ? (const double *)x0->sxx : NULL, *szz = g ? (const double *)x0->szz : NULL;
  const double *sxz = g ? (const double *)x0->sxz : NULL, *psi = g ? (const double *)x0->psi : NULL;
  for (int j = L; j < nz - L; ++j)
    for (int i = L; i < nx - L; ++i) {
      const size_t q = (size_t)j * nx + i;
      const double bxv = 2.0 / (rho[q] + rho[q + 1]), bzv = 2.0 / (rho[q] + rho[q + nx]);
      if (g) {
        double d0 = dp(sxx, q, 1, c.Dx), d1 = dm(sxz, q, nx, c.Dz);
        double d2 = dm(sxz, q, 1, c.Dx), d3 = dp(szz, q, nx, c.Dz);
        d0 = d0 * c.ikxh[i] + (c.bxh[i] * psi[q] + c.axh[i] * d0);
        d1 = d1 * c.ikz[j] + (c.bz[j] * psi[np + q] + c.az[j] * d1);
        d2 = d2 * c.ikx[i] + (c.bx[i] * psi[2 * np + q] + c.ax[i] * d2);
        d3 = d3 * c.ikzh[j] + (c.bzh[j] * psi[3 * np + q] + c.azh[j] * d3);
        const double wx = dt * (d0 + d1) * (-0.5 * bxv * bxv) * avx[q];
        const double wz = dt * (d2 + d3) * (-0.5 * bzv * bzv) * avz[q];
        g[q] += wx + wz;
        g[q + 1] += wx;
        g[q + nx] += wz;
      }
      const double dbx = dt * bxv * avx[q], dbz = dt * bzv * avz[q];
      tp(asxx, q, 1, c.Dx, cpml_t(dbx, &ap[q], c.axh[i], c.bxh[i], c.ikxh[i]));
      tm(asxz, q, nx, c.Dz, cpml_t(dbx, &ap[np + q], c.az[j], c.bz[j], c.ikz[j]));
      tm(asxz, q, 1, c.Dx, cpml_t(dbz, &ap[2 * np + q], c.ax[i], c.bx[i], c.ikx[i]));
      tp(aszz, q, nx, c.Dz, cpml_t(dbz, &ap[3 * np + q], c.azh[j], c.bzh[j], c.ikzh[j]));
    }
  free(c.tab);
  return VI_OK;
}

/* The whole transposed step, no sources or receivers (the linear state
 * map's transpose, for the dot-product test). */
int or_adjoint_step_f64(const vi_config *cfg, const vi_medium *m, or_state *a) {
  int rc = or_adjoint_stress_f64(cfg, m, NULL, NULL, a, NULL);
  if (rc) return rc;
  return or_adjoint_velocity_f64(cfg, m, NULL, a, NULL, 0, NULL, NULL, 0, 0);
}

/* Misfit J = 1/2 sum (d - obs)^2 over the vx, vz traces of an nt-step run
 * from rest, and dJ/d(rho, c11, c13, c15, c33, c35, c55, tau) into grad
 * (8 planes, overwritten; ISO: dJ/dlambda in the c13 plane, dJ/dmu in the
 * c55 plane, as vi_gradient).  Every forward state is kept: small grids. */
int or_gradient_f64(const vi_config *cfg, const vi_medium *m, int nsrc, const vi_source *src,
                    const double *wavelet, int wavelet_nt, int nrec, const vi_receiver *rec, const double *obs,
                    int nt, double *grad, double *misfit) {
  if (cfg->free_surface == 2) return VI_ERR_ARG;
  const size_t np = (size_t)cfg->nx * cfg->nz;
  const int N = cfg->nsls;
  const size_t nm = 3 * (size_t)(N > 0 ? N : 1);
  const size_t per = (5 + nm + 8) * np;
  double *X = (double *)calloc((size_t)(nt + 1) * per, sizeof(double));
  double *A = (double *)calloc(per, sizeof(double));
  double *tr = (double *)calloc(2 * (size_t)nrec * nt + 1, sizeof(double));
  if (!X || !A || !tr) {
    free(X);
    free(A);
    free(tr);
    return VI_ERR_BUDGET;
  }
  or_state st[2];
#define MKST(s, base)                                     \
  do {                                                    \
    (s).vx = (base);                                      \
    (s).vz = (base) + np;                                 \
    (s).sxx = (base) + 2 * np;                            \
    (s).szz = (base) + 3 * np;                            \
    (s).sxz = (base) + 4 * np;                            \
    (s).m = (base) + 5 * np;                              \
    (s).psi = (base) + (5 + nm) * np;                     \
  } while (0)
  int rc = VI_OK;
  for (int it = 0; it < nt && !rc; ++it) {
    memcpy(X + (size_t)(it + 1) * per, X + (size_t)it * per, per * sizeof(double));
    MKST(st[0], X + (size_t)(it + 1) * per);
    rc = or_run_f64(cfg, m, &st[0], it, 1, nsrc, src, wavelet, wavelet_nt, nrec, rec, tr, nt);
  }
  double J = 0;
  for (size_t k = 0; k < 2 * (size_t)nrec * nt; ++k) {
    const double d = tr[k] - obs[k];
    J += 0.5 * d * d;
  }
  memset(grad, 0, 8 * np * sizeof(double));
  or_state a;
  MKST(a, A);
  for (int it = nt - 1; it >= 0 && !rc; --it) {
    MKST(st[0], X + (size_t)it * per);
    MKST(st[1], X + (size_t)(it + 1) * per);
    rc = or_adjoint_stress_f64(cfg, m, &st[0], &st[1], &a, grad);
    if (rc) break;
    for (int r = 0; r < nrec; ++r) { /* receivers sampled the new velocities */
      const size_t q = (size_t)rec[r].j * cfg->nx + rec[r].i;
      ((double *)a.vx)[q] += tr[(size_t)r * nt + it] - obs[(size_t)r * nt + it];
      ((double *)a.vz)[q] += tr[(size_t)(nrec + r) * nt + it] - obs[(size_t)(nrec + r) * nt + it];
    }
    rc = or_adjoint_velocity_f64(cfg, m, &st[0], &a, grad, nsrc, src, wavelet, wavelet_nt, it);
  }
#undef MKST
  if (!rc && cfg->medium == VI_MEDIUM_ISO)
    for (size_t q = 0; q < np; ++q) {
      const double g11 = grad[np + q], g13 = grad[2 * np + q], g33 = grad[4 * np + q], g55 = grad[6 * np + q];
      grad[2 * np + q] = g11 + g13 + g33;      /* C11 = C33 = lambda + 2 mu, C13 = lambda */
      grad[6 * np + q] = 2 * (g11 + g33) + g55; /* C55 = mu */
      grad[np + q] = 0;
      grad[4 * np + q] = 0;
    }
  *misfit = J;
  free(X);
  free(A);
  free(tr);
  return rc;
}
