/*
 * visco_b200.h — C ABI of the B200 (sm_100a) 2D viscoelastic / anisotropic
 * staggered-grid velocity–stress time step.
 *
 * The reference (haralddd/ViscoelasticInversion) is Julia; its hot path is the
 * set of KernelAbstractions kernels in src/visco-kernels.jl,
 * src/diff-funcs.jl, src/free-surface-kernels.jl and the custom_solver
 * Solver/PointSource types.  Each entry point below names the reference item
 * it replaces (file:line).  The reference binds nothing over an FFI; a Julia
 * `ccall` veneer or the Python host package calls these.
 *
 * Conventions
 *   - Arrays are x-fastest (Julia column-major [Nx,Nz]): element (i,j) of a
 *     plane lives at i + j*nx, 0 <= i < nx, 0 <= j < nz.
 *   - Staggering (Virieux): sxx, szz, rho, C, tau at (i, j); vx at (i+1/2, j);
 *     vz at (i, j+1/2); sxz at (i+1/2, j+1/2).  Memory variables sit with the
 *     stress component they drive.
 *   - Only the update region U = [4, nx-4) x [4, nz-4) is ever written; cells
 *     outside U stay as the caller left them (zero), as the reference's
 *     `worksize = size - 2*pad` launch (visco-kernels.jl:95-98) does.
 *   - With the free surface on, row 4 is the surface (sxx, szz, vx level) and
 *     rows 0..3 hold the stress images.
 *   - All calls return an int status (VI_OK = 0).  vi_last_error() gives the
 *     message of the last failing call on the calling thread.  No C++
 *     exception or device trap crosses this boundary.
 *   - Pointers named *_dev are device pointers; *_host are host pointers.
 *     The precision of every real array is the plan's precision (float for
 *     VI_F32, double for VI_F64).
 */
#ifndef VISCO_B200_H
#define VISCO_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VI_ABI_VERSION 1
#define VI_HALF 4          /* half-length of the 8th-order staggered stencil */
#define VI_MAX_SLS 5       /* maximum number of standard linear solids */

/* status codes */
#define VI_OK 0
#define VI_ERR_ARG 1        /* bad argument / configuration */
#define VI_ERR_CFL 2        /* CFL condition violated */
#define VI_ERR_BUDGET 3     /* HBM budget or capacity exceeded */
#define VI_ERR_TIMEOUT 4    /* a bounded device wait gave up */
#define VI_ERR_CUDA 5       /* CUDA runtime error */
#define VI_ERR_NONFINITE 6  /* a non-finite value was detected */
#define VI_ERR_STATE 7      /* call not valid in the object's current state */

/* medium kinds (sciml_solver/Models.jl:3-43) */
#define VI_MEDIUM_ISO 0     /* reads rho, c13 (= lambda), c55 (= mu), tau */
#define VI_MEDIUM_VTI 1     /* reads rho, c11, c13, c33, c55, tau */
#define VI_MEDIUM_TTI 2     /* reads rho, c11, c13, c15, c33, c35, c55, tau */

#define VI_F32 0
#define VI_F64 1
/* FP32 fields whose split-pair stress update is compensated: each cell's
 * rounding error of sxx, szz and sxz is kept in a bfloat16 residue plane
 * of the plan and folded into the next update (an error-free two-sum), so
 * the float stresses do not drift over long runs.  Costs 12 bytes per cell
 * per step (about 13 % of the 2048 x 1024 VTI step); kernel variants 0, 5
 * and 8 only (the others return VI_ERR_ARG). */
#define VI_F32C 2

/* source kinds */
#define VI_SRC_EXPLOSIVE 0  /* sxx, szz += dt*amp*w(t) */
#define VI_SRC_FORCE_X 1    /* vx += dt*b*amp*w(t)   (Source.jl:35-58 form) */
#define VI_SRC_FORCE_Z 2    /* vz += dt*b*amp*w(t)   (ViscoelasticProblem.jl:165-171) */

/* Plan configuration.  Mirrors Parameters(;Nx,Nz,dx,dz,dt,...)
 * (sciml_solver/Parameters.jl:47-86), CPMLConfig (sciml_solver/CPML.jl:40-63)
 * and QModel's tau_n (sciml_solver/Models.jl:90-102). */
typedef struct vi_config {
  int32_t nx, nz;
  double dx, dz, dt;
  int32_t medium;          /* VI_MEDIUM_* */
  int32_t precision;       /* VI_F32 / VI_F64 / VI_F32C */
  int32_t nsls;            /* 0..VI_MAX_SLS */
  int32_t free_surface;    /* 0 none (top CPML allowed); 1 stress-imaging
                              free surface at row VI_HALF (CPML.jl:366-393);
                              2 H-AFDA free surface at row VI_HALF: the z
                              derivatives whose stencil would reach above it
                              are one-sided (free-surface-kernels.jl:16-213,
                              Stencil.jl:52-105), nothing is written above
                              it; kernel variants 0, 1, 5 and 8 only */
  double tau_sls[VI_MAX_SLS]; /* relaxation times tau_n of the mechanisms */
  /* CPML */
  int32_t pml_thickness;   /* cells, counted from the array edge */
  int32_t pml_left, pml_right, pml_top, pml_bottom;
  double pml_d0;           /* <= 0: Collino–Tsogka d0 from vmax and R */
  double pml_vmax;
  double pml_reflection;   /* R in d0 = -(p+1) vmax ln R / (2 L h) */
  double pml_power;
  double pml_alpha_max;
  double pml_kappa_max;
} vi_config;

/* Medium planes (nx*nz each).  For VI_MEDIUM_ISO, c11 = c33 = c13 + 2*c55
 * is derived on chip and c11/c15/c33/c35 are ignored. */
typedef struct vi_medium {
  const void *rho, *c11, *c13, *c15, *c33, *c35, *c55, *tau;
} vi_medium;

/* Wavefield state.  Maps both the reference's stacked Fields(s, M, v)
 * arrays (visco-kernels.jl:102-106: s[Nx,Nz,3], v[Nx,Nz,2], M[Nx,Nz,N,3])
 * and the custom Solver(vx,vz,sxx,szz,sxz) planes (custom_solver/Model.jl:4-10)
 * without a copy.  m holds 3*nsls planes; plane (c*nsls + n) is memory
 * variable n of component c (0 = xx, 1 = zz, 2 = xz), each m_plane_stride
 * elements apart. */
typedef struct vi_fields {
  void *vx, *vz, *sxx, *szz, *sxz, *m;
  int64_t m_plane_stride;
} vi_fields;

typedef struct vi_source {
  int32_t i, j, kind;
  int32_t pad_;
  double amp;
} vi_source;

typedef struct vi_receiver {
  int32_t i, j;            /* samples vx(i+1/2, j) and vz(i, j+1/2) */
} vi_receiver;

/* Shot description for the time loop.  wavelet_dev holds nsrc rows of
 * wavelet_nt samples (plan precision); step it uses sample
 * w[s*wavelet_nt + it] (zero when it >= wavelet_nt).  traces_dev receives
 * 2*nrec rows of traces_nt samples: row r is vx of receiver r, row nrec+r is
 * vz; step it writes column it (when it < traces_nt).  Index lists are host
 * pointers copied by the call. */
typedef struct vi_shot {
  int32_t nsrc;
  const vi_source *src_host;
  const void *wavelet_dev;
  int32_t wavelet_nt;
  int32_t nrec;
  const vi_receiver *rec_host;
  void *traces_dev;
  int32_t traces_nt;
} vi_shot;

typedef struct vi_plan vi_plan;

/* ---- library ---------------------------------------------------------- */
int vi_version(void);
const char *vi_last_error(void);

/* ---- plan ------------------------------------------------------------- */
/* Builds the CPML profiles (CPML.jl:109-221, evaluated at the staggered
 * positions), checks CFL and allocates the plan's device workspace (CPML
 * psi strips).  Replaces the host set-up of Parameters(;...)
 * (Parameters.jl:47-86) for the leapfrog path. */
int vi_plan_create(const vi_config *cfg, vi_plan **out);
int vi_plan_destroy(vi_plan *plan);
/* Zeroes the plan's CPML memory variables (CPMLMemory, CPML.jl:246-263)
 * and, for VI_F32C plans, the stress rounding residues (see VI_F32C).  Call
 * it whenever the caller resets or replaces the fields between calls. */
int vi_plan_reset(vi_plan *plan, void *stream);
/* Bytes of device memory the plan holds. */
int vi_plan_workspace_bytes(const vi_plan *plan, int64_t *bytes);
/* Synchronizes `stream` and reports (then clears) the plan's device error
 * word: VI_ERR_TIMEOUT when a bounded in-kernel wait gave up,
 * VI_ERR_NONFINITE when a stress value came out NaN or infinite (a
 * non-finite medium or state, or an unstable run; the split pair checks
 * every step in its stress pass, the other paths once at the end of each
 * vi_step call).  Kernels never trap; this is how a device-side failure
 * reaches the caller. */
int vi_plan_status(vi_plan *plan, void *stream);
/* Which kernel the last vi_step ran: 1 plain, 2 fused, 3 fused TMA-staged,
 * 4 fused TMA-staged single-stage, 5 split velocity/stress pair, 6 split
 * pair, persistent and TMA-pipelined, 7 streaming, 8 split pair with the
 * direct-load velocity pass. */
int vi_plan_last_kernel(const vi_plan *plan, int32_t *kernel);

/* ---- time stepping ------------------------------------------------------ */
/* Advances the caller's wavefields by nsteps leapfrog steps starting at step
 * index it0, in place, on `stream` (asynchronous).  One step = velocity
 * update from the stress divergence (+ force sources, receivers sampled),
 * then the SLS stress + memory-variable update (+ explosive sources), the
 * free-surface condition and the stress images.  Replaces
 * leapfrog_step!(fields, parameters, dt) (visco-kernels.jl:87-100) together
 * with _vel_1Q! (:3-20), _stress_1Q! (:59-85), the free-surface kernels
 * (free-surface-kernels.jl:16-213) and the CPML/ψ recursion
 * (sciml_solver/CPML.jl:291-328).  `shot` may be NULL (no sources or
 * receivers).  kernel_variant: 0 = default (with nx % 4 == 0 and 16-byte
 * aligned planes the split pair, else the fused kernel), 1 = plain
 * multi-kernel path (in place), 2 = fused kernel without TMA, 3 = TMA-staged
 * fused kernel (persistent, two stages when they fit), 4 = TMA-staged fused
 * kernel with one stage, 5 = split velocity/stress kernel pair (one tile
 * per CTA; in place, TTI with memory variables and CPML psi ping-ponging
 * through the plan), 6 = the ISO/VTI split pair as persistent
 * TMA-pipelined kernels,
 * 7 = streaming kernel (FP32 ISO/VTI: persistent CTAs march down 128-column
 * strips with TMA row rings, one launch per step),
 * 8 = the split pair of 5 with its velocity pass reading the stress taps
 * straight through L1 instead of TMA boxes, 9 = the split pair's tiles
 * time-blocked: one persistent kernel per call runs sweeps of several
 * steps as a wavefront over 8-row bands, so the next steps re-read a
 * band's state from L2 (ISO/VTI, imaging or no free surface, not
 * VI_F32C; depth and lag set by vi_plan_set_wave; results bitwise equal
 * to variant 5).
 * Variants 3-9 return VI_ERR_ARG when not eligible.
 * VI_F32C plans (split pair only) keep the stresses' rounding residues as
 * plan state, continued across calls like the CPML memory: vi_plan_reset
 * zeroes them. */
int vi_step(vi_plan *plan, const vi_medium *med_dev, vi_fields *fields_dev,
            const vi_shot *shot, int32_t it0, int32_t nsteps,
            int32_t kernel_variant, void *stream);

/* Time blocking of kernel variant 9: sweeps of `depth` steps (0 = the
 * default, 4) with a lag of `lag` 8-row bands between consecutive passes
 * (0 = the default, 8; else 2 .. 64).  Deeper sweeps re-read more steps'
 * state from L2; a longer lag lets a pass's units find their inputs done
 * but keeps more bands in flight.  No counterpart in the reference, which
 * runs one launch per step (visco-kernels.jl:87-100). */
int vi_plan_set_wave(vi_plan *plan, int32_t depth, int32_t lag);

/* Same steps as vi_step with kernel_variant 1 (plain, in place), but it
 * allocates no device memory: its strain planes and source/receiver lists
 * live in one static device array of VI_NOALLOC_SCRATCH_BYTES per device
 * and process.  No counterpart in the reference.  For callers
 * that must not call cudaMalloc/cudaFree mid-run (a serving process sharing
 * the GPU, whose allocations would synchronize it; a fully reserved HBM
 * pool).  Limit: 6*nx*nz reals of the plan's precision plus the lists
 * (<= 256 sources; each of the three blocks rounded up to 256 bytes) must
 * fit in VI_NOALLOC_SCRATCH_BYTES, else VI_ERR_ARG.  Every call looks up
 * the array's address in the current context; the first call on a device
 * loads the module that holds it, so make that first call before any
 * stream capture.  With sources or receivers (nsrc > 0 or nrec > 0) the
 * call blocks the host thread until their lists are staged on the device.
 * Each call clears the strain planes first.  Calls overlapping in time on
 * one device race on the array: serialize them. */
#define VI_NOALLOC_SCRATCH_BYTES (24u * 1024u * 1024u)
int vi_step_noalloc(vi_plan *plan, const vi_medium *med_dev, vi_fields *fields_dev,
                    const vi_shot *shot, int32_t it0, int32_t nsteps, void *stream);

/* One whole forward solve with host buffers: uploads the medium and the
 * wavelets, runs nt steps from a zero state and downloads the traces and
 * (optionally) the final wavefields.  Synchronous.  The end-to-end form of
 * the time loop the reference leaves unwritten (call stack of
 * leapfrog_step!, visco-kernels.jl:87-100). */
int vi_forward_host(vi_plan *plan, const vi_medium *med_host,
                    int32_t nsrc, const vi_source *src, const void *wavelet_host,
                    int32_t nrec, const vi_receiver *rec, int32_t nt,
                    void *traces_host, vi_fields *final_host);

/* ---- batched shots ---------------------------------------------------- */
/* Many shots of different grids and step counts advancing together.  The
 * reference solves one problem per call (ViscoelasticProblem.jl:273-309)
 * and has no batch; this is the B200 form of running its time step for a
 * whole shot gather: each launch covers the tiles of every shot still
 * running (one fused launch, or the split velocity and stress launches,
 * per time step), and the sequence of launches is one CUDA graph.
 * Shots must share the medium kind, precision and nsls, and have nx % 4 == 0. */
typedef struct vi_batch vi_batch;
#define VI_BATCH_NO_GRAPH 1  /* launch step by step instead of one CUDA graph */
#define VI_BATCH_RETUNE 2    /* forget the cached kernel-form choice and retune */
int vi_batch_create(const vi_config *cfgs, int32_t nshots, vi_batch **out);
int vi_batch_destroy(vi_batch *batch);
/* Binds shot i: device medium and fields (borrowed until the batch is
 * destroyed or the shot re-bound), sources/receivers (host lists copied),
 * and its step count.  Shots start from the state in their fields. */
int vi_batch_set_shot(vi_batch *batch, int32_t i, const vi_medium *med_dev,
                      const vi_fields *fields_dev, const vi_shot *shot, int32_t nt);
/* Runs every shot to its step count on `stream` (asynchronous).  The first
 * run (or VI_BATCH_RETUNE) times the kernel forms on the bound shots for a
 * few steps, keeps the faster one for this problem class, and resets the
 * shots to rest (fields, memory variables and CPML memory zeroed) before
 * the run proper.  Every run zeroes the CPML memory first. */
int vi_batch_run(vi_batch *batch, int32_t flags, void *stream);
/* Synchronizes, reports the kernel form in use (4 per shot on 8
 * concurrent streams: each shot's own vi_step loop, shots side by side, 3
 * per shot one after the other, 2 split velocity/stress pair over all
 * shots' tiles, 1 two-stage persistent fused, 0 one-stage fused) and any
 * device-side wait failure (VI_ERR_TIMEOUT). */
int vi_batch_status(vi_batch *batch, void *stream, int32_t *kernel_form);

/* ---- misfit gradient (discrete adjoint) ------------------------------ */
/* The reference has no receivers, misfit, adjoint or gradient: its only
 * gradient path is a printed sketch (examples/energy_natural_gradient_example.jl:252-315)
 * around an optimizer (EnergyNaturalGradient.jl:239-321) that takes a
 * grad_fn.  This is that grad_fn for the leapfrog step:
 *   J = 1/2 sum_{t,r} (d - obs)^2 over the vx and vz traces,
 * d the traces of an nt-step run from rest with the shot's sources and
 * receivers, obs_dev the observed traces in the same layout
 * ([2][nrec][nt], plan precision).  grad_dev (8 planes of nx*nz, FP64) gets
 * dJ/d(rho, c11, c13, c15, c33, c35, c55, tau) in vi_medium's order; for
 * ISO media the c13 plane holds dJ/dlambda and the c55 plane dJ/dmu (the
 * others zero).  ISO, VTI and TTI media (TTI fills all eight planes: the
 * tilted law of custom_solver/Model.jl:59-108 transposed, its 4-point means
 * of C15/C35/C55 and of the effective rates and the surface relation with
 * C35 included); the H-AFDA surface returns VI_ERR_ARG.  The adjoint
 * is the exact transpose of the plain in-place step (kernel variant 1),
 * with the state checkpointed every checkpoint_every steps in the plan's
 * workspace and each segment recomputed; checkpoint_every <= 0 keeps every
 * state of the forward sweep in HBM when they fit in 60 % of the device's
 * memory and in what is free (nothing recomputed; 88 GB for a 1024 x 512,
 * 3000-step VTI FP32 shot), else checkpoints every ceil(sqrt(nt)) steps.
 * The result is bitwise the same for every interval.  accumulate != 0 adds into grad_dev
 * (shots summed), else grad_dev is overwritten.  *misfit_host = J (FP64).
 * The shot's traces_dev, if given with traces_nt >= nt, receives d.
 * Synchronous on `stream`. */
int vi_gradient(vi_plan *plan, const vi_medium *med_dev, const vi_shot *shot, int32_t nt,
                const void *obs_dev, int32_t checkpoint_every, int32_t accumulate,
                double *grad_dev, double *misfit_host, void *stream);
/* Chain rule from grad (as vi_gradient leaves it) to (vp, vs, rho, 1/Q)
 * planes: out4 = [dJ/dvp, dJ/dvs, dJ/drho at fixed velocities, dJ/d(1/Q)].
 * vp, vs, rho (and for VTI eps, delta; NULL means 0) are FP64 device
 * planes of np cells; the stiffnesses follow Models.jl:27-52 (ISO:
 * lambda = rho (vp^2 - 2 vs^2), mu = rho vs^2; VTI: Thomsen).  tau_scale =
 * d tau / d(1/Q) = N / Kbar of the Q fit (Models.jl:67). */
int vi_gradient_velocity(int32_t medium, int64_t np, const double *grad8, const double *vp,
                         const double *vs, const double *rho, const double *eps,
                         const double *delta, double tau_scale, double *out4, void *stream);
/* VTI: from the same grad planes to the Thomsen parameters at fixed vp,
 * vs, rho: out2 = [dJ/d(epsilon), dJ/d(delta)] (C11 = C33 (1 + 2 epsilon),
 * C13 from delta as in Models.jl:27-52; custom_solver/Model.jl:12-16
 * carries epsilon, delta, gamma).  gamma enters only SH motion, so dJ/dgamma
 * is zero in 2D P-SV and not written.  delta NULL means 0.  FP64 device
 * planes of np cells; asynchronous on `stream`. */
int vi_gradient_thomsen(int64_t np, const double *grad8, const double *vp, const double *vs,
                        const double *rho, const double *delta, double *out2, void *stream);

/* TTI: from the same grad planes to out7 = [dJ/dvp, dJ/dvs, dJ/drho,
 * dJ/d(1/Q), dJ/d(epsilon), dJ/d(delta), dJ/d(theta)] through the map of
 * vi_medium_from_velocity (Thomsen's VTI law, Models.jl:27-52 and
 * custom_solver/Model.jl:12-16, tilted by theta with the 2D Bond rotation);
 * dJ/drho at fixed velocities includes the buoyancy term.  eps, delta,
 * theta NULL mean 0.  gamma enters only SH motion: no 2D P-SV gradient.
 * FP64 device planes of np cells; asynchronous on `stream`. */
int vi_gradient_tti(int64_t np, const double *grad8, const double *vp, const double *vs, const double *rho,
                    const double *eps, const double *delta, const double *theta, double tau_scale,
                    double *out7, void *stream);

/* ---- medium parameterisation ------------------------------------------ */
/* Writes the medium planes the step reads from FP64 parameter planes of np
 * cells on the device: ISO rho, c13 = lambda = rho (vp^2 - 2 vs^2), c55 =
 * mu = rho vs^2; VTI rho, c11, c13, c33, c55 from Thomsen epsilon, delta
 * (Models.jl:27-52, custom_solver/Model.jl:12-16); TTI the VTI stiffness
 * tilted by theta (radians, symmetry axis from z towards x; 2D Bond
 * rotation) into c11, c13, c15, c33, c35, c55.  With q (the quality factor
 * plane) also tau = tau_scale / q, tau_scale = N / Kbar of the Q fit
 * (Models.jl:67).  eps, delta, theta NULL mean 0.  `out` names the device
 * planes to write, in `precision` (VI_F32 / VI_F64); those the medium kind
 * needs must be non-NULL.  Asynchronous on `stream`.  The reference does
 * this on the host before every solve. */
int vi_medium_from_velocity(int32_t medium, int32_t precision, int64_t np, const double *vp,
                            const double *vs, const double *rho, const double *eps,
                            const double *delta, const double *theta, const double *q,
                            double tau_scale, const vi_medium *out, void *stream);

/* ---- request server ---------------------------------------------------- */
/* Forward solves and misfit gradients submitted from any host thread and
 * run by `lanes` worker threads, each resident request on its own stream.
 * The reference solves one problem per call and has no server
 * (ViscoelasticProblem.jl:273-309).  Admission against an HBM budget;
 * requests join and leave between slices of slice_steps steps (continuous
 * batching), each idle lane taking the next slice of the idle resident
 * request with the least remaining work (cells x steps left), so short
 * requests preempt long ones; gradient requests run whole.
 * Every request has its own plan: its results equal a vi_forward_host /
 * vi_gradient call on the same inputs, whatever else is resident. */
typedef struct vi_server vi_server;
typedef struct vi_serve_config {
  int32_t device;
  int32_t slice_steps;      /* steps per scheduling slice (<= 0: 1024) */
  int32_t max_active;       /* requests resident at once (<= 0: 64) */
  int32_t policy;           /* VI_SERVE_SHORTEST_FIRST or VI_SERVE_ROUND_ROBIN */
  int64_t hbm_budget_bytes; /* device bytes the requests may hold (<= 0: 150 GB) */
  int32_t lanes;            /* worker threads, i.e. requests advancing on the
                               device at once, each on its own stream
                               (<= 0: 2; at most 16); 1 = one at a time */
  int32_t pad_;
} vi_serve_config;

#define VI_SERVE_SHORTEST_FIRST 0 /* each slice to the request with the least work left */
#define VI_SERVE_ROUND_ROBIN 1    /* every resident request advances one slice per round */
#define VI_REQ_FORWARD 0
#define VI_REQ_GRADIENT 1
#define VI_REQ_QUEUED 0
#define VI_REQ_RUNNING 1
#define VI_REQ_DONE 2
#define VI_REQ_FAILED 3

/* One request.  Host buffers are borrowed until the request is done or
 * failed: medium planes (plan precision), wavelets (nsrc rows of
 * wavelet_nt), the traces out ([2][nrec][nt]); for a gradient also the
 * observed traces in, the FP64 gradient out ([8][nz][nx], vi_gradient's
 * planes) and the misfit out.  Source and receiver lists are copied at
 * submit. */
typedef struct vi_request {
  int32_t kind;             /* VI_REQ_FORWARD / VI_REQ_GRADIENT */
  int32_t nt;
  vi_config cfg;
  vi_medium medium_host;
  int32_t nsrc, wavelet_nt;
  const vi_source *src_host;
  const void *wavelet_host;
  int32_t nrec, pad_;
  const vi_receiver *rec_host;
  void *traces_host;
  const void *obs_host;
  double *grad_host;
  double *misfit_host;
} vi_request;

int vi_serve_start(const vi_serve_config *cfg, vi_server **out);
/* Queues a request; VI_ERR_BUDGET when it could never fit the budget. */
int vi_serve_submit(vi_server *server, const vi_request *req, uint64_t *ticket);
/* Non-blocking: state (VI_REQ_*) and the latency so far or, when done,
 * from submit to results in the host buffers; returns the request's error
 * when it failed. */
int vi_serve_poll(vi_server *server, uint64_t ticket, int32_t *state, double *latency_ms);
/* Blocks until the request is done or failed, or timeout_s (< 0: no limit). */
int vi_serve_wait(vi_server *server, uint64_t ticket, double timeout_s, int32_t *state);
/* Finishes every queued and resident request, then frees the server. */
int vi_serve_stop(vi_server *server);

/* ---- staggered derivatives (diff-funcs.jl:3-32) ----------------------- */
/* du = D(u) over the update region for one plane (device pointers, plan
 * precision).  op: 0 = ddxp, 1 = ddxm, 2 = ddzp, 3 = ddzm.  h is the grid
 * spacing along the operator's axis. */
int vi_diff(int32_t precision, int32_t op, const void *u_dev, void *du_dev,
            int32_t nx, int32_t nz, double h, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* VISCO_B200_H */
