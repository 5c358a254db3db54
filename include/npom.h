/*
 * npom.h -- C ABI of the B200 (sm_100a) NeuralPOM physical time step.
 *
 * The library advances the state of one POM core (explicit mode-split or
 * semi-implicit free surface) by whole internal steps, on one GPU, on the
 * caller's CUDA stream.  All memory is owned by the caller: every field is a
 * C-contiguous float32 device array laid out like the reference core's
 * tensors -- 3-D fields (im, jm, kb) with the sigma level k fastest, 2-D
 * fields (im, jm), 1-D fields (kb) -- and the workspace buffers are caller
 * allocated too.  No entry point allocates or frees device memory.
 *
 * Reference interfaces replaced (paths relative to src/neuralpom/):
 *   npom_step_explicit  <- cores/explicit/time_loop.py:20 TimeLoopMixin.run_time_loop
 *   npom_step_implicit  <- cores/implicit_p0_fixed/time_loop.py:38 TimeLoopMixin.run_time_loop
 *   npom_proft          <- cores/explicit/tracers.py:890 TracersMixin.proft
 *                          (twin: cores/implicit_p0_fixed/strict_vertical.py:103 _reference)
 *   npom_pcg_solve      <- cores/implicit_p0_fixed/core.py:775 POM2K_Core.solve_implicit_eta_cg
 *   npom_run_phase      <- the individual operators of the two time loops
 *                          (advct baroclinic.py:14, baropg momentum.py:543,
 *                          advave baroclinic.py:262, vertvl baroclinic.py:930,
 *                          advq tracers.py:14, profq tracers.py:158,
 *                          advt1 tracers.py:433, dens momentum.py:467,
 *                          advu/advv momentum.py:14/133, profu/profv
 *                          momentum.py:250/359, bcond baroclinic.py:496 and
 *                          implicit_p0_fixed/boundary/closed_basin.py:27)
 *
 * Error model: every entry point returns an npom_status; device-detected
 * conditions (velocity above vmaxl, a barrier that timed out, PCG at
 * max_iter) are OR-ed into a device status word that npom_status_read
 * returns.
 */
#ifndef NPOM_H
#define NPOM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ */
/* Fields: one device pointer per reference tensor attribute.          */
/* ------------------------------------------------------------------ */
#define NPOM_FIELD_LIST(X)                                                   \
  /* static 2-D geometry */                                                  \
  X(h) X(dx) X(dy) X(art) X(aru) X(arv) X(fsm) X(dum) X(dvm) X(cor) X(cbc)   \
  X(north_e)                                                                 \
  /* 1-D vertical grid (kb) */                                               \
  X(z) X(zz) X(dz) X(dzz)                                                    \
  /* open-boundary arrays of the explicit core (jm / im / (jm,kb) / (im,kb)) */\
  X(ele) X(elw) X(eln) X(els) X(uabe) X(uabw) X(vabn) X(vabs)                \
  X(tbe) X(sbe) X(tbw) X(sbw) X(tbn) X(sbn) X(tbs) X(sbs)                    \
  /* 3-D state */                                                            \
  X(u) X(ub) X(uf) X(v) X(vb) X(vf) X(w) X(t) X(tb) X(s) X(sb) X(rho)        \
  X(rmean) X(tclim) X(sclim) X(q2) X(q2b) X(q2l) X(q2lb) X(km) X(kh) X(kq)   \
  X(l) X(aam) X(advx) X(advy) X(drhox) X(drhoy) X(curv)                      \
  /* 2-D state */                                                            \
  X(el) X(elb) X(elf) X(et) X(etb) X(etf) X(d) X(dt) X(ua) X(uab) X(uaf)     \
  X(va) X(vab) X(vaf) X(utf) X(utb) X(vtf) X(vtb) X(egf) X(egb) X(adx2d)     \
  X(ady2d) X(drx2d) X(dry2d) X(aam2d) X(advua) X(advva) X(fluxua) X(fluxva)  \
  X(wubot) X(wvbot) X(wusurf) X(wvsurf) X(wtsurf) X(wssurf) X(vfluxf)        \
  X(vfluxb) X(swrad) X(e_atmos) X(tps) X(tsurf) X(ssurf)

typedef enum npom_field {
#define NPOM_X_ENUM(n) NPOM_F_##n,
  NPOM_FIELD_LIST(NPOM_X_ENUM)
#undef NPOM_X_ENUM
  NPOM_NFIELDS
} npom_field;

/* Workspace buffers (caller-allocated device memory). */
#define NPOM_WS_LIST(X)                                                      \
  /* float32, im*jm each */                                                  \
  X(us) X(vs) X(den_u) X(den_v) X(d_baro) X(rhs) X(x) X(r) X(p) X(zv) X(ap)  \
  X(ce) X(cw) X(cn) X(cs) X(inv_art) X(diag)                                 \
  /* float32: DST-I matrices (ni*ni, nj*nj), inverse eigenvalues and two     \
     transform buffers (ni*nj each) of the spectral preconditioner */        \
  X(sx) X(sy) X(inv_eigs) X(t1) X(t2)

typedef enum npom_wsbuf {
#define NPOM_X_ENUM(n) NPOM_W_##n,
  NPOM_WS_LIST(NPOM_X_ENUM)
#undef NPOM_X_ENUM
  NPOM_NWS
} npom_wsbuf;

typedef struct npom_workspace {
  float *buf[NPOM_NWS];
  double *partials;        /* >= 4 * NPOM_MAX_COOP_BLOCKS doubles          */
  unsigned int *sync;      /* >= 4 unsigned ints, zero before first use    */
  unsigned int *status;    /* >= 1 unsigned int: OR of NPOM_ERR_* bits     */
  int *cg_iters;           /* >= nsteps ints: PCG iterations of each step  */
  float *mp3d;             /* nadv 2 only (else may be null): >= 12 *     */
                           /* im*jm*kb floats of MPDATA scratch            */
  float *tide;             /* NPOM_OBC_COASTAL only (else may be null):    */
                           /* 3 planes of im*jm: 1 at tide cells, their   */
                           /* amplitude (m) and phase (degrees)           */
  double *robin;           /* NPOM_OBC_SEAMOUNT on the semi-implicit core  */
                           /* only (else may be null): 5 * im*jm doubles  */
                           /* of the FP64 Robin solve                     */
} npom_workspace;

#define NPOM_MAX_COOP_BLOCKS 1024
#define NPOM_MAX_BATCH 64  /* members of one npom_step_batch call         */

/* ------------------------------------------------------------------ */
/* Scalar settings (the Python attributes of the reference BaseCore).  */
/* ------------------------------------------------------------------ */
/* Launch shapes of the step (the autotuner's search space).  Every form
 * computes the same values: bit for bit, except the cooperative-grid PCG,
 * whose FP64 dot products are summed over its blocks (equal to rounding).
 * 0 in every field keeps the library's rules; the NPOM_* environment
 * switches (comparisons) take precedence over these fields.  No
 * counterpart in the reference, whose PyTorch step has no launch shapes. */
typedef struct npom_tuning {
  int32_t a1_form;             /* A1 (advct): 0 rule (tiles from 16384 cells), 1 points, 2 flux-once tiles */
  int32_t b5_form;             /* B5 (advt1): the same choices                                           */
  int32_t tile_blocks_per_sm;  /* A1/B5 tiles: rows per tile for about this many blocks per SM (0: 16) */
  int32_t column_form;         /* kb = 16 column phases: 0 rule (lanes; PROFT one thread per column
                                  from 16384 columns), 1 lanes everywhere, 2 one thread per column     */
  int32_t subcycle_form;       /* explicit subcycle: 0 rule, 1 one cluster (up to 16384 cells),
                                  2 grid barrier, 3 one launch per substep phase                        */
  int32_t pcg_form;            /* 0 rule (cluster: bulk, replicated, pushed; else cooperative grid),
                                  1 pushed-residual cluster, 2 replicated cluster with cluster
                                  barriers, 3 cooperative grid                                          */
  int32_t pcg_ctas;            /* cluster PCG: 0 rule (8 CTAs first), 16 (16 CTAs first)               */
  int32_t batch_pcg_blocks;    /* npom_step_batch: cap on each member's cooperative-PCG blocks (0 none) */
  int32_t reserved[2];
} npom_tuning;

typedef struct npom_params {
  int32_t device;          /* CUDA device ordinal the pointers live on     */
  int32_t im, jm, kb;
  int32_t core;            /* NPOM_CORE_EXPLICIT / NPOM_CORE_IMPLICIT      */
  int32_t isplit, ispadv, nbct, nbcs, ntp, mode, nadv;
  int32_t eta_max_iter;
  int32_t eta_precond;     /* NPOM_PRECOND_JACOBI / NPOM_PRECOND_SPECTRAL  */
  int32_t wind_forcing;    /* implicit: rewrite wusurf/wvsurf every step   */
  int32_t has_vmix;        /* clamp kh/km/kq to [0, vmix]                  */
  int32_t lramp;
  double dti, dte, dti2, dte2, ispi, isp2i;
  double alpha, smoth, horcon, grav, umol, tprni, small, kappa, rhoref;
  double tbias, sbias, vmaxl, hmax, rfe, rfw, rfn, rfs, aam_min, pi;
  double eta_tol, eta_rel_tol, barotropic_shapiro, tracer_shapiro;
  double velocity_shapiro, wind_tau0, vmix;
  double period;           /* inertial period in days (ramp = time/period) */
  double inverse_scale;    /* spectral preconditioner: 4 (ni+1)(nj+1)      */
  double sw;               /* MPDATA antidiffusion weight (nadv 2)         */
  int32_t nitera;          /* MPDATA iterations (nadv 2)                   */
  int32_t profq_form;      /* NPOM_PROFQ_PRODUCTION or NPOM_PROFQ_POM08    */
  int32_t obc_form;        /* NPOM_OBC_NATIVE, _SEAMOUNT or _COASTAL       */
  npom_tuning tuning;      /* launch shapes (all zero: the library's rules) */
  double zsh;              /* POM08-WAD profq: roughness added to the mixing length (m) */
  int32_t periodic_x;      /* 1: periodic in x (implicit core; see below)  */
} npom_params;

/* PROFQ forms.  PRODUCTION: the cores' own operator (explicit/tracers.py:158,
 * implicit_p0_fixed/tracers.py:156).  POM08: the POM08-WAD closure of the
 * reference's case policies (cores/case_adapters/fortran_compat.py:26-147,
 * installed by dg_policy.py, coastal_compat.py, jzb_compat.py): forward
 * only, as in the reference, which validates it for forward comparisons. */
enum { NPOM_PROFQ_PRODUCTION = 0, NPOM_PROFQ_POM08 = 1 };

/* Boundary policy (obc_form).  NATIVE: the core's own bcond (closed walls,
 * or the explicit core's Flather/upstream open boundary).  SEAMOUNT: the
 * explicit core with the seamount case policy's boundary
 * (cores/case_adapters/seamount_boundary.py:9-43): η ghost copies and
 * characteristic radiation on the east and west edges, Orlanski radiation
 * of u and of T/S (with the exterior profile on inflow), 1e-10 turbulence
 * edges; the north and south edges are walls.  Forward only (the reference
 * refuses gradients through its case policies). */
enum { NPOM_OBC_NATIVE = 0, NPOM_OBC_SEAMOUNT = 1, NPOM_OBC_COASTAL = 2, NPOM_OBC_JZB = 3 };
/* SEAMOUNT on the semi-implicit core (barotropic_shapiro 0; the Robin
 * solve's FP64 planes in npom_workspace.robin): the policy's predictor
 * (the incident transport on the east and west edges), its free-surface
 * solve -- Picard iterations on the boundary depth around a CG with the
 * characteristic (Robin) flux of the east and west edges in the operator,
 * in FP64 (its 1e-11 m Picard test is a float64 criterion) -- its
 * corrector with the old and new face depths and the edge radiation, the
 * body continuity that rewrites utf, vtf and etf after the filter
 * (seamount_boundary.py:45-147), and its bcond 1 and 3-6. */
/* COASTAL and JZB on the semi-implicit core (barotropic_shapiro 0): the
 * policy's step copy (the old depth in the corrector's pressure-gradient
 * transport, cbc after the filter), its bcond 2 on u* and on the corrected
 * transports, its own free-surface solve -- CG on the interior sea cells
 * that are not tide cells, weighted by the cell areas, for the part beyond
 * the tidal lift (coastal_boundary.py:31-54, jzb_boundary.py:150-197) --
 * and the explicit step copy's bcond 3-6. */
/* JZB: the explicit core with the Jiaozhou Bay tide policy
 * (cores/case_adapters/jzb_boundary.py, jzb_compat.py and the coastal
 * policy's step copies): the coastal policy's machinery (tide planes, no
 * 1e-8 in the bottom-drag speed, cbc after the substeps) with the bay's
 * M2 speed, the tide times fsm at its cells and the edges copying the
 * adjacent cell (bcond 1); Sommerfeld radiation of the transports on all
 * four edges (bcond 2) and of the internal velocities (bcond 3), both
 * ramped; cbc from depths >= 0.05 m with z0b 0.01 m.  Forward only. */
/* COASTAL: the explicit core with the coastal tide policy
 * (cores/case_adapters/coastal_boundary.py:9-30, coastal_compat.py and the
 * policy's step copies): the tidal elevation
 * amp cos(w t - phase) imposed at the cells the workspace's tide planes
 * flag, at every external substep; characteristic radiation on all four
 * edges with the total depth d; the bcond 3 blend weight from d; no 1e-8
 * in the bottom-drag speed; cbc from the new depth after the external
 * substeps (zsh 0.01 m, z0b 0.005 m, clipped to [0.0025, 1]).  Forward
 * only. */

/* Periodic x (periodic_x = 1).  No counterpart in the reference, whose
 * only lateral boundaries are walls and open edges (its cores zero or
 * radiate the ring).  The semi-implicit core only, with native boundaries,
 * nadv 1 and the Jacobi preconditioner (the DST-I assumes walls in x).
 * Columns 0, 1 and im-2, im-1 are halo copies of im-4, im-3 and 2, 3:
 * the unique columns are 2..im-3 (period im-4), walls stay on the j
 * edges.  After every phase of the step each plane of the state gets the
 * halo copy, and the free-surface solve's unknowns are the unique columns
 * with the operator's x neighbours wrapped.  Two halo columns because the
 * reference's operators compute some intermediates only from column 1 or
 * 2 on; with them every unique column is computed exactly as an interior
 * column of a wider basin (the step is translation-equivariant in x).
 * Forward only: the step adjoints and npom_step_batch refuse it. */

enum { NPOM_CORE_EXPLICIT = 0, NPOM_CORE_IMPLICIT = 1 };
enum { NPOM_PRECOND_JACOBI = 0, NPOM_PRECOND_SPECTRAL = 1 };

/* Return codes. */
typedef enum npom_status {
  NPOM_OK = 0,
  NPOM_ERR_ARG = 1,        /* bad argument (null pointer, size, kb)        */
  NPOM_ERR_CUDA = 2,       /* a CUDA runtime call failed                   */
  NPOM_ERR_DEVICE = 3,     /* the device status word is non-zero           */
  NPOM_ERR_TOO_LARGE = 4   /* grid above NPOM_STATIC_MAX_CELLS (static)    */
} npom_status;

/* Device status bits. */
#define NPOM_DEV_VMAX      0x1u  /* |vaf| > vmaxl in an external step     */
#define NPOM_DEV_TIMEOUT   0x2u  /* a grid barrier wait ran out            */
#define NPOM_DEV_PCG_MAXIT 0x4u  /* PCG reached eta_max_iter               */
#define NPOM_DEV_NONFINITE 0x8u  /* a non-finite elevation was produced    */

/* Per-call clock: the reference's time/time0/iint bookkeeping. */
typedef struct npom_clock {
  double time0;            /* clock at the start of the call (days)        */
  int32_t first_iint;      /* iint of the first step (1 for a fresh call)  */
  int32_t nsteps;
} npom_clock;

/* Library identity and layout checks (used by the host bindings). */
int npom_abi_version(void);
int npom_field_count(void);
const char *npom_field_name(int index);
int npom_ws_count(void);
const char *npom_ws_name(int index);
size_t npom_params_size(void);
size_t npom_workspace_struct_size(void);

/* Advance nsteps internal steps of the explicit mode-split core. */
npom_status npom_step_explicit(const npom_params *p, float *const *fields,
                               const npom_workspace *ws, const npom_clock *clk,
                               void *stream);

/* Advance nsteps internal steps of the semi-implicit free-surface core. */
npom_status npom_step_implicit(const npom_params *p, float *const *fields,
                               const npom_workspace *ws, const npom_clock *clk,
                               void *stream);

/* Advance nsteps internal steps of nmembers members of ONE core (each with
 * its own grid size, state and workspace) over the same clock: every phase
 * of the step is one launch over all members, and the step is replayed as
 * one CUDA graph.  Members must share core, kb, isplit, ispadv, mode, nadv,
 * nitera and device.  Each member computes what npom_step_explicit /
 * npom_step_implicit computes for it alone (bitwise, except the semi-
 * implicit members whose PCG runs in the cooperative form, whose FP64 dot
 * products are summed over a different block count: equal to rounding).
 * Replaces the reference's per-member loop over run_time_loop
 * (cores/explicit/time_loop.py:20, cores/implicit_p0_fixed/time_loop.py:38)
 * for an ensemble; the reference's only batched GPU code is its batched
 * 5-point elliptic operator (cores/implicit_p0_fixed/triton_kernels.py:104),
 * one operator, not a step. */
npom_status npom_step_batch(int32_t nmembers, const npom_params *const *params,
                            float *const *const *fields,
                            const npom_workspace *const *ws,
                            const npom_clock *clk, void *stream);

/* Kernels the last npom_step_batch call of this process launched (graph
 * replays count their kernel nodes); for launch accounting. */
long long npom_batch_launches(void);

/* Run one named phase of a step on the current state (operator tests). */
npom_status npom_run_phase(const npom_params *p, float *const *fields,
                           const npom_workspace *ws, int phase, double ramp,
                           void *stream);
int npom_phase_count(void);
const char *npom_phase_name(int index);

/* Implicit vertical diffusion of ncol tracer columns of kb levels
 * (kb <= 64), boundary type nbc 1-4, exactly like TracersMixin.proft:
 * f_out may alias f_in; dh_out receives h + etf. */
npom_status npom_proft(int ncol, int kb, const float *f_in, const float *wfsurf,
                       const float *fsurf, int nbc, const float *h,
                       const float *etf, double dti2, const float *dz,
                       const float *dzz, const float *swrad, int ntp,
                       const float *kh, double umol, const float *z,
                       float *f_out, float *dh_out, void *stream);

/* One PCG free-surface solve: fields[elf] holds the initial guess on entry
 * and the solution on exit (before the Shapiro filter / boundary); rhs is
 * read from ws->buf[NPOM_W_rhs].  Iterations go to ws->cg_iters[0].  The
 * native boundary only (obc_form 0; a case policy's solve is part of its
 * step), as for npom_pcg_adjoint and npom_pcg_solve_static. */
npom_status npom_pcg_solve(const npom_params *p, float *const *fields,
                           const npom_workspace *ws, void *stream);

/* Backward of the free-surface solve x = A(d)^-1 rhs for the cotangent
 * grad_x = dJ/dx (all arrays im*jm device float32):
 *   grad_rhs = dJ/drhs = A^-T grad_x, solved as M A^-1 M^-1 with relative
 *              cell areas, the right-hand side scaled by max|.| clamped to 1
 *              and the absolute PCG tolerance by the same factor, from a
 *              zero guess (ws->cg_iters[0] receives the iterations);
 *   grad_d   = dJ/dd, the transposed depth stencil of the operator at the
 *              forward solution x.
 * d2d is the depth the forward solve used.  The rhs scale stays on the
 * device; the call synchronises its stream once, to check the cotangent
 * before the solve, so it is not capturable.
 * Replaces cores/implicit_p0_fixed/core.py:24 _ImplicitEtaSolveFunction
 * (backward :46-59, _solve_implicit_eta_adjoint :231-252,
 * _apply_elliptic_operator_depth_adjoint :645-675).  A non-finite
 * cotangent sets NPOM_DEV_NONFINITE and returns NPOM_ERR_DEVICE. */
npom_status npom_pcg_adjoint(const npom_params *p, float *const *fields,
                             const npom_workspace *ws, const float *grad_x,
                             const float *x, const float *d2d, float *grad_rhs,
                             float *grad_d, void *stream);

/* Largest im*jm that npom_pcg_solve_static accepts. */
#define NPOM_STATIC_MAX_CELLS 32768

/* No-allocation variant of npom_pcg_solve.  This entry point has no
 * counterpart in the reference (whose solve allocates its work tensors
 * with torch).  It is for callers that cannot allocate device memory: a
 * host ocean model that owns only its state arrays and has no device
 * allocator of its own, or a real-time loop that forbids allocation once
 * it has started.  Same solve, same kernels and same result as
 * npom_pcg_solve: fields[elf] holds the initial guess on entry and the
 * solution on exit; rhs (im*jm) is read, not modified; sx (ni*ni),
 * sy (nj*nj) and inv_eigs (ni*nj) are the spectral operator inputs
 * (unused, may be null, with the Jacobi preconditioner).
 *   - Scratch: one file-scope __device__ array of the library (~2 MB:
 *     15 planes of NPOM_STATIC_MAX_CELLS floats, 4096 doubles, 8 words),
 *     one copy per device.  Nothing is allocated or freed.
 *   - Limit: im*jm > NPOM_STATIC_MAX_CELLS returns NPOM_ERR_TOO_LARGE.
 *   - Zeroing: the caller zeroes nothing; the call clears the scratch's
 *     control words itself, and the solve writes every other scratch word
 *     before reading it.
 *   - First call per device: looks up the scratch address with
 *     cudaGetSymbolAddress (device p->device current); make it before any
 *     stream capture.  The address is kept per device together with the
 *     calling thread's current context, and looked up again when a call
 *     comes from another context of that device (after cudaDeviceReset,
 *     or under a context the caller made current).
 *   - Concurrency: calls on one device share the scratch; overlapping
 *     calls (other streams, other threads) race.  Serialise them.
 *   - Outputs: iters_out and status_out (device int / unsigned int, may be
 *     null) receive the iteration count and the device status bits.  */
npom_status npom_pcg_solve_static(const npom_params *p, float *const *fields,
                                  const float *rhs, const float *sx,
                                  const float *sy, const float *inv_eigs,
                                  int *iters_out, unsigned int *status_out,
                                  void *stream);

/* ------------------------------------------------------------------ */
/* Adjoint of one explicit internal step (reverse mode).               */
/* The reference differentiates its step with torch autograd           */
/* (explicit/time_loop.py:20-709 under SparsePhysics.advance with      */
/* differentiable=True, sparse_physics.py:91-149); this is the         */
/* hand-written vector-Jacobian product of the same step.              */
/* ------------------------------------------------------------------ */
typedef struct npom_adjoint_ws {
  float *lam[NPOM_NFIELDS];  /* one array per field, sized like it      */
  float *save;               /* >= npom_adjoint_save_floats(p) floats   */
  size_t save_floats;        /* capacity of save                        */
  const float *pcg_x;        /* semi-implicit core, may be NULL: the raw */
                             /* solution of this step's free-surface    */
                             /* solve (the workspace plane "x" after     */
                             /* the forward npom_step_implicit call of   */
                             /* the step), so the recomputation replays  */
                             /* it instead of solving again             */
} npom_adjoint_ws;

/* Size of the per-step save area (floats) for these settings. */
size_t npom_adjoint_save_floats(const npom_params *p);

/* Differentiates the internal step clk->first_iint (clk->nsteps must be
 * 1).  fields: the state at the START of that step (a checkpoint the
 * caller kept); it is used as scratch and holds the start state again on
 * return, apart from the zero surface-forcing fields.  grads[f]: on entry
 * the cotangent of field f after the step, on exit the cotangent of f
 * before it (vector-Jacobian product, accumulated in place).  Geometry,
 * forcing and open-boundary arrays are constants.  Supported settings:
 * explicit core, mode 3, nadv 1 or 2 (MPDATA), nbct/nbcs 1 or 3, the
 * production PROFQ; else NPOM_ERR_ARG.
 * The caller's save area also holds the step's scratch:
 * npom_adjoint_save_floats includes it. */
npom_status npom_step_explicit_adjoint(const npom_params *p, float *const *fields,
                                       const npom_workspace *ws,
                                       const npom_clock *clk, float *const *grads,
                                       const npom_adjoint_ws *aws, void *stream);

/* The same for the semi-implicit step (implicit_p0_fixed/time_loop.py:
 * 38-688 under torch autograd; the free-surface solve differentiates as
 * _ImplicitEtaSolveFunction, core.py:24-59).  Supported settings: mode 3,
 * nadv 1, nbct/nbcs 1 or 3, zero barotropic and tracer Shapiro filters.
 * No host synchronisation: the solve's rhs scale stays on the device, and
 * a non-finite cotangent propagates into the gradients as it does under
 * the reference's autograd.  Both step adjoints are replayed from a cached
 * CUDA graph per (pointers, constants, ramp) after their first call. */
npom_status npom_step_implicit_adjoint(const npom_params *p, float *const *fields,
                                       const npom_workspace *ws,
                                       const npom_clock *clk, float *const *grads,
                                       const npom_adjoint_ws *aws, void *stream);

/* ------------------------------------------------------------------ */
/* Operators of the corrector coupling (hybrid/sparse_coupling.py:10-82) */
/* and the cores' dens()/baropg() methods.  fields supplies geometry    */
/* (h, zz, fsm, dx, dy, dt, dum, dvm) and, for DENS, the ghost level of */
/* rho; arrays are (im, jm, kb), k fastest.                            */
/* ------------------------------------------------------------------ */

/* explicit/momentum.py:467-541: rho_out = DENS(t, s) on levels < kb-1,
 * the ghost level copied from fields[rho]. */
npom_status npom_dens(const npom_params *p, float *const *fields, const float *t,
                      const float *s, float *rho_out, void *stream);
/* Its vector-Jacobian product: grad_t, grad_s (levels < kb-1) and
 * grad_rho_in (the ghost level) from grad_rho; all outputs written. */
npom_status npom_dens_adjoint(const npom_params *p, float *const *fields,
                              const float *t, const float *s, const float *grad_rho,
                              float *grad_t, float *grad_s, float *grad_rho_in,
                              void *stream);
/* explicit/momentum.py:543-700 (the ramp passed in): drhox/drhoy from
 * rho - rmean; rho_out = (rho - rmean) + rmean, the method's round trip. */
npom_status npom_baropg(const npom_params *p, float *const *fields, const float *rho,
                        const float *rmean, double ramp, float *rho_out, float *drhox,
                        float *drhoy, void *stream);
/* Its vector-Jacobian product, ACCUMULATED into grad_rho and grad_dt
 * (d/d rmean = -d/d rho; the round trip has derivative one). */
npom_status npom_baropg_adjoint(const npom_params *p, float *const *fields,
                                const float *rho, const float *rmean, double ramp,
                                const float *grad_drhox, const float *grad_drhoy,
                                float *grad_rho, float *grad_dt, void *stream);

/* Reads (and with clear != 0 zeroes) the device status word; blocks on
 * the stream. */
npom_status npom_status_read(const npom_workspace *ws, int clear,
                             unsigned int *out_bits, void *stream);

/* Failure-path diagnostic (no reference counterpart): runs one of the
 * library's bounded waits on a condition that nothing satisfies, so that
 * it runs out the way a lost block or a lost peer CTA would make it:
 *   which = 0  the grid barrier of the cooperative kernels (one block of a
 *              two-block grid; gives up after 2 s),
 *   which = 1  the mbarrier wait of the cluster PCG's bulk exchanges (its
 *              own arrival, with bytes that never come; 0.5 s).
 * The wait records NPOM_DEV_TIMEOUT in ws's status word and the kernel
 * returns; the context stays usable.  Clears ws's barrier words first. */
npom_status npom_wait_selftest(int which, const npom_workspace *ws, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* NPOM_H */
