/*
 * nrqcd_b200 — C ABI of the B200 implementation of the two per-timestep hot
 * paths of the NRQCD + classical-statistical SU(3) simulation
 * (alexanderlehmann/NRQCD, Fortran 2008):
 *
 *   1. the SU(3) leapfrog of the gauge field      (GaugeConfiguration%Update)
 *   2. the NRQCD Crank-Nicolson propagator step   (NRQCDField%Update)
 *
 * plus the observables those paths are checked with.  Every entry point is a
 * plain C function over plain pointers and sizes so that the reference's
 * Fortran can bind it with ISO_C_BINDING; each declaration names the
 * reference procedure (file:line, paths within the reference project) whose
 * call site it replaces.
 *
 * Host array layouts are the reference's Fortran arrays (column-major) with
 * the memory index slowest; complex numbers are interleaved (re, im)
 * doubles, i.e. Fortran complex(c_double_complex):
 *   links(3,3,3,V)  : ((site*3 + dir)*3 + col)*3 + row      (complex)
 *   efield(8,3,V)   : (site*3 + dir)*8 + a                  (real)
 *   prop(6,6,V)     : (site*6 + col)*6 + row                (complex)
 * site = lattice index - 1 = x + Nx*(y + Ny*z) (src/lattice.f90:883-898) —
 * the single-rank memory order of the reference.
 *
 * All calls of one context are ordered on that context's CUDA stream.  Calls
 * that return host scalars synchronise; update calls may return before the
 * device work ends.  Calls are not re-entrant per context.  Every call
 * returns an nrq_status; nonzero codes carry a message via nrq_last_error.
 */
#ifndef NRQCD_B200_H
#define NRQCD_B200_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  NRQ_OK = 0,
  NRQ_ERR_NOT_INITIALISED = 1,     /* mirrors src/nrqcd.f90:206-211          */
  NRQ_ERR_ALREADY_INITIALISED = 2, /* mirrors src/nrqcd.f90:180-181          */
  NRQ_ERR_BAD_ARG = 3,
  NRQ_ERR_CUDA = 4,
  NRQ_ERR_NOT_CONVERGED = 5,       /* the reference never checks KSP convergence */
  NRQ_ERR_TIMEOUT = 6,
  NRQ_ERR_NONFINITE = 7,
  NRQ_ERR_NO_DEVICE = 8,
  NRQ_ERR_OOM = 9,
  NRQ_ERR_CAPACITY = 10            /* lattice larger than a fixed scratch array */
} nrq_status;

typedef struct nrq_ctx nrq_ctx;     /* lattice + device + stream          */
typedef struct nrq_gauge nrq_gauge; /* type(GaugeConfiguration)           */
typedef struct nrq_heavy nrq_heavy; /* type(NRQCDField)                   */
typedef struct nrq_cn nrq_cn;       /* module state of src/nrqcd.f90:120-158 */

typedef struct {
  int64_t iterations;      /* Krylov iterations of the last update (max over columns) */
  int64_t matvecs;         /* stencil applications (12 columns each)  */
  int64_t vector_streams;  /* 12-column vector passes (read or write)  */
  double max_rel_residual; /* max over the 12 columns of ||b-Ax||/||b||: the true
                              residual, or the recursive one where the plain
                              solve ended on it (nrq_cn_true_residual_info) */
  int converged;           /* 1 when every column reached the tolerance */
  double initial_rel_residual; /* the same maximum for the starting guess
                                  (0 where a batch step did not read it back) */
} nrq_cn_stats;

/* ---- context: replaces lattice%InitModule (src/lattice.f90:124-228) and
 *      halocomm%InitModule (src/halocomm.f90:70-90); on one GPU the halo
 *      exchange becomes periodic indexing inside the kernels.               */
int nrq_init(const int64_t extents[3], const double spacings[4] /* a0, ax, ay, az */,
             int device, nrq_ctx **ctx);
int nrq_finalize(nrq_ctx *ctx);
const char *nrq_last_error(const nrq_ctx *ctx);
const char *nrq_status_string(int status);
int nrq_synchronize(nrq_ctx *ctx);
/* The CUDA stream (cudaStream_t) every kernel of this context runs on, so a
 * caller can order its own work or time with CUDA events on it.            */
void *nrq_cuda_stream(nrq_ctx *ctx);

/* Per-kernel-class timing with CUDA events recorded around every launch on
 * the context stream (off by default; enabling adds two event records per
 * launch).  Classes: 0 CN stencil (matvec), 1 CN vector update, 2 CN
 * scalar stages, 3 CN per-step gauge preparation, 4 leapfrog link update,
 * 5 leapfrog E update.  nrq_profile_read synchronises and returns, per
 * class, the launch count, summed device milliseconds and the algorithmic
 * HBM bytes those launches had to move (each field read or written once);
 * it then clears the counters.                                             */
enum { NRQ_PROF_CLASSES = 6 };
int nrq_profile_enable(nrq_ctx *ctx, int enable);
int nrq_profile_read(nrq_ctx *ctx, int64_t launches[6], double milliseconds[6], double bytes[6]);
/* The initial conditions' random stream drawn on the device (no reference
 * counterpart: a check of the device draw against the reference's
 * generator, src/ranlxd_generator.f90:251-350).  normals = 0: count numbers
 * (count even) from number `first` (even) of the ranlxd stream of (level,
 * seed); normals = 1: the real parts of the Box-Muller normals of count
 * consecutive pairs from `first` (src/random.f90:238-255).  Into the host
 * array out.                                                             */
int nrq_ranlxd_draw(nrq_ctx *ctx, int level, int64_t seed, uint64_t first, int64_t count, int normals,
                    double *out);

/* ---- gauge configuration: src/gaugeconfiguration_su3.f90:33-116 -------- */
int nrq_gauge_create(nrq_ctx *ctx, nrq_gauge **g);      /* Allocate (:124-140)   */
int nrq_gauge_destroy(nrq_gauge *g);                    /* Deallocate            */
int nrq_gauge_upload(nrq_gauge *g, const double *links, const double *efield);
int nrq_gauge_download(const nrq_gauge *g, double *links, double *efield);
int nrq_gauge_copy(nrq_gauge *dst, const nrq_gauge *src); /* configuration copies, src/main.f90:2320 */
/* ColdInit, src/gaugeconfiguration_su3.f90:363-378 */
int nrq_gauge_cold_init(nrq_gauge *g);
/* TransversePolarisedOccupiedInit_Box, src/gaugeconfiguration_su3.f90:906-951
 * (-> :1263-1446) after random%InitModule(seed) (src/random.f90:126-140);
 * identity_links != 0 keeps U = 1 while drawing the same random stream.     */
int nrq_gauge_transverse_box_init(nrq_gauge *g, double saturation_scale, double amplitude,
                                  double coupling, int64_t seed, int identity_links);
/* Update_Leapfrog(StepWidth), src/gaugeconfiguration_su3.f90:2082-2111 */
int nrq_gauge_update(nrq_gauge *g, double stepwidth);
/* Precision form of the leapfrog (no reference counterpart; the reference
 * is FP64 throughout, src/precision.f90:20).  prec = 1: the links evolve in
 * FP32 storage (staple products in FP32, staple sums, force projection and
 * Ẽ in FP64, group exponential in FP64), with an FP64 reunitarisation onto
 * SU(3) every reunit_every steps.  Energy, Gauss law, downloads and the CN
 * step read the FP64 view of the links, refreshed on demand.  prec = 0 (the
 * default) is the FP64 leapfrog.  Ensemble members must stay at prec 0.    */
int nrq_gauge_set_precision(nrq_gauge *g, int prec, int reunit_every);
/* max over sites and directions of |(U U^+ - 1)_ij| and of |det U - 1|     */
int nrq_gauge_unitarity(nrq_gauge *g, double *max_dev, double *max_det_dev);
/* GetEnergy, src/gaugeconfiguration_su3.f90:1769-1817 */
int nrq_gauge_energy(nrq_gauge *g, double *energy);
/* GetDeviationFromGaussLaw (:1480-1531) -> ref_measure, and the max-norm
 * GetGdeviation of EquilibriumInit (:724-768) -> max_norm                   */
int nrq_gauge_gauss(nrq_gauge *g, double *ref_measure, double *max_norm);
/* The Gauss projection loop of EquilibriumInit,
 * src/gaugeconfiguration_su3.f90:455-500 (no charges): Jacobi sweeps of the
 * electric field until the max-norm deviation (:724-768) is at most tol.
 * *sweeps gets the sweeps taken and *deviation the final deviation (either
 * may be NULL).  max_sweeps <= 0 means no limit, as in the reference;
 * otherwise NRQ_ERR_NOT_CONVERGED after max_sweeps sweeps.                  */
int nrq_gauge_gauss_project(nrq_gauge *g, double tol, int64_t max_sweeps, int64_t *sweeps, double *deviation);
/* EquilibriumInit(beta, nefieldinit, nequilibrium, tol), same file :380-814
 * after random%InitModule(seed) (src/random.f90:126-140), without charges and
 * without the file output of MeasureEnergy: cold links, then nefieldinit
 * rounds of a thermal field (E^a_k(x) = Re(sqrt(4/beta) r) a0 for complex
 * normals r drawn per site and direction, :432-444), the Gauss projection and
 * nequilibrium leapfrog steps.  Per round (arrays of nefieldinit entries,
 * each may be NULL): projection sweeps, energy and max-norm deviation after
 * the steps (the values the reference writes and prints).  max_sweeps bounds
 * each projection as in nrq_gauge_gauss_project.                            */
int nrq_gauge_equilibrium_init(nrq_gauge *g, double beta, int64_t nefieldinit, int64_t nequilibrium,
                               double tol, int64_t seed, int64_t max_sweeps, int64_t *sweeps,
                               double *energies, double *deviations);
/* CoulombGaugefixing(Tolerance, alpha, MaxIterations) ->
 * CoulombGaugefixing_Links, src/gaugeconfiguration_su3.f90:2269-2456: Fourier
 * accelerated steepest descent on the links (the electric field is not
 * transformed, as in the reference).  *iterations gets the reference's loop
 * counter after the loop (the iteration whose divergence met tol, or
 * max_iterations + 1); deviations[k] (max_iterations entries, or NULL) the
 * maximum |div|_F / 9 checked at iteration k + 1 (the value the reference
 * prints).                                                                  */
int nrq_gauge_coulomb_gaugefix(nrq_gauge *g, double tol, double alpha, int64_t max_iterations,
                               int64_t *iterations, double *deviations);
/* GetTransverseAACorrelator / GetTransverseEECorrelator, same file
 * :1825-1972, and GetNorm2Momentum_G (src/lattice.f90:1081-1089): per
 * momentum site in lattice order, V entries each (any may be NULL).         */
int nrq_gauge_transverse_correlators(nrq_gauge *g, double *aa, double *ee, double *momenta);

/* ---- heavy-quark field: src/nrqcd.f90:58-117 -------------------------- */
int nrq_heavy_create(nrq_ctx *ctx, nrq_heavy **h);      /* NRQCDField() (:235-248) */
int nrq_heavy_destroy(nrq_heavy *h);                    /* Destructor (:255-260)   */
int nrq_heavy_upload(nrq_heavy *h, const double *quark, const double *antiq);
int nrq_heavy_download(const nrq_heavy *h, double *quark, double *antiq);
int nrq_heavy_copy(nrq_heavy *dst, const nrq_heavy *src); /* assignment(=) (:219-228) */
/* InitSinglePoint(LatticeIndex_quark, LatticeIndex_antiq), src/nrqcd.f90:324-350
 * (1-based lattice indices)                                                 */
int nrq_heavy_init_single_point(nrq_heavy *h, int64_t lattice_index_quark,
                                int64_t lattice_index_antiq);
/* GetNorm_Quark / GetNorm_AntiQ, src/nrqcd.f90:547-611 */
int nrq_heavy_norms(nrq_heavy *h, double *norm_quark, double *norm_antiq);
/* GetMesoncorrelator_{O1_1S0,O1_3S1,O8_1S0,O8_3S1}_ZeroMomentum,
 * src/nrqcd.f90:1484-1661; out[8] = re/im of the four correlators          */
int nrq_heavy_correlators(nrq_heavy *h, double out[8]);
/* GetMesoncorrelator_{O1_1S0,O1_3S1,O8_1S0,O8_3S1}_ZeroMomentum_gconjg,
 * src/nrqcd.f90:1728-1905 (conjg(AntiQProp) in place of its hermitian
 * conjugate); out[8] as above                                              */
int nrq_heavy_correlators_gconjg(nrq_heavy *h, double out[8]);

/* ---- Crank-Nicolson solver module: src/nrqcd.f90:167-212, 619-869 ------ */
/* InitModule(Mass, WilsonCoeffs, StepWidth, kspTol); c = 4 complex (8 doubles).
 * form: 0 = plain FP64 (BiCGStab, fused stencil/axpy/dot kernels);
 *       1 = precision (FP32 Chebyshev inner iterations inside FP64
 *           iterative refinement to the same tol; real Wilson coefficients).
 * maxits bounds the Krylov iterations (the reference's PETSc default 1e4):
 * BiCGStab iterations of the plain form, FP32 Chebyshev inner steps of the
 * precision forms (over all refinement passes of one update).              */
int nrq_cn_init(nrq_ctx *ctx, double mass, const double c[8], double stepwidth, double tol,
                int64_t maxits, int form, nrq_cn **cn);
/* FinalizeModule, src/nrqcd.f90:199-212 */
int nrq_cn_finalize(nrq_cn *cn);
/* FP64 stencils of the solver (no reference counterpart: PETSc applies its
 * assembled matrix; these apply the same operator matrix-free).
 * REGISTER: register-tiled; TMA: TMA-staged; TENSOR: FP64 tensor-core MMAs
 * on per-update 6x6 blocks; FMA: FP64 FMAs on the same per-update blocks
 * (TENSOR and FMA need real Wilson coefficients; otherwise the TMA or
 * register-tiled stencil runs).                                           */
#define NRQ_STENCIL_REGISTER 0
#define NRQ_STENCIL_TMA 1
#define NRQ_STENCIL_TENSOR 2
#define NRQ_STENCIL_FMA 3
/* The stencil the solver uses and the per-launch milliseconds of each one
 * measured on its first update (index = NRQ_STENCIL_*; -1 before it, or for
 * one that does not apply to the lattice or coefficients).               */
int nrq_cn_stencil_info(const nrq_cn *cn, int *stencil, double ms[4]);
/* Test hook of the FMA stencil's bounded pipeline waits (no reference
 * counterpart).  wait_cycles bounds every wait (0 restores the default,
 * about two seconds); stall_load >= 0 makes the stencil's loader stop
 * before that load of every CTA, so the wait for it runs out: the update
 * then returns NRQ_ERR_TIMEOUT, nothing faults, and the context stays
 * usable.  -1 (the default) stops nowhere.                                */
int nrq_cn_set_wait_test(nrq_cn *cn, int64_t wait_cycles, int stall_load);
/* Force a stencil (NRQ_STENCIL_*) or restore the timed choice (-1).
 * NRQ_ERR_BAD_ARG if the stencil cannot describe this lattice.            */
int nrq_cn_set_stencil(nrq_cn *cn, int stencil);
/* The FP32 Chebyshev step of the precision forms (forms 1 and 2; no
 * reference counterpart).  REGISTER: the operator assembled from FP32 links
 * and field strengths per launch; BLOCKS: FP32 FMAs on per-update 6x6
 * blocks staged by TMA (V a multiple of 4, V >= 36, nx even).  -1 (the
 * default) times both on the first update where BLOCKS applies and keeps
 * the faster; forcing BLOCKS on a lattice it cannot describe is
 * NRQ_ERR_BAD_ARG.  nrq_cn_cheb_info gives the step the last update ran
 * (-1 before any) and the per-launch milliseconds of each (index NRQ_CHEB_*;
 * -1 where not timed); either pointer may be NULL.                        */
#define NRQ_CHEB_REGISTER 0
#define NRQ_CHEB_BLOCKS 1
int nrq_cn_set_cheb_stencil(nrq_cn *cn, int which);
int nrq_cn_cheb_info(const nrq_cn *cn, int *last, double ms[2]);
/* Plain and precision forms (no reference counterpart): on = 1 (the
 * default) starts every solve from 2b - psi plus the extrapolation of the
 * corrections t to that start of the field's last steps (the depth below),
 * kept per field in FP32 (576 B per site and step); 0 starts from 2b - psi.
 * Any upload, copy or point source restarts the history.  The tolerance is
 * the same either way.  The learned form uses its network's start.        */
int nrq_cn_set_history_guess(nrq_cn *cn, int on);
/* The history vectors the extrapolated start uses (1-4, default
 * 4): x0 = 2b - psi + the degree depth - 1 extrapolation of the field's last
 * depth corrections t (t1; 2 t1 - t2; 3 t1 - 3 t2 + t3; 4 t1 - 6 t2 + 4 t3
 * - t4), fewer while the field has fewer steps of history.  Each history
 * vector is 576 B per site (FP32).  No reference counterpart (PETSc's KSP
 * starts from zero: the solution vector holds psi, src/nrqcd.f90:1108-1123,
 * but KSPSetInitialGuessNonzero is never called).                          */
int nrq_cn_set_history_depth(nrq_cn *cn, int depth);
/* The solve's acceptance.  always = 1 confirms every converged solve with
 * the true residual b - A^H x (one residual pass); 0 (the default) accepts,
 * as PETSc's KSP (src/nrqcd.f90:803) tests its recursive residual:
 *  - plain form: BiCGStab's recursive residual, where every column's meets
 *    the tolerance with a margin of four times the largest gap between
 *    recursive and true residual that this solver's confirmed solves showed;
 *  - precision forms: the Chebyshev prediction of the last pass (the
 *    previous residual over the pass's guaranteed gain), where twice it,
 *    scaled by the largest true-to-predicted ratio of this solver's
 *    confirmed passes, meets the tolerance;
 * the first solve and every 16th after an unconfirmed run confirm.
 * nrq_cn_true_residual_info: whether the last update's max_rel_residual is
 * the true residual (1) or the recursive or predicted one (0).            */
/* Plain form on the FMA stencil: on = 1 (the default) updates x, r and p of
 * an iteration in one pass, beta taken from rh.t, which the t = A^H s launch
 * reduces (rh.s vanishes by the choice of alpha, so rho_new = -omega rh.t),
 * with the shadow residual rh kept in FP32 (every product with it, rho_0
 * included, uses the same rounded values); 0 keeps two passes (x and r,
 * then p) with rho_new = rh.r reduced and rh in FP64.  No reference
 * counterpart (PETSc's KSPBCGS, src/nrqcd.f90:803).                       */
int nrq_cn_set_merged_update(nrq_cn *cn, int on);
int nrq_cn_set_true_residual(nrq_cn *cn, int always);
int nrq_cn_true_residual_info(const nrq_cn *cn, int *last_true);
/* NRQCDField%Update(GaugeConf, Mass, WilsonCoeffs, StepWidth) =
 * Update_CrankNicholson, src/nrqcd.f90:1053-1168: quark (+M, c) and
 * antiquark (-M, conj c); per column RHS = A psi, solve A^H psi' = RHS with
 * A the operator PETSc assembles (blocks transposed, src/nrqcd.f90:1014-1018).
 * Returns NRQ_ERR_NOT_CONVERGED if a column missed the tolerance within
 * maxits (the fields are still updated); stats may be NULL.                  */
int nrq_heavy_update_cn(nrq_cn *cn, nrq_heavy *h, const nrq_gauge *g, double mass,
                        const double c[8], double stepwidth, nrq_cn_stats *stats);
/* Apply the assembled operator A (herm = 0) or A^H (herm = 1) to all 6
 * propagator columns of both species: quark with (+M, c), antiquark with
 * (-M, conj c); out = A in.  MatMult of src/nrqcd.f90:1112, exposed for
 * verification.                                                            */
int nrq_cn_apply(nrq_cn *cn, const nrq_gauge *g, double mass, const double c[8],
                 double stepwidth, int herm, const nrq_heavy *in, nrq_heavy *out);

/* ---- batching: many fields, one gauge field, one launch per kernel ---- */
/* No single counterpart in the reference, whose driver advances one
 * NRQCDField per NRQCDField%Update call (src/nrqcd.f90:1053), field after
 * field where it evolves several (src/main.f90:983-985).  A batch holds n fields (propagator sources x
 * heavy masses) of one context; nrq_cn_batch_update advances every field by
 * one Crank-Nicolson step in the gauge field g with the precision form of
 * nrq_heavy_update_cn (form 1) at tolerance tol, each kernel launch covering
 * every field.  The result of field i equals that of nrq_heavy_update_cn on
 * field i alone to within the tolerance.  Fields must be distinct and belong
 * to ctx; masses[i] is the heavy mass of fields[i].
 *
 * The first update (and the first after c or stepwidth change) calibrates:
 * it runs the refinement adaptively with host synchronisation, times the
 * candidate Chebyshev kernels (tile and register variants x block order)
 * and keeps the fastest, and records the per-pass inner step counts as the schedule.
 * Later updates replay the schedule without host synchronisation, as one
 * CUDA graph when use_graph != 0, and verify every field's FP64 residual at
 * the end; a field that missed the tolerance gets adaptive passes and
 * extends the schedule.  The fields' device buffers are exchanged with the
 * batch's work buffers on every update (as in nrq_heavy_update_cn).        */
typedef struct nrq_cn_batch nrq_cn_batch;
int nrq_cn_batch_create(nrq_ctx *ctx, int nfields, nrq_heavy *const *fields, const double *masses,
                        double tol, nrq_cn_batch **batch);
int nrq_cn_batch_destroy(nrq_cn_batch *batch);
/* stats: iterations = FP32 inner steps, matvecs = stencil applications per
 * field, max_rel_residual = max over fields and columns.                    */
int nrq_cn_batch_update(nrq_cn_batch *batch, const nrq_gauge *g, const double c[8], double stepwidth,
                        int use_graph, nrq_cn_stats *stats);
/* Start every field's solve from the learned guess of `net` (a network of
 * the same context, see nrq_learn_*; NULL detaches).  The fields keep their
 * two-step history as with nrq_heavy_update_cn in form 2; the schedule is
 * recalibrated while the history fills (depth 0, 1, 2).  Declared in the
 * learned-guess section below.                                            */
struct nrq_learn;
int nrq_cn_batch_attach_learned(nrq_cn_batch *batch, struct nrq_learn *net);
/* Relative residual ||b - A^H x|| / ||b|| of every field (max over its 12
 * columns) after the last update, in the order of `fields`.                 */
int nrq_cn_batch_residuals(const nrq_cn_batch *batch, double *rel);
/* Tuning and schedule: the chosen Chebyshev kernel variant (0: one field
 * per tile, 2 blocks per SM; 1: one field per tile, 3 blocks per SM; 2: two
 * fields of one mass per tile; 3: the FP32 block step, per-update blocks of
 * every mass staged by TMA with the fields' vectors, where the lattice
 * allows it: V a multiple of 4, V >= 36, nx even) and block order (0: field
 * fastest, 1: site block fastest), the measured milliseconds per launch of
 * every candidate (NRQ_BATCH_CANDIDATES entries, index variant*2 + order;
 * -1 where not applicable), and the inner steps of each refinement pass (up
 * to 16).                                                                 */
#define NRQ_BATCH_CANDIDATES 8
int nrq_cn_batch_info(const nrq_cn_batch *batch, int *variant, int *order, double candidate_ms[8],
                      int *npasses, int steps[16]);
/* Force the Chebyshev kernel variant and block order (as in
 * nrq_cn_batch_info; NRQ_ERR_BAD_ARG where the variant does not apply) or
 * restore the timed choice (variant -1).  The next update recalibrates.    */
int nrq_cn_batch_set_variant(nrq_cn_batch *batch, int variant, int order);
/* The FP64 stencil of the batch's right-hand side and residuals: 0 the
 * register-tiled one, 1 FP64 FMAs on per-update blocks of every mass staged
 * by TMA (V even, V >= 34).  The batch times both with its Chebyshev
 * candidates on the first update (ms, index = which; -1 where not timed);
 * nrq_cn_batch_set_fp64 forces one (the next update recalibrates).        */
int nrq_cn_batch_fp64_info(const nrq_cn_batch *batch, int *which, double ms[2]);
/* The gate of an attached learned guess: the calibration with the guess's
 * full two-step history measures the guess's cost and prices the inner
 * steps and refinement passes it saved against the last schedule without
 * it (same step width and coefficients); when the saving is below 1.25
 * times the cost the guess is switched off (gate 0) and the batch runs the
 * plain start.  gate: -2 no guess attached, -1 not decided yet, 1 on, 0
 * off; guess_ms, saving_ms: the measured cost and the value of the saving
 * (-1 before).                                                             */
int nrq_cn_batch_learned_info(const nrq_cn_batch *batch, int *gate, double *guess_ms, double *saving_ms);
/* The scheduled steps' predicted acceptance (no reference counterpart):
 * after the last pass each unconverged column's residual is predicted from
 * its residual before the pass and the pass's guaranteed Chebyshev gain;
 * where twice the prediction, scaled by the largest true-to-predicted
 * ratio the measured columns showed, meets the tolerance, the column is
 * accepted on it and the final residual check skips the fields accepted in
 * full (the first scheduled step and every 16th predict nothing).  ratio:
 * that largest ratio (-1 before the first measurement); steps: scheduled
 * steps taken.  Synchronises the batch's stream.                          */
int nrq_cn_batch_prediction_info(const nrq_cn_batch *batch, double *ratio, int64_t *steps);
/* Without a learned guess every field of the batch starts from 2b - psi plus
 * the cubic extrapolation of its last four corrections, as the single-field
 * solves do (on = 1, the default); 0 starts from 2b - psi.  No reference
 * counterpart.                                                             */
int nrq_cn_batch_set_history(nrq_cn_batch *batch, int on);
int nrq_cn_batch_set_fp64(nrq_cn_batch *batch, int which);

/* An ensemble of independent members (batch[i], gauge[i]); the members may
 * sit on contexts of different lattice sizes on the same device.  One step
 * advances every member by the coupled timestep of the reference's driver
 * loop (src/main.f90:346-348): the batch's Crank-Nicolson update, then the
 * leapfrog of its gauge field.  With use_graph != 0 the step after the
 * calibration is captured once as one CUDA graph (one child graph per
 * member, members independent) and every later step is one graph launch.
 * stats aggregate over members (max residual, sum of matvecs).             */
typedef struct nrq_ensemble nrq_ensemble;
int nrq_ensemble_create(int nmembers, nrq_cn_batch *const *batches, nrq_gauge *const *gauges,
                        nrq_ensemble **ens);
int nrq_ensemble_destroy(nrq_ensemble *ens);
int nrq_ensemble_step(nrq_ensemble *ens, const double c[8], double stepwidth, int use_graph,
                      nrq_cn_stats *stats);

/* ---- learned initial guess (form 2) ----------------------------------- */
/* No counterpart in the reference (PETSc KSP starts from zero,
 * src/nrqcd.f90:1108-1123).  Per sample (site, species) a
 * 16 -> 64 -> 64 -> 6 MLP (ReLU, BF16 weights and activations, FP32
 * accumulation on the tensor cores) maps local invariants of the right-hand
 * side b = A psi, of the field's history and of the gauge field
 * (plaquettes, E^2) to complex (w0, w1, w2); the solve of form 2 starts from
 *   x0 = 2 b - psi + w0 |tau| (b - psi) + w1 v1 + w2 v2,   tau = dt a0 / 2,
 * with v1, v2 = x - (2 b - psi) of the field's previous two steps (a
 * learned per-site linear prediction).  The FP64 residual check of the
 * precision form decides convergence, as without the network.
 * Parameters: W1[64][16], b1[64], W2[64][64], b2[64], W3[6][64] and the
 * output bias b3[6][6] per group (quark with 0, 1, 2 history vectors, then
 * the antiquark's), FP32, this order.  Training refits b3 in closed form
 * (the loss is quadratic in it).                                          */
#define NRQ_LEARN_NPARAMS 5668
typedef struct nrq_learn nrq_learn;
int nrq_learn_create(nrq_ctx *ctx, uint64_t seed, nrq_learn **net);
int nrq_learn_destroy(nrq_learn *net);
/* get (set = 0) or set (set = 1) the FP32 parameters; setting resets Adam */
int nrq_learn_params(nrq_learn *net, float *params, int set);
/* mark the network usable by form 2 (nrq_learn_train sets it)             */
int nrq_learn_set_trained(nrq_learn *net, int trained);
/* training data: room for max_samples samples (2 per site and step)       */
int nrq_learn_dataset_reserve(nrq_learn *net, int64_t max_samples);
int nrq_learn_dataset_size(const nrq_learn *net, int64_t *n);
/* features (n x 16) and normalised Gram statistics (n x 16) of samples
 * [first, first+count)                                                    */
int nrq_learn_dataset_read(nrq_learn *net, int64_t first, int64_t count, float *features, float *stats);
/* One CN step of h (cn's form, without the network) that appends the
 * step's 2V samples to the dataset and leaves h's history for the next one. */
int nrq_learn_record(nrq_learn *net, nrq_cn *cn, nrq_heavy *h, const nrq_gauge *g, double mass,
                     const double c[8], double stepwidth, nrq_cn_stats *stats);
/* Adam on random batches of the dataset; learning rate lr with cosine decay
 * to 5 %; the loss (mean squared guess error relative to the plain
 * extrapolation's) of the first and last batch.                            */
int nrq_learn_train(nrq_learn *net, int64_t iterations, int64_t batch, double lr, uint64_t seed,
                    double *loss_first, double *loss_last);
/* Loss and gradient (NRQ_LEARN_NPARAMS) of n samples given in host memory
 * (features n x 16, statistics n x 16), for checks against a CPU oracle.   */
int nrq_learn_loss_grad(nrq_learn *net, const float *features, const float *stats, int64_t n,
                        double *loss, float *grad);
/* Network outputs (n x 6: Re/Im of w0, w1, w2) of host features.          */
int nrq_learn_forward(nrq_learn *net, const float *features, int64_t n, float *out);
/* Use net for the initial guess of cn (form 2); NULL detaches.            */
int nrq_cn_attach_learned(nrq_cn *cn, nrq_learn *net);

/* ---- energy without any device allocation ---------------------------- */
/* No counterpart in the reference.  This is for callers that cannot call
 * cudaMalloc, for example a driver port whose fields live in device memory
 * owned by another runtime (OpenACC or CUDA Fortran data regions, a
 * framework's caching allocator) and that must not grow the device footprint
 * inside its time loop.  Computes the same energy as nrq_gauge_energy without
 * a context or handle.  It allocates nothing.
 *
 * Inputs are in caller-owned device memory in the device plane layout:
 *   links_soa  : 27 planes of V complex (interleaved re, im),
 *                plane = dir*9 + row*3 + col
 *   efield_soa : 24 planes of V doubles, plane = dir*8 + a
 * The energy goes to energy_out, one double of device-accessible memory.
 * The launches go onto `stream`, a cudaStream_t of the current device
 * (NULL = default stream), and the function returns without synchronising.
 *
 * Partial sums go into a fixed 128 KiB device array in the library.  That
 * caps the lattice at NRQ_NOALLOC_MAX_SITES sites (for example 160^3);
 * larger lattices return NRQ_ERR_CAPACITY.  The first call in a CUDA
 * context looks up the array's address and caches it under the context's
 * unique id, so make that first call before any stream capture.  The cached
 * address is not reused in another context: after cudaDeviceReset (or under
 * another driver-API context) the next call looks it up again, and should
 * likewise come before any capture.  An error already pending from the
 * caller's earlier work returns NRQ_ERR_CUDA and is left pending.  All calls
 * share the array: calls that overlap on the GPU race and must be
 * serialised.                                                               */
#define NRQ_NOALLOC_MAX_SITES 4194304
int nrq_gauge_energy_noalloc(const int64_t extents[3], const double spacings[4],
                             const double *links_soa, const double *efield_soa,
                             double *energy_out, void *stream);

#ifdef __cplusplus
}
#endif
#endif
