/*
 * polystokes_b200.h -- C-ABI of the B200-native PolyStokes per-timestep hot path.
 *
 * One context holds a batch of independent systems ("replicas"); a single
 * PolyStokes system is a batch of one.  Vector arguments are DEVICE pointers
 * to the concatenation of the replicas' segments, except where a declaration
 * says otherwise (ps_set_state, ps_step_inputs' noise arrays and ps_set_aux also
 * accept host pointers; ps_obs_read writes host arrays).  Each segment is laid
 * out exactly as the reference lays out its PETSc vectors:
 *
 *   saddle vector (length n = 6 Nm + 17 Nc per replica):
 *     [ F_m (3Nm) | F_c (3Nc) | T_c (3Nc) | S_c (5Nc) | U_m (3Nm) | U_c (3Nc) | W_c (3Nc) ]
 *   positions: 3 Np doubles per replica (monomers first, then colloids)
 *   quaternions: 4 Nc doubles per replica
 *
 * Return value: 0 success; negative = error (PS_ERR_*); ps_ksp_solve returns the
 * KSP-style converged reason of the worst replica (>0 converged, <0 diverged).
 * Streams are passed as void* (a cudaStream_t; NULL = legacy default stream).
 *
 * Reference interfaces replaced (paths within sgnagella/polystokes_brownian):
 *   ps_matmult        <- ArrowheadMult(Mat,Vec,Vec)          src/matfree_A.cpp:38-80
 *                        and dense MatMult(A) of mm_HI        src/arrays.cpp:371-408, src/mob.cpp:843-1160
 *   ps_get_diagonal   <- ArrowheadGetDiagonal(Mat,Vec)        src/matfree_A.cpp:84-102
 *   ps_ksp_solve      <- KSPSolve(ksp,rhs,X), MINRES+Jacobi   src/vel.cpp:7-66, src/init.cpp:27-72
 *   ps_build_pairs    <- check_dist / build_monomer_cell_list src/check_dist.cpp:12-87, src/cell_list.cpp:23-96
 *   ps_assemble       <- mob() + sync_mcc_schur_correction()  src/mob.cpp:635-1213, src/slip_vel.cpp:81-203
 *   ps_rhs            <- RHS(bool drift)                      src/rhs.cpp:246-346
 *   ps_sqrtm_apply    <- solve_slip_vel()                     src/slip_vel.cpp:19-79,205-477
 *   ps_step           <- one iteration of the run() loop      src/run.cpp:70-162
 */
#ifndef POLYSTOKES_B200_H
#define POLYSTOKES_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PS_OK 0
#define PS_ERR_ARG (-1)
#define PS_ERR_CUDA (-2)
#define PS_ERR_NOMEM (-3)
#define PS_ERR_STATE (-4)
#define PS_ERR_UNSUPPORTED (-5)
#define PS_ERR_TOO_LARGE (-6)

/* AB (monomer-colloid) translational block mode: the reference's assembly
 * (mob.cpp:447-453, 845-904: zero in the shell path, the stale last monomer-pair
 * tensor in the dense path) or the unequal-radii far-field RPY scalars
 * (mob.cpp:410-411). */
#define PS_AB_REFERENCE 0
#define PS_AB_RPY 1
/* PS_AB_RPY with the overlap and full-overlap branches of the unequal-radii RPY
 * (Zuk et al. 2014) for the translation and rotation couplings; the stresslet
 * coupling stays far-field.  The reference carries these branches commented out
 * (mob.cpp:414-453, mobdat/rpy_kk_mobilities.tex). */
#define PS_AB_RPY_REG 2

/* Monomer-monomer translation scalars: the reference's own (mob.cpp:122-131)
 * or the equal-sphere RPY of radius beta with its overlap form. */
#define PS_AA_REFERENCE 0
#define PS_AA_RPY 1

/* Saddle solver.  PS_SOLVE_MINRES: preconditioned MINRES with Jacobi, as the
 * reference's KSPSolve.  PS_SOLVE_STRUCTURED: exact elimination of the
 * constraint block -- F_t = -b_bot, one dense colloid-stresslet solve
 * M_SS F_S = b_S - (M F)_S, then U = (M F)_t - b_t (two operator applies) --
 * followed by warm-started MINRES only where the elimination is not exact
 * (lubrication, or more than 12 colloids in a replica). */
#define PS_SOLVE_MINRES 0
#define PS_SOLVE_STRUCTURED 1

/* precision of the far-field matvec and Krylov vectors */
#define PS_PREC_FP64 0
#define PS_PREC_MIXED 1

/* One system; mirrors PolyStokes(...) + particle_info(...) + trap_info(...)
 * (src/bindings.cpp:45-91, src/Stokes.cpp:11-252). */
typedef struct ps_desc {
    int32_t Nm, Nc, Npoly, Nmono_per_chain;
    double beta, kT, epsilon, kbond, r0, Lmax, tau;
    double dt;
    int32_t mm_HI, chain_HI, fene, tether, mono_ev, record_forces;
    int32_t box_on;
    double box[3];
    double ktrap, tstart, trun, weaken_trap;
    double t0;          /* start time (restart) */
    int32_t restart;    /* nonzero: trap centres are not re-derived from x */
    int32_t ab_mode;    /* PS_AB_REFERENCE | PS_AB_RPY | PS_AB_RPY_REG */
    double hs_kpref;    /* HS_KPREF, default 1.0 */
    int32_t hs_kmode;   /* HS_KMODE, default 0 */
    int32_t lanczos_nc; /* POLYSTOKES_LANCZOS_NC (slip_vel.cpp:283-288): shell replicas with
                           nc11 above it (or above 64, the dense limit here) take the Schur
                           Lanczos noise; 0 sends every shell replica there; negative = 64 */
    int32_t lub_on;     /* near-field lubrication (not in the reference) */
    double lub_gap;     /* lubricated pairs: gap < lub_gap * radius */
    int32_t aa_mode;    /* PS_AA_REFERENCE | PS_AA_RPY: monomer-monomer scalars */
    int32_t lub_bonded; /* nonzero: bonded chain neighbours are lubricated too (default 0: skipped) */
} ps_desc;

typedef struct ps_ksp_opts {
    double rtol;        /* relative tolerance (reference hard-codes 1e-6) */
    int32_t maxit;      /* iteration cap (PETSc default 10000) */
    int32_t warm;       /* nonzero: x holds the initial guess */
    int32_t check_every;/* host convergence poll period in iterations (0 = 8) */
    int32_t method;     /* PS_SOLVE_MINRES (the reference's MINRES + Jacobi) or PS_SOLVE_STRUCTURED */
} ps_ksp_opts;

typedef struct ps_ksp_result {
    int32_t reason;     /* worst replica reason */
    int32_t iters_max;  /* max iterations over replicas */
    int64_t iters_sum;  /* sum of iterations over replicas */
    double rnorm_max;   /* largest final residual-norm estimate */
} ps_ksp_result;

typedef struct ps_sqrt_opts {
    int32_t kmax;       /* Lanczos subspace cap */
    double tol;         /* relative change between successive estimates */
} ps_sqrt_opts;

typedef struct ps_sqrt_result {
    int32_t iters_max;
    int32_t nneg;       /* negative projected eigenvalues floored (sum over replicas) */
} ps_sqrt_result;

/* Optional injected noise for one step (device or host pointers, concatenated
 * per replica; host arrays are copied in by the call); NULL members are drawn on
 * the device from the replicas' Philox streams. */
typedef struct ps_step_inputs {
    const double *fb;   /* nm3nc11 per replica: slip-velocity white noise (slip_vel.cpp:11-17) */
    const double *wrfd; /* nm3nc6 per replica: RFD displacement (drift.cpp:9-15) */
    const double *zlub; /* 12 per lubricated pair (monomer pairs use 6), canonical pair order */
    double rtol;        /* MINRES rtol for the five solves */
    int32_t maxit;
    int32_t sqrt_kmax;  /* Lanczos subspace cap of the noise (0: 40) */
    double sqrt_tol;    /* Lanczos relative tolerance of the noise (0: 1e-6) */
    int32_t solver;     /* PS_SOLVE_MINRES (default) or PS_SOLVE_STRUCTURED */
    int32_t refine;     /* mixed precision only: FP64 iterative-refinement sweeps per solve (0: none).
                           Each sweep forms the saddle residual b - A x with the FP64 operator and
                           adds the mixed-precision solution of A d = r (same rtol) to x.  No
                           reference counterpart (the reference solves in FP64 throughout). */
} ps_step_inputs;

typedef struct ps_step_result {
    int32_t iters[5];   /* max over replicas, per solve */
    int32_t reason;     /* worst KSP reason over the five solves */
    int32_t lanczos_iters;  /* Lanczos subspace size of the noise (max over replicas) */
    int32_t lanczos_nneg;   /* negative projected eigenvalues floored (sum over replicas) */
} ps_step_result;

typedef struct ps_ctx ps_ctx;

/* context ------------------------------------------------------------------ */
int ps_ctx_create(const ps_desc *descs, int32_t nrep, int32_t precision, ps_ctx **out);
int ps_ctx_destroy(ps_ctx *ctx);
int ps_ctx_sizes(const ps_ctx *ctx, int64_t *out8); /* ntot_beads, nvec, ntop, nvel, ncoll, nrep, 0, 0 */
int ps_ctx_offsets(const ps_ctx *ctx, int32_t rep, int64_t *out4); /* bead, vec, top, vel offsets */
int ps_set_lub_table(ps_ctx *ctx, const double *host_tab, int32_t nrow, int32_t ncol);
int ps_set_seed(ps_ctx *ctx, uint64_t seed);
/* Per-replica noise streams (no reference counterpart; the reference draws from
 * one std::mt19937_64 per process, Stokes.h:111-112).  Device draws of replica r
 * at its step k use Philox keyed by seeds[r], subsequence = the DOF's index
 * within the replica, offset by k: a replica's noise does not depend on the
 * other replicas of the batch.  ps_set_seed(ctx, s) sets seeds[r] =
 * splitmix64(s + r) and all step counters to 0.  steps may be NULL (unchanged). */
int ps_set_replica_seeds(ps_ctx *ctx, const uint64_t *host_seeds, const uint64_t *host_steps);
int ps_get_replica_steps(ps_ctx *ctx, uint64_t *host_steps);
/* Per-replica auxiliary state: time (R), trap constant ktrap (R; weaken_trap
 * changes it, rhs.cpp:46-100), trap centres xpos0 (3 Nc per replica, colloid
 * order).  Host or device pointers; NULL members are skipped.  With
 * ps_get_state/ps_set_state and ps_get_replica_steps/ps_set_replica_seeds this
 * moves a trajectory between contexts (continuous batching) or restarts it;
 * the reference restarts from its own files instead (Stokes.cpp:19-34). */
int ps_get_aux(ps_ctx *ctx, double *time, double *ktrap, double *xpos0, void *stream);
int ps_set_aux(ps_ctx *ctx, const double *time, const double *ktrap, const double *xpos0, void *stream);
const char *ps_last_error(void);

/* Trajectory observables accumulated on the device, per replica (the analysis
 * the reference runs on its output files: bond and trap statistics,
 * test_sim_dumbbells_thermal.py:178-330; the windowed MSD tensor of the
 * colloids, get_msd.py:5-28).  Host arrays; NULL members are skipped.
 *   bond  R x 10: count, sum of bond vectors (3), sum |b|, sum |b|^2,
 *                 increment count, sum of bond-vector increments between samples (3)
 *   trap  R x 9:  count, sum of displacements from the trap centre (3), sum |d|,
 *                 sum |d|^2, sum d_x^2, d_y^2, d_z^2
 *   bond_hist, trap_hist  R x nbins: counts of |b| in [0, bond_max), |d| in [0, trap_max)
 *   msd  R x lags x 6: sums over colloids and time origins of dx dx, dy dy, dz dz,
 *                 dx dy, dx dz, dy dz at lag l samples; msd_count R x lags       */
typedef struct ps_obs_out {
    double *bond;
    uint64_t *bond_hist;
    double *trap;
    uint64_t *trap_hist;
    double *msd;
    uint64_t *msd_count;
} ps_obs_out;
int ps_obs_reset(ps_ctx *ctx, int32_t nbins, double bond_max, double trap_max, int32_t lags);
int ps_observe(ps_ctx *ctx, void *stream);        /* one sample of the current state */
int ps_obs_read(ps_ctx *ctx, ps_obs_out *out, void *stream);

/* state --------------------------------------------------------------------- */
/* x (3 Np per replica), q (4 Nc per replica): device or host pointers; reads
 * into host memory are complete when the call returns.  Host inputs are checked
 * before any copy or launch: a non-finite coordinate or quaternion component
 * returns PS_ERR_ARG (ps_last_error names the index) and leaves the state as it
 * was.  Device inputs are taken as given. */
int ps_set_state(ps_ctx *ctx, const double *x, const double *q, void *stream);
int ps_get_state(ps_ctx *ctx, double *x, double *q, void *stream);
int ps_set_time(ps_ctx *ctx, double t);

/* stage pieces (check_dist, RHS, mob) --------------------------------------- */
int ps_build_pairs(ps_ctx *ctx, void *stream);
int ps_pair_list(ps_ctx *ctx, int32_t which, int32_t *pi, int32_t *pj, int64_t maxp,
                 int64_t *count, void *stream);  /* which: 0 Verlet, 1 monomer WCA, 2 lubrication */
int ps_rhs(ps_ctx *ctx, int32_t drift, const double *fext, double *rhs, void *stream);
int ps_assemble(ps_ctx *ctx, void *stream);

/* operator and solver (MatShell MatMult / GetDiagonal / KSPSolve) ----------- */
int ps_matmult(ps_ctx *ctx, const double *x, double *y, void *stream);
int ps_mobility_apply(ps_ctx *ctx, const double *u, double *y, void *stream);
int ps_get_diagonal(ps_ctx *ctx, double *d, void *stream);
int ps_ksp_solve(ps_ctx *ctx, const double *b, double *x, const ps_ksp_opts *opts,
                 ps_ksp_result *res, void *stream);

/* Brownian noise: w = M^{1/2} z (unscaled), as solve_slip_vel before scaling */
int ps_sqrtm_apply(ps_ctx *ctx, const double *z, double *w, const ps_sqrt_opts *opts,
                   ps_sqrt_result *res, void *stream);

/* one predictor-corrector step of every replica */
int ps_step(ps_ctx *ctx, const ps_step_inputs *in, ps_step_result *res, void *stream);
int ps_step_outputs(ps_ctx *ctx, double *up, double *udiff, double *sb, double *fext, void *stream);

/* allocation-free entry point ----------------------------------------------
 * ps_mobility_apply_noalloc: y = M u for ONE system of N monomers (the
 * monomer-monomer far-field mobility with full HI and the reference's pair
 * scalars, PS_AA_REFERENCE: beta^{-1} u plus the pair blocks, skipping
 * same-chain pairs when chain_HI; chains are contiguous runs of
 * Nmono_per_chain monomers).  x: 3N positions, u: 3N forces, y: 3N velocities,
 * all device pointers.  It has no counterpart in the reference: it exists for
 * callers that must not allocate device memory (an operator callback run inside
 * a host solver that owns the device memory pool, or a latency-critical loop
 * where cudaMalloc's implicit synchronisation or failure is not acceptable).
 * It allocates nothing: its scratch is a fixed 3.4 MB __device__ array held by
 * every GPU that loads this library until exit, so N is limited to 8192
 * (larger N returns PS_ERR_TOO_LARGE).  The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress) and caches it for the device.
 * With CUDA's lazy module loading (the CUDA 12 default) that first call may also
 * be where the library's device code is loaded and the 3.4 MB array placed,
 * which can synchronise the device or fail under memory pressure: make the first
 * call at start-up, before any stream capture and before the device fills up.
 * After cudaDeviceReset the cached address is stale; do not call it again in
 * that process.  Calls share the array, so calls that overlap on the GPU race;
 * serialise them. */
int ps_mobility_apply_noalloc(const double *x, const double *u, double *y, int32_t N, double beta,
                              int32_t chain_HI, int32_t Nmono_per_chain, void *stream);

/* diagnostics ---------------------------------------------------------------
 * ps_time_kernel: average device time (ms, CUDA events on `stream`) of `reps`
 * launches of one far-field kernel on mobility-layout input u; which: 0 the
 * monomer-monomer pair kernel, 1 monomer-colloid, 2 colloid-colloid, 3 the whole
 * mobility apply.  ps_fma_peak: measured FMA throughput (TFLOP/s) of the current
 * device, FP64 when fp64 != 0, else FP32 (the larger of scalar and packed FP32x2
 * FMA chains). */
int ps_time_kernel(ps_ctx *ctx, int32_t which, int32_t reps, const double *u, double *ms, void *stream);
int ps_fma_peak(int32_t fp64, double *tflops, void *stream);
/* ps_rsqrt_check (no reference counterpart): the largest distance, in units in the
 * last place, between the FP64 pair kernel's reciprocal square root (single-
 * precision seed + second-order binomial correction) and CUDA's rsqrt over the
 * n device values a. */
int ps_rsqrt_check(const double *a, int64_t n, uint64_t *max_ulp, void *stream);
/* number of kernels the library has launched since it was loaded */
uint64_t ps_kernel_launches(void);
/* Autotuner (no counterpart in the reference): times the whole mobility apply
 * of this context (the monomer far-field kernel, whose column-chunk width is
 * tuned, plus the combine that reads one partial sum per chunk) for each width
 * in {128, 256, 512, 1024} (reps applies each, CUDA events) and keeps the
 * fastest for this context and
 * for every context created afterwards in the process.  The width is
 * process-wide so that a replica's arithmetic stays independent of its batch.
 * best_cols / ms (4 timings, candidate order) may be NULL. */
int ps_autotune(ps_ctx *ctx, int32_t reps, int32_t *best_cols, double *ms, void *stream);

#ifdef __cplusplus
}
#endif
#endif
