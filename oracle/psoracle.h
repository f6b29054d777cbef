/*
 * psoracle.h -- CPU oracle for the PolyStokes per-timestep Stokesian-dynamics path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference's
 * algorithm, used by tests/, by __graft_entry__.smoke() and by bench.py's
 * cpu_baseline leg as the checker.  The product (the CUDA path behind
 * include/polystokes_b200.h) never links, loads or calls it.
 *
 * Every function cites the reference file:line it restates (paths relative to
 * the sgnagella/polystokes_brownian project).  Parity pin: the tensor formulas
 * are checked against the dense grand-mobility dump mob.csv that ships with the
 * reference (tests/golden/mobcsv_*.npz); everything else (the PETSc MINRES, the
 * SLEPc MFN square root, LAPACK dsyev) is a restatement of the published
 * algorithm of that library, pinned only by the reference's own call sites.
 */
#ifndef PSORACLE_H
#define PSORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* How the monomer-colloid translational block (colloid U <- monomer F and its
 * transpose) is formed.  The reference's mobility_AB (mob.cpp:362-537) computes
 * x12a/y12a but its mob_a fill is commented out (mob.cpp:447-453), so:
 *   OR_AB_REFERENCE: shell path (mm_HI=0): zero (the local `la` is never written,
 *                    mob.cpp:998,1015); dense path (mm_HI=1): the stale global
 *                    mob_a left by the last pair tensor evaluated before the AB
 *                    loop (mob.cpp:845-904).
 *   OR_AB_RPY:       the unequal-radii far-field RPY scalars that mobility_AB
 *                    computes but never uses (mob.cpp:410-411).
 *   OR_AB_RPY_REG:   OR_AB_RPY plus the overlap / full-overlap branches of the
 *                    unequal-radii RPY (Zuk et al. 2014) for the translation and
 *                    rotation couplings, commented out in mob.cpp:414-453.    */
enum { OR_AB_REFERENCE = 0, OR_AB_RPY = 1, OR_AB_RPY_REG = 2 };

/* Monomer-monomer translation scalars.  OR_AA_REFERENCE: mob.cpp:122-131
 * (x = 3/(8r) - 2/r^3, y = 3/(4r) - 1/(2r^3); overlap x = 3r/8 - 1, y = 1 - 9r/32).
 * OR_AA_RPY: equal-sphere Rotne-Prager-Yamakawa of radius beta in the units of
 * the reference (6 pi eta = 1): x = 3/(2r) - b^2/r^3, y = 3/(4r) + b^2/(2r^3) for
 * r > 2b; overlap x = (1 - 3r/(16b))/b, y = (1 - 9r/(32b))/b. */
enum { OR_AA_REFERENCE = 0, OR_AA_RPY = 1 };

typedef struct or_params {
    int    Nm, Nc, Npoly, Nmono_per_chain;
    double beta, kT, epsilon, kbond, r0, Lmax, tau;
    double dt;
    int    mm_HI, chain_HI, fene, tether, mono_ev, record_forces;
    int    box_on;
    double box[3];
    double ktrap, tstart, trun, weaken_trap;
    double t0;              /* initial time (restart) */
    int    restart;         /* nonzero: trap centres are not taken from x */
    int    ab_mode;         /* OR_AB_REFERENCE or OR_AB_RPY */
    double hs_kpref;        /* HS_KPREF (pair_interaction.cpp:185), default 1 */
    int    hs_kmode;        /* HS_KMODE (pair_interaction.cpp:186), default 0 */
    int    lanczos_nc;      /* POLYSTOKES_LANCZOS_NC (slip_vel.cpp:97), default 64 */
    /* lubrication (absent from the reference; restated from Fiore & Swan 2019) */
    int    lub_on;
    double lub_gap;         /* pairs with gap < lub_gap * a get a resistance block */
    int    noise_lanczos;   /* mm_HI noise: 0 exact eigen square root, 1 Lanczos (kmax 40, tol 1e-6) */
    int    aa_mode;         /* OR_AA_REFERENCE or OR_AA_RPY */
    int    lub_bonded;      /* nonzero: bonded chain neighbours are lubricated too */
} or_params;

typedef struct or_sim or_sim;

/* construction / state (Stokes.cpp:11-36,171-317; init.cpp:185-360) */
or_sim *or_create(const or_params *p);
void    or_destroy(or_sim *s);
void    or_set_state(or_sim *s, const double *x, const double *q);
void    or_get_state(const or_sim *s, double *x, double *q);
void    or_set_time(or_sim *s, double t);
double  or_get_time(const or_sim *s);
int     or_sizes(const or_sim *s, int *out8);   /* nm3,nc11,nm3nc6,nm3nc11,n,Np,nc5,n3 */
void    or_set_lub_tables(or_sim *s, const double *tab, int nrow, int ncol);

/* pair tensors (mob.cpp:30-537), outputs as the double the reference stores */
void or_tensor_aa(double r, double rinv, const double e[3], double beta, int mode, double a[9]);
void or_tensor_ab(double r, double rinv, const double e[3], double beta, int reg,
                  double b[9], double gt[15]);
void or_tensor_ab_rpy(double r, double rinv, const double e[3], double beta, int reg, double a[9]);
/* regularised translation (x along e, y across) and rotation-translation (yb) scalars */
void or_ab_reg_scalars(double r, double beta, double *x, double *y, double *yb);
void or_tensor_bb(double r, double rinv, const double e[3], double a[9], double b[9],
                  double c[9], double gt[15], double ht[15], double m[25]);

/* stage: check_dist + cell list + RHS + mob + Schur sync (run.cpp:87-93) */
void or_check_dist(or_sim *s);                      /* check_dist.cpp:12-87 */
int  or_verlet_pairs(const or_sim *s, int *pi, int *pj, int maxp);
int  or_cell_pairs(or_sim *s, int *pi, int *pj, int maxp); /* cell_list.cpp:23-172 */
void or_rhs(or_sim *s, int drift, const double *fext, double *rhs); /* rhs.cpp:246-346 */
void or_mob(or_sim *s);                             /* mob.cpp:635-1213 */
void or_schur_sync(or_sim *s);                      /* slip_vel.cpp:81-203 */
void or_stale_a(const or_sim *s, double *tab9);     /* AB trans block of the last or_mob */

/* operators (matfree_A.cpp:38-102, arrays.cpp:349-408) */
void or_dense_mobility(const or_sim *s, double *M);                 /* nm3nc11^2 row-major */
void or_mobility_apply(const or_sim *s, const double *u, double *y); /* matrix-free */
void or_saddle_apply(const or_sim *s, const double *x, double *y);
void or_saddle_diag(const or_sim *s, double *d);
void or_mcm(const or_sim *s, double *Mcm);   /* nc11 x nm3 row-major (arrowhead) */
void or_mcc(const or_sim *s, double *Mcc);   /* nc11 x nc11 row-major, current Mcc_block */

/* KSP (init.cpp:27-72, vel.cpp:7-113): preconditioned MINRES, Jacobi */
int  or_minres(const or_sim *s, const double *b, double *x, int warm, double rtol,
               int maxit, int *iters, double *rnorm);

/* Brownian noise (slip_vel.cpp:19-477) */
void or_slip_noise(or_sim *s, const double *fb, double *W);       /* unscaled W */
void or_sqrtm_eig(const double *M, int n, const double *z, double *w); /* sqrt(max(M,0)) z */
int  or_lanczos_sqrt(const or_sim *s, const double *z, double *w, int kmax, double tol);
void or_jacobi_eig(double *A, int n, double *lam, double *Q);    /* sym. eig, ascending */

/* lubrication (new) */
int  or_lub_pairs(const or_sim *s, int *pi, int *pj, int maxp);
void or_lub_apply(const or_sim *s, const double *u, double *y);  /* y = R_lub u (nm3nc6) */

/* one predictor-corrector step with injected noise (run.cpp:70-162) */
typedef struct or_step_out {
    double *v_det_n, *v_det_c, *v_brown, *up, *udiff, *sb, *fext; /* may be NULL */
    int iters[5];
} or_step_out;
void or_step(or_sim *s, const double *fb, const double *wrfd, const double *zlub,
             double rtol, or_step_out *out);

#ifdef __cplusplus
}
#endif
#endif
