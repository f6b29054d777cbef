/*
 * psoracle.c -- CPU oracle (plain C, FP64 with the reference's long-double
 * tensor arithmetic) for the PolyStokes per-timestep hot path.
 *
 * TEST INFRASTRUCTURE ONLY: used as the checker by tests/, smoke() and the
 * cpu_baseline leg of bench.py.  The shipped CUDA path never calls it.
 *
 * Reference files restated (paths within sgnagella/polystokes_brownian):
 *   src/mob.cpp, src/matfree_A.cpp, src/arrays.cpp, src/vel.cpp, src/init.cpp,
 *   src/check_dist.cpp, src/cell_list.cpp, src/rhs.cpp, src/pair_interaction.{h,cpp},
 *   src/slip_vel.cpp, src/drift.cpp, src/traj.cpp, src/quat.cpp, src/box.cpp,
 *   src/run.cpp, src/Stokes.cpp.
 * Third-party algorithms restated from their published descriptions:
 *   PETSc KSPMINRES (Paige & Saunders 1975, preconditioned form) with PCJACOBI
 *   fix-diagonal; LAPACK dsyev replaced by the cyclic Jacobi eigenvalue method
 *   (Golub & Van Loan, Matrix Computations, sec. 8.5); SLEPc MFN+FNSQRT replaced
 *   by the exact eigendecomposition square root (equal in exact arithmetic for
 *   SPD M); lubrication (absent from the reference) per Fiore & Swan,
 *   J. Fluid Mech. 878 (2019) 544, saddle lower-right block -R_lub.
 */
#include "psoracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>

typedef long double ld;

/* ------------------------------------------------------------------------- */
/* system                                                                     */
/* ------------------------------------------------------------------------- */
struct or_sim {
    or_params p;
    int Np, nm3, nc3, nc5, nc6, nc11, nm3nc3, nm3nc6, nm3nc11, n, n3;
    /* float-stored cutoffs, init.cpp:332-338 (Data holds std::vector<float>) */
    float rverl[3], sig[3], rcut[3];
    double beta_inv, beta2;
    double tstop, ktrap;  /* ktrap is mutated by weaken_trap (rhs.cpp:151-153) */
    double t;
    double *x, *q, *xpos0;
    int *chain;           /* chain id per monomer (init.cpp:207-212) */
    int nbonds; int *bi, *bj;   /* bond list (init.cpp:296-321) */
    /* stored pair list (init.cpp:225-291): all pairs if mm_HI else AB+BB */
    long npair;
    int *pi, *pj; unsigned char *ptype;
    double *pd;           /* 5 per pair: e0,e1,e2,r,1/r (check_dist.cpp:67-71) */
    unsigned char *inverl; /* pair is in the Verlet list (check_dist.cpp:59) */
    /* arrowhead pieces (mm_HI=0) */
    double *Mcm;          /* nc11 x nm3 row-major */
    double *Mcc_base, *Mcc_block, *Mcc_delta, *schurQ, *schurL;   /* nc11 x nc11 */
    int schur_valid;
    /* AB translational block used by the last or_mob (stale mob_a) */
    double tab[9];
    double stale[9];      /* global mob_a state carried between mob() calls */
    /* lubrication tables: rows of r, then 10 columns (r2babc.dat layout) */
    double *lub; int lub_nrow;
};

static void *xcalloc(size_t n, size_t s) { void *p = calloc(n ? n : 1, s); return p; }
static long pair_index(const or_sim *s, int a, int b);

int or_sizes(const or_sim *s, int *o)
{
    o[0] = s->nm3; o[1] = s->nc11; o[2] = s->nm3nc6; o[3] = s->nm3nc11;
    o[4] = s->n; o[5] = s->Np; o[6] = s->nc5; o[7] = s->n3;
    return 0;
}

or_sim *or_create(const or_params *p)
{
    or_sim *s = (or_sim *)xcalloc(1, sizeof(or_sim));
    s->p = *p;
    int Nm = p->Nm, Nc = p->Nc, Np = Nm + Nc;
    s->Np = Np;
    /* Stokes.cpp:67-98 */
    s->nm3 = 3 * Nm; s->nc3 = 3 * Nc; s->nc5 = 5 * Nc; s->nc6 = 6 * Nc;
    s->nc11 = s->nc5 + s->nc6; s->nm3nc3 = s->nm3 + s->nc3;
    s->nm3nc6 = s->nm3 + s->nc6; s->nm3nc11 = s->nm3 + s->nc11;
    s->n = s->nm3nc11 + s->nm3nc6; s->n3 = 3 * Np;
    s->beta_inv = 1.0 / p->beta; s->beta2 = p->beta * p->beta;
    double pref = pow(2.0, 1.0 / 6.0);
    s->rverl[0] = (float)(0.05 + 2 * p->beta); s->rverl[1] = (float)(1.5 + p->beta); s->rverl[2] = 2.5f;
    s->sig[0] = (float)(2. * p->beta); s->sig[1] = (float)(1. + p->beta); s->sig[2] = 2.0f;
    for (int k = 0; k < 3; k++) s->rcut[k] = (float)(pref * (double)s->sig[k]);
    s->tstop = p->tstart + p->trun; s->ktrap = p->ktrap;
    s->t = p->t0;
    s->x = (double *)xcalloc(3 * Np, sizeof(double));
    s->q = (double *)xcalloc(4 * (Nc ? Nc : 1), sizeof(double));
    s->xpos0 = (double *)xcalloc(3 * (Nc ? Nc : 1), sizeof(double));
    for (int c = 0; c < Nc; c++) s->q[4 * c] = 1.0;
    s->chain = (int *)xcalloc(Nm, sizeof(int));
    for (int i = 0; i < p->Npoly; i++)
        for (int j = 0; j < p->Nmono_per_chain; j++) {
            int k = i * p->Nmono_per_chain + j;
            if (k < Nm) s->chain[k] = i;
        }
    /* bonds (init.cpp:296-321) */
    int nbp = p->Nmono_per_chain - 1;
    s->nbonds = nbp * p->Npoly + (p->tether ? p->Npoly : 0);
    s->bi = (int *)xcalloc(s->nbonds, sizeof(int));
    s->bj = (int *)xcalloc(s->nbonds, sizeof(int));
    int kk = 0;
    for (int i = 0; i < p->Npoly; i++)
        for (int j = 0; j < nbp; j++) { int a = i * p->Nmono_per_chain + j; s->bi[kk] = a; s->bj[kk] = a + 1; kk++; }
    if (p->tether) {
        int cpc = Nc ? p->Npoly / Nc : 1; if (cpc < 1) cpc = 1;
        for (int i = 0; i < p->Npoly; i++) {
            int host = Nm + i / cpc; if (host >= Np) host = Np - 1;
            s->bi[kk] = i * p->Nmono_per_chain; s->bj[kk] = host; kk++;
        }
    }
    /* stored pairs (init.cpp:225-291) */
    long npAA = (long)Nm * (Nm - 1) / 2, npAB = (long)Nm * Nc, npBB = (long)Nc * (Nc - 1) / 2;
    s->npair = (p->mm_HI ? npAA : 0) + npAB + npBB;
    s->pi = (int *)xcalloc(s->npair, sizeof(int));
    s->pj = (int *)xcalloc(s->npair, sizeof(int));
    s->ptype = (unsigned char *)xcalloc(s->npair, 1);
    s->pd = (double *)xcalloc(5 * s->npair, sizeof(double));
    s->inverl = (unsigned char *)xcalloc(s->npair, 1);
    long k = 0;
    if (p->mm_HI)
        for (int i = 0; i < Nm; i++) for (int j = i + 1; j < Nm; j++) { s->pi[k] = i; s->pj[k] = j; s->ptype[k] = 0; k++; }
    for (int i = 0; i < Nm; i++) for (int j = Nm; j < Np; j++) { s->pi[k] = i; s->pj[k] = j; s->ptype[k] = 1; k++; }
    for (int i = Nm; i < Np; i++) for (int j = i + 1; j < Np; j++) { s->pi[k] = i; s->pj[k] = j; s->ptype[k] = 2; k++; }
    s->Mcm = (double *)xcalloc((size_t)s->nc11 * s->nm3, sizeof(double));
    s->Mcc_base = (double *)xcalloc((size_t)s->nc11 * s->nc11, sizeof(double));
    s->Mcc_block = (double *)xcalloc((size_t)s->nc11 * s->nc11, sizeof(double));
    s->Mcc_delta = (double *)xcalloc((size_t)s->nc11 * s->nc11, sizeof(double));
    s->schurQ = (double *)xcalloc((size_t)s->nc11 * s->nc11, sizeof(double));
    s->schurL = (double *)xcalloc(s->nc11, sizeof(double));
    /* fill_self leaves mob_a = I (mob.cpp:65-86,568) */
    for (int a = 0; a < 9; a++) s->stale[a] = (a % 4 == 0) ? 1.0 : 0.0;
    /* Mcc_base: colloid self FTS (mob.cpp:586-622) */
    for (int c = 0; c < Nc; c++) {
        int t = 3 * c, r = s->nc3 + 3 * c, st = s->nc6 + 5 * c, n11 = s->nc11;
        for (int a = 0; a < 3; a++) { s->Mcc_base[(t + a) * n11 + t + a] = 1.0; s->Mcc_base[(r + a) * n11 + r + a] = 0.75; }
        for (int a = 0; a < 5; a++) s->Mcc_base[(st + a) * n11 + st + a] = 9. / 5.;
        s->Mcc_base[(st + 0) * n11 + st + 4] = 9. / 10.;
        s->Mcc_base[(st + 4) * n11 + st + 0] = 9. / 10.;
    }
    memcpy(s->Mcc_block, s->Mcc_base, sizeof(double) * s->nc11 * s->nc11);
    return s;
}

void or_destroy(or_sim *s)
{
    if (!s) return;
    free(s->x); free(s->q); free(s->xpos0); free(s->chain); free(s->bi); free(s->bj);
    free(s->pi); free(s->pj); free(s->ptype); free(s->pd); free(s->inverl);
    free(s->Mcm); free(s->Mcc_base); free(s->Mcc_block); free(s->Mcc_delta); free(s->schurQ); free(s->schurL);
    free(s->lub); free(s);
}

void or_set_lub_tables(or_sim *s, const double *tab, int nrow, int ncol)
{
    free(s->lub);
    s->lub = (double *)xcalloc((size_t)nrow * 11, sizeof(double));
    for (int i = 0; i < nrow; i++)
        for (int c = 0; c < 11; c++) s->lub[i * 11 + c] = (c < ncol) ? tab[i * ncol + c] : 0.0;
    s->lub_nrow = nrow;
}

/* Stokes.cpp:254-317: positions; trap centres from the colloids on a fresh start */
void or_set_state(or_sim *s, const double *x, const double *q)
{
    memcpy(s->x, x, sizeof(double) * s->n3);
    if (!s->p.restart) for (int a = 0; a < s->nc3; a++) s->xpos0[a] = x[s->nm3 + a];
    if (q) memcpy(s->q, q, sizeof(double) * 4 * s->p.Nc);
}
void or_get_state(const or_sim *s, double *x, double *q)
{
    if (x) memcpy(x, s->x, sizeof(double) * s->n3);
    if (q) memcpy(q, s->q, sizeof(double) * 4 * s->p.Nc);
}
void or_set_time(or_sim *s, double t) { s->t = t; }
double or_get_time(const or_sim *s) { return s->t; }

/* box.cpp:40-84 (orthorhombic, nearbyint) */
static void min_image(const or_sim *s, double *dx, double *dy, double *dz)
{
    if (!s->p.box_on) return;
    const double *L = s->p.box;
    *dx -= L[0] * nearbyint(*dx * (1.0 / L[0]));
    *dy -= L[1] * nearbyint(*dy * (1.0 / L[1]));
    *dz -= L[2] * nearbyint(*dz * (1.0 / L[2]));
}
static void wrap(const or_sim *s, double *x)
{
    if (!s->p.box_on) return;
    for (int d = 0; d < 3; d++) x[d] -= s->p.box[d] * nearbyint(x[d] * (1.0 / s->p.box[d]));
}

/* ------------------------------------------------------------------------- */
/* pair tensors, mob.cpp:30-537                                               */
/* ------------------------------------------------------------------------- */
static const ld EPS3[3][3][3] = {
    {{0, 0, 0}, {0, 0, 1}, {0, -1, 0}},
    {{0, 0, -1}, {0, 0, 0}, {1, 0, 0}},
    {{0, 1, 0}, {-1, 0, 0}, {0, 0, 0}}};
static ld DEL(int i, int j) { return i == j ? 1.0L : 0.0L; }
static int third(int a, int b) { int k = 3 - a - b; if (k == -1) k = 2; if (k == 3) k = 0; return k; }

/* monomer-monomer translation block, mob.cpp:122-147 (reference-specific formula) */
void or_tensor_aa(double r, double rinv, const double e[3], double beta, int mode, double a9[9])
{
    double x, y;
    double ri3 = rinv * rinv * rinv;
    if (mode == OR_AA_RPY) {
        double b2 = beta * beta;
        if (r > 2.0 * beta) { x = 1.5 * rinv - b2 * ri3; y = 0.75 * rinv + 0.5 * b2 * ri3; }
        else { x = (1.0 - 3.0 * r / (16.0 * beta)) / beta; y = (1.0 - 9.0 * r / (32.0 * beta)) / beta; }
    } else if (r > 2.0 * beta) { x = (3. / 8.) * rinv - 2.0 * ri3; y = (3. / 4.) * rinv - (1. / 2.) * ri3; }
    else { x = (3. / 8.) * r - 1.0; y = 1.0 - (9. / 32.) * r; }
    for (int i = 0; i < 3; i++) {
        ld ee = (ld)(e[i] * e[i]);
        a9[i * 3 + i] = (double)(x * ee + y * (1. - ee));
        for (int j = i + 1; j < 3; j++) {
            ld eij = (ld)(e[i] * e[j]);
            double v = (double)(x * eij - y * eij);
            a9[i * 3 + j] = v; a9[j * 3 + i] = v;
        }
    }
}

/* unequal-radii far-field translation block computed (and left unused) by
 * mobility_AB, mob.cpp:410-411; used only in OR_AB_RPY mode */
/* Zuk et al. (2014) unequal-radii RPY, colloid radius 1, monomer radius beta < 1,
 * in the reference's units (6 pi eta = 1) and sign convention (yb = -mu^rt),
 * the branches of mob.cpp:414-453 (commented out there) and
 * mobdat/rpy_kk_mobilities.tex eqs. for mu^tt and mu^rt. */
void or_ab_reg_scalars(double r, double beta, double *x, double *y, double *yb)
{
    double b2 = beta * beta;
    if (r >= 1.0 + beta) {
        *x = 1.5 / r - 0.5 * (1.0 + b2) / (r * r * r);
        *y = 0.75 / r + 0.25 * (1.0 + b2) / (r * r * r);
        *yb = -0.75 / (r * r);
    } else if (r > 1.0 - beta) {
        double rd = 1.0 - beta, r2 = r * r, r3 = r2 * r;
        double t = rd * rd + 3.0 * r2, u = rd * rd - r2;
        double I = (16.0 * r3 * (1.0 + beta) - t * t) / (32.0 * r3);
        *y = I / beta;
        *x = (I + 3.0 * u * u / (32.0 * r3)) / beta;
        *yb = -(3.0 / (8.0 * beta)) * (rd + r) * (rd + r) * (b2 + 2.0 * beta * (1.0 + r) - 3.0 * (1.0 - r) * (1.0 - r))
              / (8.0 * r2);
    } else {
        *x = 1.0;
        *y = 1.0;
        *yb = -0.75 * r;
    }
}

void or_tensor_ab_rpy(double r, double rinv, const double e[3], double beta, int reg, double a9[9])
{
    double ri3 = rinv * rinv * rinv, b2 = beta * beta, yb;
    double x = (3. / 2.) * rinv - (1. / 2.) * (1.0 + b2) * ri3;
    double y = (3. / 4.) * rinv + (1. / 4.) * (1.0 + b2) * ri3;
    if (reg) or_ab_reg_scalars(r, beta, &x, &y, &yb);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            double ee = e[i] * e[j];
            a9[i * 3 + j] = x * ee + y * ((i == j) - ee);
        }
}

/* monomer-colloid rotation-force and stresslet-force blocks, mob.cpp:455-537 */
void or_tensor_ab(double r, double rinv, const double e[3], double beta, int reg, double b9[9], double gt15[15])
{
    double ee[3][3];
    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) ee[i][j] = e[i] * e[j];
    double ri2 = rinv * rinv, ri3 = ri2 * rinv, ri4 = ri3 * rinv;
    (void)ri3;
    double b2 = beta * beta;
    double y12b = -(3. / 4.) * ri2;
    if (reg) { double xx, yy; or_ab_reg_scalars(r, beta, &xx, &yy, &y12b); }
    double x12g = (9. / 4.) * ri2 - (9. / 20.) * ri4 * (3 + 5 * b2);
    double y12g = (9. / 10.) * ri4 * ((1. / 2.) + (5. / 6.) * b2);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            int k = third(i, j);
            b9[i * 3 + j] = (double)(y12b * EPS3[i][j][k] * e[k]);
        }
    double gt[3][3][3];
    for (int k = 0; k < 3; k++)
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++)
                gt[k][i][j] = (double)(-x12g * (ee[i][j] - (1. / 3.) * DEL(i, j)) * e[k]
                                       + y12g * (e[i] * DEL(j, k) + e[j] * DEL(i, k) - 2. * ee[i][j] * e[k]));
    for (int i = 0; i < 3; i++) {
        gt15[i * 5 + 0] = gt[i][0][0] - gt[i][2][2];
        gt15[i * 5 + 1] = 2. * gt[i][0][1];
        gt15[i * 5 + 2] = 2. * gt[i][0][2];
        gt15[i * 5 + 3] = 2. * gt[i][1][2];
        gt15[i * 5 + 4] = gt[i][1][1] - gt[i][2][2];
    }
}

/* colloid-colloid FTS blocks, mob.cpp:96-358 */
void or_tensor_bb(double r, double rinv, const double e[3], double a9[9], double b9[9],
                  double c9[9], double gt15[15], double ht15[15], double m25[25])
{
    (void)r;
    ld ee[3][3];
    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) ee[i][j] = (ld)(e[i] * e[j]);
    double ri2 = rinv * rinv, ri3 = ri2 * rinv, ri4 = ri3 * rinv, ri5 = ri4 * rinv;
    double x12a = (3. / 2.) * rinv - ri3;
    double y12a = (3. / 4.) * rinv + (1. / 2.) * ri3;
    for (int i = 0; i < 3; i++) {
        a9[i * 3 + i] = (double)(x12a * ee[i][i] + y12a * (1. - ee[i][i]));
        for (int j = i + 1; j < 3; j++) {
            double v = (double)(x12a * ee[i][j] - y12a * ee[i][j]);
            a9[i * 3 + j] = v; a9[j * 3 + i] = v;
        }
    }
    double y12b = -(3. / 4.) * ri2;
    double x12g = (9. / 4.) * ri2 - (18. / 5.) * ri4;
    double y12g = (6. / 5.) * ri4;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            int k = third(i, j);
            b9[i * 3 + j] = (double)(y12b * EPS3[i][j][k] * e[k]);
        }
    ld gt[3][3][3];
    for (int k = 0; k < 3; k++)
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++)
                gt[k][i][j] = -x12g * (ee[i][j] - (1. / 3.) * DEL(i, j)) * e[k]
                              + y12g * (e[i] * DEL(j, k) + e[j] * DEL(i, k) - 2. * ee[i][j] * e[k]);
    for (int i = 0; i < 3; i++) {
        gt15[i * 5 + 0] = (double)(gt[i][0][0] - gt[i][2][2]);
        gt15[i * 5 + 1] = (double)(2. * gt[i][0][1]);
        gt15[i * 5 + 2] = (double)(2. * gt[i][0][2]);
        gt15[i * 5 + 3] = (double)(2. * gt[i][1][2]);
        gt15[i * 5 + 4] = (double)(gt[i][1][1] - gt[i][2][2]);
    }
    double x12c = (3. / 4.) * ri3, y12c = -(3. / 8.) * ri3;
    double y12h = -(9. / 8.) * ri3;
    double x12m = -(9. / 2.) * ri3 + (54. / 5.) * ri5;
    double y12m = (9. / 4.) * ri3 - (36. / 5.) * ri5;
    double z12m = (9. / 5.) * ri5;
    for (int i = 0; i < 3; i++) {
        c9[i * 3 + i] = (double)(x12c * ee[i][i] + y12c * (1. - ee[i][i]));
        for (int j = i + 1; j < 3; j++) {
            /* reference: off-diagonal uses +y12c (mob.cpp:252) */
            double v = (double)(x12c * ee[i][j] + y12c * ee[i][j]);
            c9[i * 3 + j] = v; c9[j * 3 + i] = v;
        }
    }
    ld ht[3][3][3];
    for (int k = 0; k < 3; k++)
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) {
                int l = third(j, k), m = third(i, k);
                ht[k][i][j] = y12h * (ee[i][l] * EPS3[j][k][l] + ee[j][m] * EPS3[i][k][m]);
            }
    for (int i = 0; i < 3; i++) {
        ht15[i * 5 + 0] = (double)(ht[i][0][0] - ht[i][2][2]);
        ht15[i * 5 + 1] = (double)(2. * ht[i][0][1]);
        ht15[i * 5 + 2] = (double)(2. * ht[i][0][2]);
        ht15[i * 5 + 3] = (double)(2. * ht[i][1][2]);
        ht15[i * 5 + 4] = (double)(ht[i][1][1] - ht[i][2][2]);
    }
    ld m4[3][3][3][3];
    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) for (int k = 0; k < 3; k++) for (int l = 0; l < 3; l++)
        m4[i][j][k][l] = (3. / 2.) * x12m * (ee[i][j] - (1. / 3.) * DEL(i, j)) * (ee[k][l] - (1. / 3.) * DEL(k, l))
            + (1. / 2.) * y12m * (ee[i][k] * DEL(j, l) + ee[j][k] * DEL(i, l) + ee[i][l] * DEL(j, k)
                                  + ee[j][l] * DEL(i, k) - 4. * ee[i][j] * ee[k][l])
            + (1. / 2.) * z12m * (DEL(i, k) * DEL(j, l) + DEL(j, k) * DEL(i, l) - DEL(i, j) * DEL(k, l)
                                  + ee[i][j] * DEL(k, l) + ee[k][l] * DEL(i, j)
                                  - ee[i][k] * DEL(j, l) - ee[j][k] * DEL(i, l)
                                  - ee[i][l] * DEL(j, k) - ee[j][l] * DEL(i, k) + ee[i][j] * ee[k][l]);
    static const int mes0[5] = {0, 0, 0, 1, 1}, mes1[5] = {2, 1, 2, 2, 2};   /* init.cpp:340-354 */
    for (int ii = 0; ii < 5; ii++) {
        int a = mes0[ii], b = mes1[ii];
        ld *row = NULL; (void)row;
        ld v0, v1, v2, v3, v4;
        if (ii == 0 || ii == 4) {
            v0 = m4[a][a][0][0] - m4[a][a][2][2] - (m4[b][b][0][0] - m4[b][b][2][2]);
            v1 = 2. * (m4[a][a][0][1] - m4[b][b][0][1]);
            v2 = 2. * (m4[a][a][0][2] - m4[b][b][0][2]);
            v3 = 2. * (m4[a][a][1][2] - m4[b][b][1][2]);
            v4 = m4[a][a][1][1] - m4[a][a][2][2] - (m4[b][b][1][1] - m4[b][b][2][2]);
        } else {
            v0 = 2. * (m4[a][b][0][0] - m4[a][b][2][2]);
            v1 = 4. * m4[a][b][0][1];
            v2 = 4. * m4[a][b][0][2];
            v3 = 4. * m4[a][b][1][2];
            v4 = 2. * (m4[a][b][1][1] - m4[a][b][2][2]);
        }
        m25[ii * 5 + 0] = (double)v0; m25[ii * 5 + 1] = (double)v1; m25[ii * 5 + 2] = (double)v2;
        m25[ii * 5 + 3] = (double)v3; m25[ii * 5 + 4] = (double)v4;
    }
}

/* ------------------------------------------------------------------------- */
/* check_dist, check_dist.cpp:12-87                                          */
/* ------------------------------------------------------------------------- */
void or_check_dist(or_sim *s)
{
    for (long k = 0; k < s->npair; k++) {
        int a = s->pi[k], b = s->pj[k];
        double dx = s->x[3 * a] - s->x[3 * b];
        double dy = s->x[3 * a + 1] - s->x[3 * b + 1];
        double dz = s->x[3 * a + 2] - s->x[3 * b + 2];
        min_image(s, &dx, &dy, &dz);
        double dr = sqrt(dx * dx + dy * dy + dz * dz);
        s->inverl[k] = dr < (double)s->rverl[s->ptype[k]];
        double ri = 1 / dr;
        double *pd = s->pd + 5 * k;
        pd[0] = dx * ri; pd[1] = dy * ri; pd[2] = dz * ri; pd[3] = dr; pd[4] = ri;
    }
}

int or_verlet_pairs(const or_sim *s, int *pi, int *pj, int maxp)
{
    int c = 0;
    for (long k = 0; k < s->npair; k++)
        if (s->inverl[k]) { if (c < maxp) { pi[c] = s->pi[k]; pj[c] = s->pj[k]; } c++; }
    return c;
}

/* monomer cell list, cell_list.cpp:23-96; pairs found by the 13-offset half
 * stencil of cell_list.cpp:98-172 with r^2 < rcut^2 (WCA range).  Returned as
 * (i,j) with the order the reference visits them. */
typedef struct { int nc[3]; double size[3], org[3]; int periodic; int *head, *next; } cellgrid;
static void build_cells(const or_sim *s, cellgrid *g)
{
    int Nm = s->p.Nm; double rc = (double)s->rverl[0];
    if (s->p.box_on) {
        int ncmin = 1 << 30;
        for (int d = 0; d < 3; d++) { g->nc[d] = (int)floor(s->p.box[d] / rc); if (g->nc[d] < ncmin) ncmin = g->nc[d]; }
        if (ncmin >= 3) {
            for (int d = 0; d < 3; d++) { g->size[d] = s->p.box[d] / g->nc[d]; g->org[d] = -0.5 * s->p.box[d]; }
            g->periodic = 1;
        } else {
            for (int d = 0; d < 3; d++) { double L = s->p.box[d]; g->nc[d] = 1; g->size[d] = L > 0 ? L : 1.0; g->org[d] = -0.5 * L; }
            g->periodic = 0;
        }
    } else {
        double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
        for (int i = 0; i < Nm; i++) for (int d = 0; d < 3; d++) {
            double v = s->x[3 * i + d]; if (v < lo[d]) lo[d] = v; if (v > hi[d]) hi[d] = v; }
        if (Nm == 0) for (int d = 0; d < 3; d++) { lo[d] = 0; hi[d] = 0; }
        for (int d = 0; d < 3; d++) {
            double ext = hi[d] - lo[d];
            int nc = (int)floor(ext / rc); g->nc[d] = nc > 1 ? nc : 1;
            g->size[d] = ext > 0.0 ? ext / g->nc[d] : rc;
            g->org[d] = lo[d];
        }
        g->periodic = 0;
    }
    long ncell = (long)g->nc[0] * g->nc[1] * g->nc[2];
    g->head = (int *)malloc(sizeof(int) * ncell);
    g->next = (int *)malloc(sizeof(int) * (Nm ? Nm : 1));
    for (long c = 0; c < ncell; c++) g->head[c] = -1;
    for (int i = 0; i < Nm; i++) {
        int c[3];
        for (int d = 0; d < 3; d++) {
            int ci = (int)floor((s->x[3 * i + d] - g->org[d]) / g->size[d]);
            if (ci < 0) ci = 0;
            if (ci >= g->nc[d]) ci = g->nc[d] - 1;
            c[d] = ci;
        }
        long cell = (long)c[0] + (long)g->nc[0] * (c[1] + (long)g->nc[1] * c[2]);
        g->next[i] = g->head[cell]; g->head[cell] = i;
    }
}

typedef void (*pair_cb)(or_sim *s, int i, int j, void *ctx);
static void walk_cells(or_sim *s, cellgrid *g, pair_cb cb, void *ctx)
{
    static const int OFF[13][3] = {{1, 0, 0}, {-1, 1, 0}, {0, 1, 0}, {1, 1, 0}, {-1, -1, 1}, {0, -1, 1}, {1, -1, 1},
                                   {-1, 0, 1}, {0, 0, 1}, {1, 0, 1}, {-1, 1, 1}, {0, 1, 1}, {1, 1, 1}};
    for (int cz = 0; cz < g->nc[2]; cz++) for (int cy = 0; cy < g->nc[1]; cy++) for (int cx = 0; cx < g->nc[0]; cx++) {
        long home = (long)cx + (long)g->nc[0] * (cy + (long)g->nc[1] * cz);
        int hi = g->head[home];
        if (hi < 0) continue;
        for (int i = hi; i != -1; i = g->next[i]) for (int j = g->next[i]; j != -1; j = g->next[j]) cb(s, i, j, ctx);
        for (int o = 0; o < 13; o++) {
            int nx = cx + OFF[o][0], ny = cy + OFF[o][1], nz = cz + OFF[o][2];
            if (g->periodic) {
                nx = (nx % g->nc[0] + g->nc[0]) % g->nc[0];
                ny = (ny % g->nc[1] + g->nc[1]) % g->nc[1];
                nz = (nz % g->nc[2] + g->nc[2]) % g->nc[2];
            } else {
                if (nx < 0 || nx >= g->nc[0] || ny < 0 || ny >= g->nc[1] || nz < 0 || nz >= g->nc[2]) continue;
            }
            long nb = (long)nx + (long)g->nc[0] * (ny + (long)g->nc[1] * nz);
            for (int i = hi; i != -1; i = g->next[i]) for (int j = g->head[nb]; j != -1; j = g->next[j]) cb(s, i, j, ctx);
        }
    }
}

typedef struct { int *pi, *pj, max, cnt; } paircollect;
static void collect_cb(or_sim *s, int i, int j, void *ctx)
{
    paircollect *pc = (paircollect *)ctx;
    double dx = s->x[3 * i] - s->x[3 * j], dy = s->x[3 * i + 1] - s->x[3 * j + 1], dz = s->x[3 * i + 2] - s->x[3 * j + 2];
    min_image(s, &dx, &dy, &dz);
    double dr2 = dx * dx + dy * dy + dz * dz, rc = (double)s->rcut[0];
    if (dr2 >= rc * rc || dr2 == 0.0) return;
    if (pc->cnt < pc->max) { pc->pi[pc->cnt] = i; pc->pj[pc->cnt] = j; }
    pc->cnt++;
}
int or_cell_pairs(or_sim *s, int *pi, int *pj, int maxp)
{
    cellgrid g; build_cells(s, &g);
    paircollect pc = {pi, pj, maxp, 0};
    walk_cells(s, &g, collect_cb, &pc);
    free(g.head); free(g.next);
    return pc.cnt;
}

/* ------------------------------------------------------------------------- */
/* forces and rhs, rhs.cpp:46-346, pair_interaction.{h,cpp}, cell_list.cpp   */
/* ------------------------------------------------------------------------- */
static double wca_mag(double dr, double ri, double sig, double rcut, double eps)
{
    if (dr >= rcut) return 0.0;
    double s1 = sig * ri, s2 = s1 * s1, s6 = s2 * s2 * s2, s12 = s6 * s6;
    return 24.0 * eps * ri * (2.0 * s12 - s6);
}
static void wca_cb(or_sim *s, int i, int j, void *ctx)
{
    double *f = (double *)ctx;
    double dx = s->x[3 * i] - s->x[3 * j], dy = s->x[3 * i + 1] - s->x[3 * j + 1], dz = s->x[3 * i + 2] - s->x[3 * j + 2];
    min_image(s, &dx, &dy, &dz);
    double rc = (double)s->rcut[0];
    double dr2 = dx * dx + dy * dy + dz * dz;
    if (dr2 >= rc * rc || dr2 == 0.0) return;
    double dr = sqrt(dr2), ri = 1.0 / dr;
    double fm = wca_mag(dr, ri, (double)s->sig[0], rc, s->p.epsilon);
    if (fm == 0.0) return;
    double fx = fm * dx * ri, fy = fm * dy * ri, fz = fm * dz * ri;
    f[3 * i] -= fx; f[3 * i + 1] -= fy; f[3 * i + 2] -= fz;
    f[3 * j] += fx; f[3 * j + 1] += fy; f[3 * j + 2] += fz;
}

void or_rhs(or_sim *s, int drift, const double *fext, double *rhs)
{
    memset(rhs, 0, sizeof(double) * s->n);
    if (drift) {   /* rhs.cpp:261-270 */
        for (int i = 0; i < s->nm3nc6; i++) rhs[s->nm3nc11 + i] = fext[i];
        return;
    }
    double *f = rhs + s->nm3nc11;   /* fint, nm3nc3 entries */
    /* pair_interaction_hs, pair_interaction.cpp:160-227 */
    double kp = s->p.hs_kpref;
    double k = (s->p.hs_kmode == 1) ? kp / (s->p.dt * s->p.beta) : kp / s->p.dt;
    int Nm = s->p.Nm;
    for (int a = 0; a < s->Np - 1; a++) {
        /* vlist[a] holds stored-pair indices with first particle a, ascending:
         * AA partners (mm_HI), then colloid partners */
        int jlo = (a < Nm) ? (s->p.mm_HI ? a + 1 : Nm) : a + 1;
        for (int b0 = jlo; b0 < s->Np; b0++) {
            long q = pair_index(s, a, b0);
            if (!s->inverl[q]) continue;
            int ty = s->ptype[q];
            if (ty == 0 && !s->p.mono_ev) continue;
            int b = s->pj[q];
            double sig = (double)s->sig[ty], dr = s->pd[5 * q + 3];
            double se = sig * (1.0 + 0.01);
            if (dr >= se) continue;
            double fm = k * (se - dr);
            if (fm == 0.0) continue;
            double fx = fm * s->pd[5 * q], fy = fm * s->pd[5 * q + 1], fz = fm * s->pd[5 * q + 2];
            f[3 * a] -= fx; f[3 * a + 1] -= fy; f[3 * a + 2] -= fz;
            f[3 * b] += fx; f[3 * b + 1] += fy; f[3 * b + 2] += fz;
        }
    }
    if (!s->p.mm_HI && s->p.mono_ev) {   /* monomer_wca via the cell list */
        cellgrid g; build_cells(s, &g);
        walk_cells(s, &g, wca_cb, f);
        free(g.head); free(g.next);
    }
    /* bond_forces, rhs.cpp:123-158 */
    for (int q = 0; q < s->nbonds; q++) {
        int a = s->bi[q], b = s->bj[q];
        double r[4];
        r[0] = s->x[3 * a] - s->x[3 * b]; r[1] = s->x[3 * a + 1] - s->x[3 * b + 1]; r[2] = s->x[3 * a + 2] - s->x[3 * b + 2];
        min_image(s, &r[0], &r[1], &r[2]);
        r[3] = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
        double fb[3];
        for (int d = 0; d < 3; d++) fb[d] = -s->p.kbond * (1 - (s->p.r0 / r[3])) * r[d];
        if (s->p.fene) {
            double ext2 = 1 / (1 - (r[3] / s->p.Lmax) * (r[3] / s->p.Lmax));
            for (int d = 0; d < 3; d++) fb[d] *= ext2;
        }
        for (int d = 0; d < 3; d++) { f[3 * a + d] -= fb[d]; f[3 * b + d] += fb[d]; }
    }
    /* trapping_forces, rhs.cpp:46-100 (static trap) */
    if (fabs(s->ktrap) >= 1e-12) {
        if (s->t > s->tstop && s->p.weaken_trap >= 0) s->ktrap = s->p.weaken_trap;
        for (int c = 0; c < s->p.Nc; c++) {
            int i3 = 3 * (s->p.Nm + c);
            double dx = s->x[i3] - s->xpos0[3 * c], dy = s->x[i3 + 1] - s->xpos0[3 * c + 1], dz = s->x[i3 + 2] - s->xpos0[3 * c + 2];
            min_image(s, &dx, &dy, &dz);
            f[i3] += s->ktrap * dx; f[i3 + 1] += s->ktrap * dy; f[i3 + 2] += s->ktrap * dz;
        }
    }
}

/* ------------------------------------------------------------------------- */
/* mob(), mob.cpp:635-1213                                                    */
/* ------------------------------------------------------------------------- */
static const double *pdk(const or_sim *s, int a, int b, long *kout);

void or_stale_a(const or_sim *s, double *t9) { memcpy(t9, s->tab, sizeof(double) * 9); }

/* index of stored pair (a,b), a<b */
static long pair_index(const or_sim *s, int a, int b)
{
    int Nm = s->p.Nm, Nc = s->p.Nc;
    long off = 0;
    if (a < Nm && b < Nm) {   /* AA (mm_HI only) */
        return (long)a * Nm - (long)a * (a + 1) / 2 + (b - a - 1);
    }
    if (s->p.mm_HI) off = (long)Nm * (Nm - 1) / 2;
    if (a < Nm) return off + (long)a * Nc + (b - Nm);
    off += (long)Nm * Nc;
    int ca = a - Nm, cb = b - Nm;
    return off + (long)ca * Nc - (long)ca * (ca + 1) / 2 + (cb - ca - 1);
}
static const double *pdk(const or_sim *s, int a, int b, long *kout)
{
    long k = pair_index(s, a, b);
    if (kout) *kout = k;
    return s->pd + 5 * k;
}

void or_mob(or_sim *s)
{
    int Nm = s->p.Nm, Nc = s->p.Nc;
    /* AB translational block for this call */
    if (s->p.ab_mode == OR_AB_REFERENCE && s->p.mm_HI) {
        int have = 0, li = -1, lj = -1;
        for (int i = Nm - 2; i >= 0 && !have; i--)
            for (int j = Nm - 1; j > i; j--)
                if (!(s->p.chain_HI && s->chain[i] == s->chain[j])) { li = i; lj = j; have = 1; break; }
        if (have) {
            const double *pd = pdk(s, li, lj, NULL);
            or_tensor_aa(pd[3], pd[4], pd, s->p.beta, s->p.aa_mode, s->stale);
        }
        memcpy(s->tab, s->stale, sizeof(double) * 9);
    } else if (s->p.ab_mode == OR_AB_REFERENCE) {
        memset(s->tab, 0, sizeof(double) * 9);
    }
    /* BB loop leaves mob_a = BB tensor of the last colloid pair (mob.cpp:1026-1029) */
    if (Nc >= 2) {
        const double *pd = pdk(s, Nm + Nc - 2, Nm + Nc - 1, NULL);
        double b[9], c[9], g[15], h[15], m[25];
        or_tensor_bb(pd[3], pd[4], pd, s->stale, b, c, g, h, m);
    }
    if (!s->p.mm_HI) {
        /* Mcm_block (mob.cpp:975-1024) */
        int nm3 = s->nm3, n11 = s->nc11;
        memset(s->Mcm, 0, sizeof(double) * n11 * nm3);
        for (int mI = 0; mI < Nm; mI++)
            for (int c = 0; c < Nc; c++) {
                const double *pd = pdk(s, mI, Nm + c, NULL);
                double b[9], g[15], a[9];
                or_tensor_ab(pd[3], pd[4], pd, s->p.beta, s->p.ab_mode == OR_AB_RPY_REG, b, g);
                if (s->p.ab_mode != OR_AB_REFERENCE)
                    or_tensor_ab_rpy(pd[3], pd[4], pd, s->p.beta, s->p.ab_mode == OR_AB_RPY_REG, a);
                else memset(a, 0, sizeof a);
                int t = 3 * c, r = s->nc3 + 3 * c, st = s->nc6 + 5 * c, col = 3 * mI;
                for (int i = 0; i < 3; i++) {
                    for (int j = 0; j < 3; j++) {
                        s->Mcm[(t + i) * nm3 + col + j] = a[j * 3 + i];
                        s->Mcm[(r + i) * nm3 + col + j] = b[i * 3 + j];
                    }
                    for (int j = 0; j < 5; j++) s->Mcm[(st + j) * nm3 + col + i] = g[i * 5 + j];
                }
            }
        /* colloid-colloid couplings: the reference's shell cannot hold them
         * (mob.cpp:1026-1144 writes into the MATSHELL A and aborts); here they
         * are added to the colloid block, as the dense path does. */
        double *Mb = s->Mcc_base; int n = s->nc11;
        for (int i = 0; i < n * n; i++) Mb[i] = 0.0;
        for (int c = 0; c < Nc; c++) {
            int t = 3 * c, r = s->nc3 + 3 * c, st = s->nc6 + 5 * c;
            for (int a = 0; a < 3; a++) { Mb[(t + a) * n + t + a] = 1.0; Mb[(r + a) * n + r + a] = 0.75; }
            for (int a = 0; a < 5; a++) Mb[(st + a) * n + st + a] = 9. / 5.;
            Mb[st * n + st + 4] = 9. / 10.; Mb[(st + 4) * n + st] = 9. / 10.;
        }
        for (int c1 = 0; c1 < Nc; c1++)
            for (int c2 = c1 + 1; c2 < Nc; c2++) {
                const double *pd = pdk(s, Nm + c1, Nm + c2, NULL);
                double A[9], B[9], C[9], G[15], H[15], Mm[25];
                or_tensor_bb(pd[3], pd[4], pd, A, B, C, G, H, Mm);
                int t1 = 3 * c1, t2 = 3 * c2, r1 = s->nc3 + 3 * c1, r2 = s->nc3 + 3 * c2;
                int s1 = s->nc6 + 5 * c1, s2 = s->nc6 + 5 * c2;
                for (int i = 0; i < 3; i++) {
                    for (int j = 0; j < 3; j++) {
                        Mb[(t1 + i) * n + t2 + j] = A[i * 3 + j];
                        Mb[(r1 + i) * n + t2 + j] = B[i * 3 + j];
                        Mb[(t2 + i) * n + r1 + j] = B[j * 3 + i];
                        Mb[(r1 + i) * n + r2 + j] = C[i * 3 + j];
                        Mb[(t2 + i) * n + t1 + j] = A[j * 3 + i];
                        Mb[(r2 + i) * n + t1 + j] = -B[j * 3 + i];
                        Mb[(t1 + i) * n + r2 + j] = -B[i * 3 + j];
                        Mb[(r2 + i) * n + r1 + j] = C[j * 3 + i];
                    }
                    for (int j = 0; j < 5; j++) {
                        Mb[(t1 + i) * n + s2 + j] = G[i * 5 + j]; Mb[(s2 + j) * n + t1 + i] = G[i * 5 + j];
                        Mb[(t2 + i) * n + s1 + j] = -G[i * 5 + j]; Mb[(s1 + j) * n + t2 + i] = -G[i * 5 + j];
                        Mb[(r1 + i) * n + s2 + j] = H[i * 5 + j]; Mb[(s2 + j) * n + r1 + i] = H[i * 5 + j];
                        Mb[(r2 + i) * n + s1 + j] = H[i * 5 + j]; Mb[(s1 + j) * n + r2 + i] = H[i * 5 + j];
                    }
                }
                for (int i = 0; i < 5; i++) for (int j = 0; j < 5; j++) {
                    Mb[(s1 + i) * n + s2 + j] = Mm[i * 5 + j];
                    Mb[(s2 + i) * n + s1 + j] = Mm[j * 5 + i];
                }
            }
        /* Mcc_block = Mcc_base (current positions) + Delta (last Schur sync) */
        for (int i = 0; i < n * n; i++) s->Mcc_block[i] = Mb[i] + s->Mcc_delta[i];
    }
}

/* ------------------------------------------------------------------------- */
/* symmetric eigendecomposition: cyclic Jacobi (stands in for LAPACK dsyev)   */
/* ------------------------------------------------------------------------- */
void or_jacobi_eig(double *A, int n, double *lam, double *Q)
{
    /* A is n x n row-major symmetric, destroyed; Q columns = eigenvectors */
    for (int i = 0; i < n; i++) for (int j = 0; j < n; j++) Q[i * n + j] = (i == j);
    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0, tot = 0;
        for (int i = 0; i < n; i++) for (int j = 0; j < n; j++) { double v = A[i * n + j] * A[i * n + j]; tot += v; if (i != j) off += v; }
        if (off <= 1e-30 * tot || off == 0.0) break;
        for (int p = 0; p < n - 1; p++)
            for (int q = p + 1; q < n; q++) {
                double apq = A[p * n + q];
                if (fabs(apq) < 1e-300) continue;
                double app = A[p * n + p], aqq = A[q * n + q];
                double theta = (aqq - app) / (2 * apq);
                double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1));
                double c = 1 / sqrt(t * t + 1), sn = t * c;
                for (int k = 0; k < n; k++) {
                    double akp = A[k * n + p], akq = A[k * n + q];
                    A[k * n + p] = c * akp - sn * akq; A[k * n + q] = sn * akp + c * akq;
                }
                for (int k = 0; k < n; k++) {
                    double apk = A[p * n + k], aqk = A[q * n + k];
                    A[p * n + k] = c * apk - sn * aqk; A[q * n + k] = sn * apk + c * aqk;
                }
                for (int k = 0; k < n; k++) {
                    double qkp = Q[k * n + p], qkq = Q[k * n + q];
                    Q[k * n + p] = c * qkp - sn * qkq; Q[k * n + q] = sn * qkp + c * qkq;
                }
            }
    }
    for (int i = 0; i < n; i++) lam[i] = A[i * n + i];
    /* sort ascending (selection), permuting columns of Q */
    for (int i = 0; i < n; i++) {
        int m = i;
        for (int j = i + 1; j < n; j++) if (lam[j] < lam[m]) m = j;
        if (m != i) {
            double t = lam[i]; lam[i] = lam[m]; lam[m] = t;
            for (int k = 0; k < n; k++) { double u = Q[k * n + i]; Q[k * n + i] = Q[k * n + m]; Q[k * n + m] = u; }
        }
    }
}

/* sync_mcc_schur_correction, slip_vel.cpp:81-203 */
void or_schur_sync(or_sim *s)
{
    if (s->p.mm_HI) return;
    int n = s->nc11, nm3 = s->nm3;
    int thr = s->p.lanczos_nc >= 0 ? s->p.lanczos_nc : 64;
    if (n > thr || n == 0) return;
    double *S = (double *)malloc(sizeof(double) * n * n);
    for (int a = 0; a < n; a++)
        for (int b = 0; b < n; b++) {
            double acc = 0;
            for (int k = 0; k < nm3; k++) acc += s->Mcm[a * nm3 + k] * s->Mcm[b * nm3 + k];
            S[a * n + b] = s->Mcc_base[a * n + b] - s->p.beta * acc;
        }
    double *lam = (double *)malloc(sizeof(double) * n);
    or_jacobi_eig(S, n, lam, s->schurQ);
    const double eps = 0.1;
    for (int a = 0; a < n; a++)
        for (int b = 0; b < n; b++) {
            double corr = 0;
            for (int j = 0; j < n; j++) {
                double d = lam[j] < eps ? eps - lam[j] : 0.0;
                if (d == 0.0) continue;
                corr += s->schurQ[a * n + j] * d * s->schurQ[b * n + j];
            }
            s->Mcc_delta[a * n + b] = corr;
            s->Mcc_block[a * n + b] = s->Mcc_base[a * n + b] + corr;
        }
    for (int j = 0; j < n; j++) s->schurL[j] = lam[j] < eps ? eps : lam[j];
    s->schur_valid = 1;
    free(S); free(lam);
}

/* ------------------------------------------------------------------------- */
/* grand mobility: dense form and matrix-free apply                          */
/* ------------------------------------------------------------------------- */
void or_mcm(const or_sim *s, double *Mcm) { memcpy(Mcm, s->Mcm, sizeof(double) * s->nc11 * s->nm3); }
void or_mcc(const or_sim *s, double *Mcc) { memcpy(Mcc, s->Mcc_block, sizeof(double) * s->nc11 * s->nc11); }

/* y = M u.  Dense-path blocks as written by mob.cpp:843-1144 / fill_self
 * mob.cpp:539-633; shell path as ArrowheadMult matfree_A.cpp:38-80. */
void or_mobility_apply(const or_sim *s, const double *u, double *y)
{
    int Nm = s->p.Nm, Nc = s->p.Nc, nm3 = s->nm3, n11 = s->nm3nc11;
    memset(y, 0, sizeof(double) * n11);
    for (int i = 0; i < nm3; i++) y[i] = s->beta_inv * u[i];
    if (!s->p.mm_HI) {
        const double *uc = u + nm3; double *yc = y + nm3;
        int nc = s->nc11;
        for (int a = 0; a < nc; a++) {
            double acc = 0;
            for (int k = 0; k < nm3; k++) acc += s->Mcm[a * nm3 + k] * u[k];
            for (int b = 0; b < nc; b++) acc += s->Mcc_block[a * nc + b] * uc[b];
            yc[a] += acc;
        }
        for (int k = 0; k < nm3; k++) {
            double acc = 0;
            for (int a = 0; a < nc; a++) acc += s->Mcm[a * nm3 + k] * uc[a];
            y[k] += acc;
        }
        return;
    }
    /* mm_HI: self colloid blocks */
    for (int c = 0; c < Nc; c++) {
        int t = nm3 + 3 * c, r = nm3 + s->nc3 + 3 * c, st = s->nm3nc6 + 5 * c;
        for (int a = 0; a < 3; a++) { y[t + a] += u[t + a]; y[r + a] += 0.75 * u[r + a]; }
        for (int a = 0; a < 5; a++) y[st + a] += (9. / 5.) * u[st + a];
        y[st] += (9. / 10.) * u[st + 4]; y[st + 4] += (9. / 10.) * u[st];
    }
    /* AA */
    for (int i = 0; i < Nm; i++)
        for (int j = i + 1; j < Nm; j++) {
            if (s->p.chain_HI && s->chain[i] == s->chain[j]) continue;
            const double *pd = pdk(s, i, j, NULL);
            double A[9]; or_tensor_aa(pd[3], pd[4], pd, s->p.beta, s->p.aa_mode, A);
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++) {
                    y[3 * i + a] += A[a * 3 + b] * u[3 * j + b];
                    y[3 * j + a] += A[b * 3 + a] * u[3 * i + b];
                }
        }
    /* AB */
    for (int m = 0; m < Nm; m++)
        for (int c = 0; c < Nc; c++) {
            const double *pd = pdk(s, m, Nm + c, NULL);
            double B[9], G[15], T[9];
            or_tensor_ab(pd[3], pd[4], pd, s->p.beta, s->p.ab_mode == OR_AB_RPY_REG, B, G);
            if (s->p.ab_mode != OR_AB_REFERENCE)
                or_tensor_ab_rpy(pd[3], pd[4], pd, s->p.beta, s->p.ab_mode == OR_AB_RPY_REG, T);
            else memcpy(T, s->tab, sizeof T);
            int mm = 3 * m, t = nm3 + 3 * c, r = nm3 + s->nc3 + 3 * c, st = s->nm3nc6 + 5 * c;
            for (int a = 0; a < 3; a++) {
                for (int b = 0; b < 3; b++) {
                    y[mm + a] += T[a * 3 + b] * u[t + b];
                    y[t + a] += T[b * 3 + a] * u[mm + b];
                    y[r + a] += B[a * 3 + b] * u[mm + b];
                    y[mm + a] += B[b * 3 + a] * u[r + b];
                }
                for (int b = 0; b < 5; b++) {
                    y[mm + a] += G[a * 5 + b] * u[st + b];
                    y[st + b] += G[a * 5 + b] * u[mm + a];
                }
            }
        }
    /* BB */
    for (int c1 = 0; c1 < Nc; c1++)
        for (int c2 = c1 + 1; c2 < Nc; c2++) {
            const double *pd = pdk(s, Nm + c1, Nm + c2, NULL);
            double A[9], B[9], C[9], G[15], H[15], Mm[25];
            or_tensor_bb(pd[3], pd[4], pd, A, B, C, G, H, Mm);
            int t1 = nm3 + 3 * c1, t2 = nm3 + 3 * c2, r1 = nm3 + s->nc3 + 3 * c1, r2 = nm3 + s->nc3 + 3 * c2;
            int s1 = s->nm3nc6 + 5 * c1, s2 = s->nm3nc6 + 5 * c2;
            for (int i = 0; i < 3; i++) {
                for (int j = 0; j < 3; j++) {
                    y[t1 + i] += A[i * 3 + j] * u[t2 + j];
                    y[r1 + i] += B[i * 3 + j] * u[t2 + j];
                    y[t2 + i] += B[j * 3 + i] * u[r1 + j];
                    y[r1 + i] += C[i * 3 + j] * u[r2 + j];
                    y[t2 + i] += A[j * 3 + i] * u[t1 + j];
                    y[r2 + i] += -B[j * 3 + i] * u[t1 + j];
                    y[t1 + i] += -B[i * 3 + j] * u[r2 + j];
                    y[r2 + i] += C[j * 3 + i] * u[r1 + j];
                }
                for (int j = 0; j < 5; j++) {
                    y[t1 + i] += G[i * 5 + j] * u[s2 + j]; y[s2 + j] += G[i * 5 + j] * u[t1 + i];
                    y[t2 + i] += -G[i * 5 + j] * u[s1 + j]; y[s1 + j] += -G[i * 5 + j] * u[t2 + i];
                    y[r1 + i] += H[i * 5 + j] * u[s2 + j]; y[s2 + j] += H[i * 5 + j] * u[r1 + i];
                    y[r2 + i] += H[i * 5 + j] * u[s1 + j]; y[s1 + j] += H[i * 5 + j] * u[r2 + i];
                }
            }
            for (int i = 0; i < 5; i++) for (int j = 0; j < 5; j++) {
                y[s1 + i] += Mm[i * 5 + j] * u[s2 + j];
                y[s2 + i] += Mm[j * 5 + i] * u[s1 + j];
            }
        }
}

void or_dense_mobility(const or_sim *s, double *M)
{
    int n = s->nm3nc11;
    double *u = (double *)calloc(n, sizeof(double)), *y = (double *)malloc(sizeof(double) * n);
    for (int j = 0; j < n; j++) {
        u[j] = 1.0;
        or_mobility_apply(s, u, y);
        for (int i = 0; i < n; i++) M[i * n + j] = y[i];
        u[j] = 0.0;
    }
    free(u); free(y);
}

/* ------------------------------------------------------------------------- */
/* lubrication (absent from the reference).  Equal-radius pairs only (monomer */
/* pairs of radius beta, colloid pairs of radius 1) with gap < lub_gap * a.   */
/* Table columns (r2babc.dat): r, X11A X12A Y11A Y12A Y11B Y12B X11C X12C     */
/* Y11C Y12C, each the two-body resistance minus the inverted far-field       */
/* two-body mobility, normalised by 6 pi mu a (A), 4 pi mu a^2 (B),           */
/* 8 pi mu a^3 (C).  Below the first table row (xi < 0.1) the leading         */
/* singular terms of Jeffrey & Onishi (1984) are added on top of the value at */
/* r = 2.1; xi is clamped at 1e-4.                                            */
/* ------------------------------------------------------------------------- */
#define LUB_XI_MIN 1e-4
static double lub_sing(int col, double xi)
{
    double l = log(xi);
    switch (col) {
    case 0: return 1.0 / (4.0 * xi) - (9.0 / 40.0) * l;   /* X11A */
    case 1: return -(1.0 / (4.0 * xi) - (9.0 / 40.0) * l);/* X12A */
    case 2: return -(1.0 / 6.0) * l;                      /* Y11A */
    case 3: return (1.0 / 6.0) * l;                       /* Y12A */
    case 4: return (1.0 / 4.0) * l;                       /* Y11B */
    case 5: return -(1.0 / 4.0) * l;                      /* Y12B */
    case 8: return -(1.0 / 5.0) * l;                      /* Y11C */
    case 9: return -(1.0 / 20.0) * l;                     /* Y12C */
    default: return 0.0;                                  /* X11C, X12C bounded */
    }
}
static void lub_scalars(const or_sim *s, double rr, double f[10])
{
    /* rr = r / a */
    const double *T = s->lub; int nr = s->lub_nrow;
    double r0 = T[0], rl = T[(nr - 1) * 11];
    if (rr >= rl) { for (int c = 0; c < 10; c++) f[c] = 0.0; return; }
    if (rr <= r0) {
        double xi = rr - 2.0; if (xi < LUB_XI_MIN) xi = LUB_XI_MIN;
        double xi0 = r0 - 2.0;
        for (int c = 0; c < 10; c++) f[c] = T[1 + c] + lub_sing(c, xi) - lub_sing(c, xi0);
        return;
    }
    int k = 0;
    while (k + 1 < nr && T[(k + 1) * 11] <= rr) k++;
    if (k >= nr - 1) k = nr - 2;
    double ra = T[k * 11], rb = T[(k + 1) * 11], w = (rr - ra) / (rb - ra);
    for (int c = 0; c < 10; c++) f[c] = (1 - w) * T[k * 11 + 1 + c] + w * T[(k + 1) * 11 + 1 + c];
}
int or_lub_pairs(const or_sim *s, int *pi, int *pj, int maxp)
{
    int cnt = 0, Nm = s->p.Nm, Np = s->Np;
    if (!s->p.lub_on || !s->lub) return 0;
    for (int i = 0; i < Np; i++)
        for (int j = i + 1; j < Np; j++) {
            int mi = i < Nm, mj = j < Nm;
            if (mi != mj) continue;
            /* bonded chain neighbours (init.cpp:205-321 topology) only with lub_bonded */
            if (mi && !s->p.lub_bonded && i / s->p.Nmono_per_chain == j / s->p.Nmono_per_chain && j == i + 1) continue;
            double a = mi ? s->p.beta : 1.0;
            double dx = s->x[3 * i] - s->x[3 * j], dy = s->x[3 * i + 1] - s->x[3 * j + 1], dz = s->x[3 * i + 2] - s->x[3 * j + 2];
            min_image(s, &dx, &dy, &dz);
            double r = sqrt(dx * dx + dy * dy + dz * dz);
            if (r - 2 * a < s->p.lub_gap * a) { if (cnt < maxp) { pi[cnt] = i; pj[cnt] = j; } cnt++; }
        }
    return cnt;
}
/* 12x12 (colloids: U1,U2,W1,W2) or 6x6 (monomers: U1,U2) pair block; d = (x2-x1)/r */
static int lub_block(const or_sim *s, int i, int j, double *R, int *dof)
{
    int Nm = s->p.Nm, mono = i < Nm;
    double a = mono ? s->p.beta : 1.0;
    double dx = s->x[3 * j] - s->x[3 * i], dy = s->x[3 * j + 1] - s->x[3 * i + 1], dz = s->x[3 * j + 2] - s->x[3 * i + 2];
    min_image(s, &dx, &dy, &dz);
    double r = sqrt(dx * dx + dy * dy + dz * dz), d[3] = {dx / r, dy / r, dz / r};
    double f[10]; lub_scalars(s, r / a, f);
    double sa = a, sb = (2.0 / 3.0) * a * a, sc = (4.0 / 3.0) * a * a * a;
    int nd = mono ? 6 : 12;
    for (int k = 0; k < nd * nd; k++) R[k] = 0.0;
    /* A blocks */
    for (int p = 0; p < 3; p++) for (int q = 0; q < 3; q++) {
        double dd = d[p] * d[q], id = (p == q) - dd;
        double a11 = sa * (f[0] * dd + f[2] * id), a12 = sa * (f[1] * dd + f[3] * id);
        R[(0 + p) * nd + 0 + q] = a11; R[(3 + p) * nd + 3 + q] = a11;
        R[(0 + p) * nd + 3 + q] = a12; R[(3 + p) * nd + 0 + q] = a12;
    }
    if (!mono) {
        for (int p = 0; p < 3; p++) for (int q = 0; q < 3; q++) {
            int k = third(p, q);
            double ed = (double)EPS3[p][q][k] * d[k];
            /* B_11 = Y11B eps.d, B_12 = Y12B eps.d, B_21 = -Y12B eps.d, B_22 = -Y11B eps.d */
            double b11 = sb * f[4] * ed, b12 = sb * f[5] * ed, b21 = -b12, b22 = -b11;
            /* torque rows (W1 at 6, W2 at 9) x velocity cols */
            R[(6 + p) * nd + 0 + q] = b11; R[(6 + p) * nd + 3 + q] = b12;
            R[(9 + p) * nd + 0 + q] = b21; R[(9 + p) * nd + 3 + q] = b22;
            /* transpose: force rows x rotation cols */
            R[(0 + q) * nd + 6 + p] = b11; R[(3 + q) * nd + 6 + p] = b12;
            R[(0 + q) * nd + 9 + p] = b21; R[(3 + q) * nd + 9 + p] = b22;
            double dd = d[p] * d[q], id = (p == q) - dd;
            double c11 = sc * (f[6] * dd + f[8] * id), c12 = sc * (f[7] * dd + f[9] * id);
            R[(6 + p) * nd + 6 + q] = c11; R[(9 + p) * nd + 9 + q] = c11;
            R[(6 + p) * nd + 9 + q] = c12; R[(9 + p) * nd + 6 + q] = c12;
        }
    }
    /* DOF indices in the velocity vector [U_m | U_c | W_c] */
    if (mono) {
        for (int k = 0; k < 3; k++) { dof[k] = 3 * i + k; dof[3 + k] = 3 * j + k; }
    } else {
        int c1 = i - Nm, c2 = j - Nm;
        for (int k = 0; k < 3; k++) {
            dof[k] = s->nm3 + 3 * c1 + k; dof[3 + k] = s->nm3 + 3 * c2 + k;
            dof[6 + k] = s->nm3nc3 + 3 * c1 + k; dof[9 + k] = s->nm3nc3 + 3 * c2 + k;
        }
    }
    return nd;
}
void or_lub_apply(const or_sim *s, const double *u, double *y)
{
    memset(y, 0, sizeof(double) * s->nm3nc6);
    if (!s->p.lub_on || !s->lub) return;
    int np = or_lub_pairs(s, NULL, NULL, 0);
    int *pi = (int *)malloc(sizeof(int) * (np + 1)), *pj = (int *)malloc(sizeof(int) * (np + 1));
    or_lub_pairs(s, pi, pj, np);
    double R[144]; int dof[12];
    for (int k = 0; k < np; k++) {
        int nd = lub_block(s, pi[k], pj[k], R, dof);
        for (int a = 0; a < nd; a++) {
            double acc = 0;
            for (int b = 0; b < nd; b++) acc += R[a * nd + b] * u[dof[b]];
            y[dof[a]] += acc;
        }
    }
    free(pi); free(pj);
}
/* y_bot += scale * sum_p R_p^{1/2} z_p, z packed per pair (6 or 12 entries) */
static void lub_noise(const or_sim *s, const double *z, double scale, double *ybot)
{
    int np = or_lub_pairs(s, NULL, NULL, 0);
    int *pi = (int *)malloc(sizeof(int) * (np + 1)), *pj = (int *)malloc(sizeof(int) * (np + 1));
    or_lub_pairs(s, pi, pj, np);
    double R[144], w[12]; int dof[12];
    for (int k = 0; k < np; k++) {
        /* 12 normals per pair (monomer pairs use the first 6) */
        int nd = lub_block(s, pi[k], pj[k], R, dof);
        or_sqrtm_eig(R, nd, z + 12L * k, w);
        for (int a = 0; a < nd; a++) ybot[dof[a]] += scale * w[a];
    }
    free(pi); free(pj);
}

/* saddle operator y = A x with A = [[M, B], [B^T, -R_lub]], B = [-I; 0]
 * (arrays.cpp:349-369, matfree_A.cpp:38-80) */
void or_saddle_apply(const or_sim *s, const double *x, double *y)
{
    int n11 = s->nm3nc11, n6 = s->nm3nc6;
    or_mobility_apply(s, x, y);
    for (int i = 0; i < n6; i++) y[i] -= x[n11 + i];
    for (int i = 0; i < n6; i++) y[n11 + i] = -x[i];
    if (s->p.lub_on && s->lub) {
        double *t = (double *)malloc(sizeof(double) * n6);
        or_lub_apply(s, x + n11, t);
        for (int i = 0; i < n6; i++) y[n11 + i] -= t[i];
        free(t);
    }
}

/* Jacobi diagonal (matfree_A.cpp:84-102 + PCJacobiSetFixDiagonal, init.cpp:236);
 * with lubrication the constraint-block entries are |diag(-R_lub)| */
void or_saddle_diag(const or_sim *s, double *d)
{
    int n11 = s->nm3nc11, n6 = s->nm3nc6, nm3 = s->nm3;
    for (int i = 0; i < nm3; i++) d[i] = s->beta_inv;
    if (!s->p.mm_HI) {
        for (int i = 0; i < s->nc11; i++) d[nm3 + i] = s->Mcc_block[i * s->nc11 + i];
    } else {
        for (int c = 0; c < s->p.Nc; c++) {
            for (int a = 0; a < 3; a++) { d[nm3 + 3 * c + a] = 1.0; d[nm3 + s->nc3 + 3 * c + a] = 0.75; }
            for (int a = 0; a < 5; a++) d[s->nm3nc6 + 5 * c + a] = 9. / 5.;
        }
    }
    for (int i = 0; i < n6; i++) d[n11 + i] = 0.0;
    if (s->p.lub_on && s->lub) {
        double *e = (double *)calloc(n6, sizeof(double)), *t = (double *)malloc(sizeof(double) * n6);
        for (int i = 0; i < n6; i++) { e[i] = 1.0; or_lub_apply(s, e, t); d[n11 + i] = fabs(t[i]); e[i] = 0.0; }
        free(e); free(t);
    }
    for (int i = 0; i < s->n; i++) if (d[i] == 0.0) d[i] = 1.0;
}

/* ------------------------------------------------------------------------- */
/* preconditioned MINRES (PETSc KSPMINRES semantics; Paige & Saunders 1975).  */
/* Convergence: ||B r0||_2 * prod|s_k| < rtol * ref with ref = ||B r0|| for a  */
/* zero guess, ||B b|| for a nonzero guess (PETSc KSPConvergedDefault).       */
/* Returns >0 converged, <0 diverged/max-it (PETSc reason sign convention).   */
/* ------------------------------------------------------------------------- */
static double dot(const double *a, const double *b, int n) { double s = 0; for (int i = 0; i < n; i++) s += a[i] * b[i]; return s; }

int or_minres(const or_sim *s, const double *b, double *x, int warm, double rtol, int maxit,
              int *iters, double *rnorm)
{
    int n = s->n;
    double *D = (double *)malloc(sizeof(double) * n);
    or_saddle_diag(s, D);
    double *r1 = (double *)malloc(sizeof(double) * n), *r2 = (double *)malloc(sizeof(double) * n);
    double *y = (double *)malloc(sizeof(double) * n), *v = (double *)malloc(sizeof(double) * n);
    double *w = (double *)calloc(n, sizeof(double)), *w1 = (double *)calloc(n, sizeof(double)), *w2 = (double *)calloc(n, sizeof(double));
    if (warm) {
        or_saddle_apply(s, x, y);
        for (int i = 0; i < n; i++) r1[i] = b[i] - y[i];
    } else {
        for (int i = 0; i < n; i++) { x[i] = 0.0; r1[i] = b[i]; }
    }
    for (int i = 0; i < n; i++) y[i] = r1[i] / D[i];
    double np0 = sqrt(dot(y, y, n));
    double ref = np0;
    if (warm) { double acc = 0; for (int i = 0; i < n; i++) { double z = b[i] / D[i]; acc += z * z; } ref = sqrt(acc); }
    double ttol = rtol * ref; if (ttol < 1e-50) ttol = 1e-50;
    double beta1 = dot(r1, y, n);
    int reason = 0, k = 0;
    double np = np0;
    if (beta1 < 0) { reason = -8; goto done; }
    beta1 = sqrt(beta1);
    if (np0 <= ttol || beta1 == 0.0) { reason = 2; goto done; }
    memcpy(r2, r1, sizeof(double) * n);
    double oldb = 0, beta = beta1, dbar = 0, epsln = 0, phibar = beta1, cs = -1, sn = 0;
    for (k = 1; k <= maxit; k++) {
        double sinv = 1.0 / beta;
        for (int i = 0; i < n; i++) v[i] = sinv * y[i];
        or_saddle_apply(s, v, y);
        if (k >= 2) for (int i = 0; i < n; i++) y[i] -= (beta / oldb) * r1[i];
        double alfa = dot(v, y, n);
        for (int i = 0; i < n; i++) y[i] -= (alfa / beta) * r2[i];
        double *t = r1; r1 = r2; r2 = t;
        memcpy(r2, y, sizeof(double) * n);
        for (int i = 0; i < n; i++) y[i] = r2[i] / D[i];
        oldb = beta;
        double bb = dot(r2, y, n);
        if (bb < 0) { reason = -8; break; }
        beta = sqrt(bb);
        double oldeps = epsln;
        double delta = cs * dbar + sn * alfa;
        double gbar = sn * dbar - cs * alfa;
        epsln = sn * beta;
        dbar = -cs * beta;
        double gamma = sqrt(gbar * gbar + beta * beta);
        if (gamma < DBL_MIN) gamma = DBL_MIN;
        cs = gbar / gamma; sn = beta / gamma;
        double phi = cs * phibar; phibar = sn * phibar;
        double denom = 1.0 / gamma;
        double *tt = w1; w1 = w2; w2 = w; w = tt;   /* w1 <- w2, w2 <- w */
        for (int i = 0; i < n; i++) w[i] = (v[i] - oldeps * w1[i] - delta * w2[i]) * denom;
        for (int i = 0; i < n; i++) x[i] += phi * w[i];
        np = np * fabs(sn);
        if (np <= ttol) { reason = 2; break; }
        if (beta == 0.0) { reason = 3; break; }
    }
    if (k > maxit) { reason = -3; k = maxit; }
done:
    if (iters) *iters = k;
    if (rnorm) *rnorm = np;
    free(D); free(r1); free(r2); free(y); free(v); free(w); free(w1); free(w2);
    return reason;
}

/* ------------------------------------------------------------------------- */
/* matrix square roots                                                         */
/* ------------------------------------------------------------------------- */
void or_sqrtm_eig(const double *M, int n, const double *z, double *w)
{
    double *A = (double *)malloc(sizeof(double) * n * n), *Q = (double *)malloc(sizeof(double) * n * n);
    double *lam = (double *)malloc(sizeof(double) * n), *t = (double *)malloc(sizeof(double) * n);
    memcpy(A, M, sizeof(double) * n * n);
    or_jacobi_eig(A, n, lam, Q);
    for (int j = 0; j < n; j++) {
        double acc = 0; for (int i = 0; i < n; i++) acc += Q[i * n + j] * z[i];
        t[j] = (lam[j] > 0 ? sqrt(lam[j]) : 0.0) * acc;
    }
    for (int i = 0; i < n; i++) { double acc = 0; for (int j = 0; j < n; j++) acc += Q[i * n + j] * t[j]; w[i] = acc; }
    free(A); free(Q); free(lam); free(t);
}

/* Lanczos sqrt(M) z with full two-pass reorthogonalisation and a floor of 0 on
 * the projected spectrum (the policy of schur_sqrt_lanczos, slip_vel.cpp:351-477),
 * applied to the full grand mobility.  Stops when successive estimates differ
 * by less than tol (relative) or at kmax.  Returns the subspace size used. */
int or_lanczos_sqrt(const or_sim *s, const double *z, double *w, int kmax, double tol)
{
    int n = s->nm3nc11;
    double b0 = sqrt(dot(z, z, n));
    if (b0 == 0.0) { memset(w, 0, sizeof(double) * n); return 0; }
    if (kmax > n) kmax = n;
    double *V = (double *)malloc(sizeof(double) * (size_t)n * (kmax + 1));
    double *al = (double *)calloc(kmax + 1, sizeof(double)), *be = (double *)calloc(kmax + 1, sizeof(double));
    double *q = (double *)malloc(sizeof(double) * n);
    double *wprev = (double *)calloc(n, sizeof(double));
    double *T = (double *)malloc(sizeof(double) * kmax * kmax), *Q = (double *)malloc(sizeof(double) * kmax * kmax);
    double *lam = (double *)malloc(sizeof(double) * kmax), *g = (double *)malloc(sizeof(double) * kmax);
    for (int i = 0; i < n; i++) V[i] = z[i] / b0;
    int m = 0;
    for (int j = 0; j < kmax; j++) {
        double *vj = V + (size_t)j * n;
        or_mobility_apply(s, vj, q);
        if (j > 0) for (int i = 0; i < n; i++) q[i] -= be[j - 1] * V[(size_t)(j - 1) * n + i];
        al[j] = dot(vj, q, n);
        for (int i = 0; i < n; i++) q[i] -= al[j] * vj[i];
        for (int pass = 0; pass < 2; pass++)
            for (int i = 0; i <= j; i++) {
                double h = dot(V + (size_t)i * n, q, n);
                for (int k = 0; k < n; k++) q[k] -= h * V[(size_t)i * n + k];
            }
        m = j + 1;
        /* estimate with the current subspace */
        for (int a = 0; a < m * m; a++) T[a] = 0;
        for (int a = 0; a < m; a++) T[a * m + a] = al[a];
        for (int a = 0; a < m - 1; a++) { T[a * m + a + 1] = be[a]; T[(a + 1) * m + a] = be[a]; }
        or_jacobi_eig(T, m, lam, Q);
        for (int a = 0; a < m; a++) {
            double acc = 0;
            for (int c = 0; c < m; c++) acc += Q[a * m + c] * (lam[c] > 0 ? sqrt(lam[c]) : 0.0) * Q[0 * m + c];
            g[a] = b0 * acc;
        }
        double diff = 0, nrm = 0;
        for (int i = 0; i < n; i++) {
            double acc = 0;
            for (int a = 0; a < m; a++) acc += g[a] * V[(size_t)a * n + i];
            diff += (acc - wprev[i]) * (acc - wprev[i]); nrm += acc * acc; wprev[i] = acc;
        }
        double bj = sqrt(dot(q, q, n));
        if (j > 0 && sqrt(diff) <= tol * sqrt(nrm)) break;
        if (bj <= 1e-12 * b0 || j == kmax - 1) break;
        be[j] = bj;
        for (int i = 0; i < n; i++) V[(size_t)(j + 1) * n + i] = q[i] / bj;
    }
    memcpy(w, wprev, sizeof(double) * n);
    free(V); free(al); free(be); free(q); free(wprev); free(T); free(Q); free(lam); free(g);
    return m;
}

/* solve_slip_vel up to the scaling, slip_vel.cpp:19-79 / 205-349 */
void or_slip_noise(or_sim *s, const double *fb, double *W)
{
    int n = s->nm3nc11, nm3 = s->nm3, nc = s->nc11;
    if (s->p.mm_HI && s->p.noise_lanczos) {
        or_lanczos_sqrt(s, fb, W, 40, 1e-6);
        return;
    }
    if (s->p.mm_HI) {
        double *M = (double *)malloc(sizeof(double) * n * n);
        or_dense_mobility(s, M);
        or_sqrtm_eig(M, n, fb, W);
        free(M);
        return;
    }
    /* block-Cholesky: u_m = sqrt(beta_inv) xi_m; u_c = sqrt(beta) Mcm xi_m + S^1/2 xi_c */
    for (int i = 0; i < nm3; i++) W[i] = sqrt(s->beta_inv) * fb[i];
    double *uc = W + nm3;
    for (int a = 0; a < nc; a++) {
        double acc = 0; for (int k = 0; k < nm3; k++) acc += s->Mcm[a * nm3 + k] * fb[k];
        uc[a] = acc * sqrt(s->p.beta);
    }
    int thr = s->p.lanczos_nc >= 0 ? s->p.lanczos_nc : 64;
    if (nc > thr) {
        /* schur_sqrt_lanczos, slip_vel.cpp:351-477: S q = Mcc q - beta Mcm (Mcm^T q) applied
         * matrix-free; k <= min(40, nc11) vectors, two-pass reorthogonalisation, stop on an
         * invariant subspace (||w|| <= 1e-12 ||b||) or the cap; sqrt of the projected
         * tridiagonal with negative eigenvalues floored at 0. */
        const double *b = fb + nm3;
        double b0 = sqrt(dot(b, b, nc));
        if (b0 > 0.0) {
            int kmax = nc < 40 ? nc : 40;
            double *V = (double *)malloc(sizeof(double) * (size_t)nc * kmax);
            double *w = (double *)malloc(sizeof(double) * nc), *tm = (double *)malloc(sizeof(double) * nm3 + 8);
            double *al = (double *)calloc(kmax, sizeof(double)), *be = (double *)calloc(kmax, sizeof(double));
            for (int i = 0; i < nc; i++) V[i] = b[i] / b0;
            int m = 0;
            for (int j = 0; j < kmax; j++) {
                const double *qj = V + (size_t)j * nc;
                for (int k = 0; k < nm3; k++) {
                    double acc = 0; for (int a = 0; a < nc; a++) acc += s->Mcm[a * nm3 + k] * qj[a];
                    tm[k] = acc;
                }
                for (int a = 0; a < nc; a++) {
                    double sq = 0; for (int k = 0; k < nm3; k++) sq += s->Mcm[a * nm3 + k] * tm[k];
                    double cq = 0; for (int c = 0; c < nc; c++) cq += s->Mcc_block[a * nc + c] * qj[c];
                    w[a] = cq - s->p.beta * sq;
                }
                if (j > 0) for (int a = 0; a < nc; a++) w[a] -= be[j - 1] * V[(size_t)(j - 1) * nc + a];
                al[j] = dot(qj, w, nc);
                for (int a = 0; a < nc; a++) w[a] -= al[j] * qj[a];
                for (int pass = 0; pass < 2; pass++)
                    for (int i = 0; i <= j; i++) {
                        double h = dot(V + (size_t)i * nc, w, nc);
                        for (int a = 0; a < nc; a++) w[a] -= h * V[(size_t)i * nc + a];
                    }
                m = j + 1;
                double bj = sqrt(dot(w, w, nc));
                if (bj <= 1e-12 * b0 || j == kmax - 1) break;
                be[j] = bj;
                for (int a = 0; a < nc; a++) V[(size_t)(j + 1) * nc + a] = w[a] / bj;
            }
            double *T = (double *)calloc((size_t)m * m, sizeof(double)), *Q = (double *)malloc(sizeof(double) * m * m);
            double *lam = (double *)malloc(sizeof(double) * m);
            for (int a = 0; a < m; a++) T[a * m + a] = al[a];
            for (int a = 0; a + 1 < m; a++) { T[a * m + a + 1] = be[a]; T[(a + 1) * m + a] = be[a]; }
            or_jacobi_eig(T, m, lam, Q);
            for (int a = 0; a < m; a++) {
                double g = 0;
                for (int c = 0; c < m; c++) g += Q[a * m + c] * (lam[c] > 0 ? sqrt(lam[c]) : 0.0) * Q[0 * m + c];
                g *= b0;
                for (int i = 0; i < nc; i++) uc[i] += g * V[(size_t)a * nc + i];
            }
            free(V); free(w); free(tm); free(al); free(be); free(T); free(Q); free(lam);
        }
    } else {
        const double *Q = s->schurQ;
        double *yv = (double *)malloc(sizeof(double) * (size_t)(nc > 0 ? nc : 1));
        for (int j = 0; j < nc; j++) {
            double acc = 0; for (int i = 0; i < nc; i++) acc += Q[i * nc + j] * fb[nm3 + i];
            yv[j] = sqrt(s->schurL[j]) * acc;
        }
        for (int i = 0; i < nc; i++) { double acc = 0; for (int j = 0; j < nc; j++) acc += Q[i * nc + j] * yv[j]; uc[i] += acc; }
        free(yv);
    }
}

/* ------------------------------------------------------------------------- */
/* one step, run.cpp:70-162, drift.cpp:17-62, traj.cpp:9-94, quat.cpp:40-54  */
/* ------------------------------------------------------------------------- */
static void stage(or_sim *s, double *rhs)
{
    or_check_dist(s);
    or_rhs(s, 0, NULL, rhs);
    or_mob(s);
    or_schur_sync(s);
}

void or_step(or_sim *s, const double *fb, const double *wrfd, const double *zlub, double rtol, or_step_out *o)
{
    int n = s->n, n11 = s->nm3nc11, n6 = s->nm3nc6, n3 = s->n3;
    double *rhs = (double *)malloc(sizeof(double) * n), *X = (double *)malloc(sizeof(double) * n);
    double *Xd = (double *)calloc(n, sizeof(double));
    double *xn = (double *)malloc(sizeof(double) * n3);
    double *vdn = (double *)malloc(sizeof(double) * n6), *vdc = (double *)malloc(sizeof(double) * n6);
    double *vb = (double *)calloc(n6, sizeof(double)), *up = (double *)calloc(n6, sizeof(double));
    double *ud = (double *)calloc(n6, sizeof(double)), *drift = (double *)calloc(n6, sizeof(double));
    double *sb = (double *)calloc(s->nc5 ? s->nc5 : 1, sizeof(double));
    double *fext = (double *)calloc(n6, sizeof(double));
    int it[5] = {0, 0, 0, 0, 0}; double rn;
    double kT = s->p.kT, dt = s->p.dt, eps = 1.0e-3;

    s->t += dt;
    memcpy(xn, s->x, sizeof(double) * n3);
    stage(s, rhs);
    or_minres(s, rhs, X, 0, rtol, 100000, &it[0], &rn);
    memcpy(vdn, X + n11, sizeof(double) * n6);
    if (kT > 0) {
        double *W = (double *)malloc(sizeof(double) * n11);
        or_slip_noise(s, fb, W);
        double sc = sqrt(2 * kT / dt);
        for (int i = 0; i < n11; i++) rhs[i] += sc * W[i];
        if (s->p.lub_on && s->lub && zlub) lub_noise(s, zlub, -sc, rhs + n11);
        free(W);
        or_minres(s, rhs, X, 0, rtol, 100000, &it[1], &rn);
        memcpy(up, X + n11, sizeof(double) * n6);
        if (s->p.record_forces) memcpy(fext, X, sizeof(double) * n6);
        for (int k = 0; k < n6; k++) vb[k] = up[k] - vdn[k];
        /* drift.cpp:17-62 */
        memcpy(fext, wrfd, sizeof(double) * n6);
        for (int i = 0; i < n3; i++) s->x[i] += eps * fext[i];
        or_check_dist(s); or_mob(s); or_rhs(s, 1, fext, rhs);
        or_minres(s, rhs, Xd, 0, rtol, 100000, &it[2], &rn);
        memcpy(drift, Xd + n11, sizeof(double) * n6);
        memcpy(sb, Xd + s->nm3nc6, sizeof(double) * s->nc5);
        for (int i = 0; i < n3; i++) s->x[i] -= 2.0 * eps * fext[i];
        or_check_dist(s); or_mob(s); or_rhs(s, 1, fext, rhs);
        or_minres(s, rhs, Xd, 1, rtol, 100000, &it[3], &rn);
        for (int i = 0; i < n6; i++) ud[i] = Xd[n11 + i] - drift[i];
        for (int i = 0; i < s->nc5; i++) sb[i] = (sb[i] - Xd[s->nm3nc6 + i]) / (2 * eps);
    } else {
        or_minres(s, rhs, X, 0, rtol, 100000, &it[1], &rn);
        memcpy(up, X + n11, sizeof(double) * n6);
        if (s->p.record_forces) memcpy(fext, X, sizeof(double) * n6);
    }
    /* step(), traj.cpp:9-35 */
    if (kT > 0) {
        double ds = kT / (2.0 * eps);
        for (int i = 0; i < n3; i++) { s->x[i] += eps * fext[i]; s->x[i] += ds * ud[i] * dt; }
    }
    for (int i = 0; i < n3; i++) s->x[i] += up[i] * dt;
    for (int i = 0; i < n3; i += 3) wrap(s, s->x + i);
    /* corrector */
    stage(s, rhs);
    or_minres(s, rhs, X, 0, rtol, 100000, &it[4], &rn);
    memcpy(vdc, X + n11, sizeof(double) * n6);
    for (int k = 0; k < n6; k++) up[k] = 0.5 * (vdn[k] + vdc[k]) + vb[k];
    /* step_from, traj.cpp:37-62 */
    if (kT > 0) {
        double ds = kT / (2.0 * eps);
        for (int i = 0; i < n3; i++) s->x[i] = xn[i] + ds * ud[i] * dt + up[i] * dt;
    } else {
        for (int i = 0; i < n3; i++) s->x[i] = xn[i] + up[i] * dt;
    }
    for (int i = 0; i < n3; i += 3) wrap(s, s->x + i);
    /* step_quaternion, traj.cpp:64-94 / quat.cpp:7-54 */
    for (int c = 0; c < s->p.Nc; c++) {
        double *q = s->q + 4 * c, *om = up + s->nm3nc3 + 3 * c;
        double w1 = q[0], x1 = q[1], y1 = q[2], z1 = q[3];
        double w2 = 0.0, x2 = om[0], y2 = om[1], z2 = om[2];
        double d[4] = {w1 * w2 - x1 * x2 - y1 * y2 - z1 * z2, w1 * x2 + x1 * w2 + y1 * z2 - z1 * y2,
                       w1 * y2 - x1 * z2 + y1 * w2 + z1 * x2, w1 * z2 + x1 * y2 - y1 * x2 + z1 * w2};
        double qn[4];
        for (int a = 0; a < 4; a++) qn[a] = q[a] + 0.5 * d[a] * dt;
        double nr = sqrt(qn[0] * qn[0] + qn[1] * qn[1] + qn[2] * qn[2] + qn[3] * qn[3]);
        for (int a = 0; a < 4; a++) q[a] = qn[a] / nr;
    }
    if (o) {
        if (o->v_det_n) memcpy(o->v_det_n, vdn, sizeof(double) * n6);
        if (o->v_det_c) memcpy(o->v_det_c, vdc, sizeof(double) * n6);
        if (o->v_brown) memcpy(o->v_brown, vb, sizeof(double) * n6);
        if (o->up) memcpy(o->up, up, sizeof(double) * n6);
        if (o->udiff) memcpy(o->udiff, ud, sizeof(double) * n6);
        if (o->sb) memcpy(o->sb, sb, sizeof(double) * s->nc5);
        if (o->fext) memcpy(o->fext, fext, sizeof(double) * n6);
        memcpy(o->iters, it, sizeof it);
    }
    free(rhs); free(X); free(Xd); free(xn); free(vdn); free(vdc); free(vb); free(up); free(ud);
    free(drift); free(sb); free(fext);
}
