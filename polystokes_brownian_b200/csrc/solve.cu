// solve.cu -- structured saddle solves (PS_SOLVE_STRUCTURED).
//
// The saddle system of the reference (arrays.cpp:349-408, matfree_A.cpp:38-80)
//     [ M    B    ] [F]   [b_top]        B = [-I_{nm3nc6} ; 0]
//     [ B^T  -R   ] [U] = [b_bot]        R = R_lub (0 without lubrication)
// splits F = [F_t ; F_S] (forces/torques of every bead, then colloid stresslets).
//
// Without lubrication it is solved exactly by block elimination:
//     F_t = -b_bot                          (constraint rows)
//     M_SS F_S = b_S - M_St F_t             (dense nc5 x nc5 colloid-stresslet solve)
//     U = (M F)_t - b_t                     (velocity rows)
// which costs two operator applies instead of a Krylov iteration.  The solution
// is the same one MINRES converges to (it is the unique solution of the system).
//
// With lubrication the constraint rows couple U to the forces through R_lub;
// the system is solved in pair space by preconditioned CG (pair_solve below),
// with the same exact elimination of the stresslets and velocities around it.
//
// Replicas with more than 12 colloids (M_SS not solved densely) keep the
// stresslets as CG unknowns in the same solve.  Replicas whose CG breaks down
// because M is not positive definite (the reference's own monomer pair scalars
// make it indefinite) take the result as the warm start of a MINRES polish.
#include <cmath>
#include <vector>
#include "ps_internal.h"
#include "ps_kernels.h"
#include "ps_reduce.cuh"
#include "lub_dev.cuh"

namespace ps {

constexpr int SS_MAX = 64;   // dense stresslet block limit (nc5 <= 64: up to 12 colloids)

__device__ __forceinline__ int rep_at(const int *__restrict__ offs, int R, long k)
{
    int lo = 0, hi = R;
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (offs[mid] <= k) lo = mid; else hi = mid;
    }
    return lo;
}

// x = [F_t = -b_bot ; F_S = 0 ; U = 0]
__global__ void k_struct_init(long nvec, const int *__restrict__ vec_offs, int R, const Seg *__restrict__ segs,
                              const double *__restrict__ b, double *__restrict__ x)
{
    long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nvec) return;
    int r = rep_at(vec_offs, R, k);
    const Seg &s = segs[r];
    int i = (int)(k - s.vec_off);
    x[k] = (i < s.nm3nc6) ? -b[s.vec_off + s.nm3nc11 + i] : 0.0;
}

// entry (i, j) of M_SS: self + colloid pair stresslet blocks + the Schur
// correction of the shell path
__device__ double ss_entry(const Seg &s, const double *__restrict__ pos_x, const double *__restrict__ delta, int i, int j)
{
    double v = 0.0;
    int ci = i / 5, pi = i % 5, cj = j / 5, pj = j % 5;
    if (ci == cj) {
        if (pi == pj) v = 1.8;
        else if ((pi == 0 && pj == 4) || (pi == 4 && pj == 0)) v = 0.9;
    } else {
        bool lo = ci < cj;
        long bl = (long)s.bead_off + s.Nm + (lo ? ci : cj), bh = (long)s.bead_off + s.Nm + (lo ? cj : ci);
        double dx = pos_x[3 * bl] - pos_x[3 * bh], dy = pos_x[3 * bl + 1] - pos_x[3 * bh + 1];
        double dz = pos_x[3 * bl + 2] - pos_x[3 * bh + 2];
        double r2 = dx * dx + dy * dy + dz * dz, ri = rsqrt(r2);
        double e[3] = {dx * ri, dy * ri, dz * ri};
        double ri3 = ri * ri * ri, ri5 = ri3 * ri * ri;
        double Mm[25];
        mm_flat<double>(e, -4.5 * ri3 + 10.8 * ri5, 2.25 * ri3 - 7.2 * ri5, 1.8 * ri5, Mm);
        // row of the lower colloid uses Mm, row of the upper one Mm^T (mob.cpp:1129-1143)
        v = lo ? Mm[pi * 5 + pj] : Mm[pj * 5 + pi];
    }
    if (s.shell_schur) v += delta[s.schur_off + (long)(s.nc6 + i) * s.nc11 + (s.nc6 + j)];
    return v;
}

// one block per replica with colloids: assemble M_SS, solve
// M_SS F_S = b_S - y_S by Gaussian elimination with partial pivoting.
__global__ void k_struct_ss(const Seg *__restrict__ segs, const int *__restrict__ reps, const double *__restrict__ pos_x,
                            const double *__restrict__ delta, const double *__restrict__ b,
                            const double *__restrict__ y, double *__restrict__ x)
{
    __shared__ double A[SS_MAX][SS_MAX + 1];
    __shared__ int piv;
    const int r = reps[blockIdx.x];
    const Seg &s = segs[r];
    const int n = s.nc5;
    for (int t = threadIdx.x; t < n * (n + 1); t += blockDim.x) {
        int i = t / (n + 1), j = t % (n + 1);
        A[i][j] = (j == n) ? b[s.vec_off + s.nm3nc6 + i] - y[s.vec_off + s.nm3nc6 + i] : ss_entry(s, pos_x, delta, i, j);
    }
    __syncthreads();
    for (int k = 0; k < n; k++) {
        if (threadIdx.x == 0) {
            int p = k;
            double best = fabs(A[k][k]);
            for (int i = k + 1; i < n; i++)
                if (fabs(A[i][k]) > best) { best = fabs(A[i][k]); p = i; }
            piv = p;
        }
        __syncthreads();
        if (piv != k)
            for (int j = threadIdx.x; j <= n; j += blockDim.x) { double t = A[k][j]; A[k][j] = A[piv][j]; A[piv][j] = t; }
        __syncthreads();
        double akk = A[k][k];
        for (int t = threadIdx.x; t < (n - k - 1) * (n - k); t += blockDim.x) {
            int i = k + 1 + t / (n - k), j = k + 1 + t % (n - k);
            A[i][j] -= A[i][k] / akk * A[k][j];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        for (int i = n - 1; i >= 0; i--) {
            double v = A[i][n];
            for (int j = i + 1; j < n; j++) v -= A[i][j] * A[j][n];
            A[i][n] = v / A[i][i];
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) x[s.vec_off + s.nm3nc6 + i] = A[i][n];
}

// U = (M F)_t - b_t
__global__ void k_struct_u(long nvec, const int *__restrict__ vec_offs, int R, const Seg *__restrict__ segs,
                           const double *__restrict__ b, const double *__restrict__ y, double *__restrict__ x)
{
    long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nvec) return;
    int r = rep_at(vec_offs, R, k);
    const Seg &s = segs[r];
    int i = (int)(k - s.vec_off);
    if (i >= s.nm3nc11) {
        int j = i - s.nm3nc11;
        x[k] = y[s.vec_off + j] - b[s.vec_off + j];
    }
}

// ---------------------------------------------------------------------------
// lubricated resistance-form PCG

// inverse of M_SS per replica (LU with partial pivoting in shared memory, then
// one column of the inverse per thread); stored row-major at ssinv + s.ss_off
__global__ void k_ss_inverse(const Seg *__restrict__ segs, const int *__restrict__ reps, const double *__restrict__ pos_x,
                             const double *__restrict__ delta, double *__restrict__ ssinv)
{
    __shared__ double A[SS_MAX][SS_MAX + 1];
    __shared__ int perm[SS_MAX];
    __shared__ int piv;
    const Seg &s = segs[reps[blockIdx.x]];
    const int n = s.nc5;
    for (int t = threadIdx.x; t < n * n; t += blockDim.x) A[t / n][t % n] = ss_entry(s, pos_x, delta, t / n, t % n);
    for (int t = threadIdx.x; t < n; t += blockDim.x) perm[t] = t;
    __syncthreads();
    for (int k = 0; k < n; k++) {
        if (threadIdx.x == 0) {
            int p = k;
            double best = fabs(A[k][k]);
            for (int i = k + 1; i < n; i++)
                if (fabs(A[i][k]) > best) { best = fabs(A[i][k]); p = i; }
            piv = p;
            if (p != k) { int t = perm[k]; perm[k] = perm[p]; perm[p] = t; }
        }
        __syncthreads();
        if (piv != k)
            for (int j = threadIdx.x; j < n; j += blockDim.x) { double t = A[k][j]; A[k][j] = A[piv][j]; A[piv][j] = t; }
        __syncthreads();
        for (int i = k + 1 + threadIdx.x; i < n; i += blockDim.x) A[i][k] /= A[k][k];
        __syncthreads();
        for (int t = threadIdx.x; t < (n - k - 1) * (n - k - 1); t += blockDim.x) {
            int i = k + 1 + t / (n - k - 1), j = k + 1 + t % (n - k - 1);
            A[i][j] -= A[i][k] * A[k][j];
        }
        __syncthreads();
    }
    // column c of the inverse: solve L U x = P e_c
    for (int c = threadIdx.x; c < n; c += blockDim.x) {
        double xv[SS_MAX];
        for (int i = 0; i < n; i++) {
            double v = (perm[i] == c) ? 1.0 : 0.0;
            for (int j = 0; j < i; j++) v -= A[i][j] * xv[j];
            xv[i] = v;
        }
        for (int i = n - 1; i >= 0; i--) {
            double v = xv[i];
            for (int j = i + 1; j < n; j++) v -= A[i][j] * xv[j];
            xv[i] = v / A[i][i];
        }
        for (int i = 0; i < n; i++) ssinv[s.ss_off + (long)i * n + c] = xv[i];
    }
}

// out_S = M_SS^{-1} (ca a_S + cb b_S), one block per replica with a dense
// stresslet block; layouts: 0 saddle vector, 1 mobility vector
__global__ void k_ss_apply(const Seg *__restrict__ segs, const int *__restrict__ reps, const double *__restrict__ ssinv,
                           const double *__restrict__ a, int la, double ca, const double *__restrict__ b, int lb,
                           double cb, double *__restrict__ out, int lo, const char *__restrict__ done, int dstride)
{
    __shared__ double in[SS_MAX];
    const int r = reps[blockIdx.x];
    if (done && *(const int *)(done + (long)r * dstride)) return;
    const Seg &s = segs[r];
    const int n = s.nc5;
    const long oa = (la == 0 ? s.vec_off : s.top_off) + s.nm3nc6, ob = (lb == 0 ? s.vec_off : s.top_off) + s.nm3nc6;
    const long oo = (lo == 0 ? s.vec_off : s.top_off) + s.nm3nc6;
    for (int i = threadIdx.x; i < n; i += blockDim.x) in[i] = ca * a[oa + i] + (b ? cb * b[ob + i] : 0.0);
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double *row = ssinv + s.ss_off + (long)i * n;
        double v = 0.0;
        for (int j = 0; j < n; j++) v += row[j] * in[j];
        out[oo + i] = v;
    }
}

// reference norm ||D^{-1} b|| over the saddle vector; initial scalars
__global__ void k_pcg_start(RedTable T, const Seg *__restrict__ segs, const double *__restrict__ b,
                            const double *__restrict__ D, PcgScal *pc, double rtol)
{
    __shared__ double sh[RB_THREADS / 32][1];
    const RBlk B = T.d_blk[blockIdx.x];
    double v[1] = {0.0};
    for (int e = threadIdx.x; e < B.len; e += RB_THREADS) {
        double t = b[B.start + e] / D[B.start + e];
        v[0] += t * t;
    }
    block_sum<1>(v, sh);
    double tot[1];
    if (finish_block<1>(T, B, blockIdx.x, v, tot)) {
        const Seg &s = segs[B.rep];
        PcgScal p = {};
        p.tol = rtol * sqrt(tot[0]);
        (void)s;
        p.done = 0;
        p.reason = 0;
        pc[B.rep] = p;
    }
}

// g = b_tt - (M [0 ; M_SS^{-1} b_S])_t ; velocity-layout loops over the velocity table
__global__ void k_pcg_g(RedTable T, const Seg *__restrict__ segs, const double *__restrict__ b,
                        const double *__restrict__ y2, double *__restrict__ g)
{
    const RBlk B = T.d_blk[blockIdx.x];
    const Seg &s = segs[B.rep];
    for (int e = threadIdx.x; e < B.len; e += RB_THREADS) {
        long k = B.start + e;
        int j = (int)(k - s.vel_off);
        g[k] = b[s.vec_off + j] - (s.ss_off >= 0 ? y2[s.top_off + j] : 0.0);
    }
}

// ---------------------------------------------------------------------------
// Lubricated solve in pair space.  With R = L L^T, L = [B_p K_p^{1/2}] over the
// near pairs p (K_p the 12x12 pair block, B_p its velocity DOFs), the force
// unknowns are F_t = -b_bot + L y, and y solves the SPD system
//     (I + L^T Mr L) y = L^T (g + Mr b_bot),
// of dimension 12 per pair (from (I + R Mr) F_t = R g - b_bot: F_t + b_bot lies
// in the range of R; no term of the right-hand side carries the pair stiffness,
// so the FP32 far field is not amplified by it).  CG is preconditioned
// block-diagonally with (I + K_p^{1/2} M_pp K_p^{1/2})^{-1}, M_pp the pair's own
// two-body FT mobility (self + pair blocks of the far field): the stiff squeeze
// and shear modes of each near pair are resolved by its block, the far-field
// coupling by CG.  After the solve U = Mr F_t - g exactly, so the saddle
// residual is [0 ; 0 ; L r_y]: CG stops on ||D^{-1} L r_y|| <= rtol ||D^{-1} b||,
// the MINRES test of the same system.
//
// Replicas with more than 12 colloids (no dense M_SS inverse) keep the
// stresslets as unknowns beside y: with F_t = -b_bot + L y the system in (y, F_S)
//     [ I + L^T M_tt L   L^T M_tS ] [ y  ]   [ L^T (b_tt + M_tt b_bot) ]
//     [ M_St L           M_SS     ] [F_S ] = [ b_S + M_St b_bot        ]
// is SPD too (J + P^T M P with P = diag(L, I)); each iteration costs one plain M
// apply, the stresslet part is preconditioned by the inverse self block, and the
// saddle residual is [0 ; r_S ; L r_y].  This covers colloid suspensions of any
// size, with or without lubrication.
//
// Pair vectors hold 12 entries per canonical pair q (monomer pairs use the
// first 6); pair-space sums run over the bead reduction table, each pair
// attributed to its lower bead, and stresslet sums per colloid bead.

constexpr int PS_THREADS = 64;

// per-replica done flag at done + r * stride (CG or MINRES scalars); null: none done
__device__ __forceinline__ bool rep_done(const char *done, int stride, int r)
{
    return done && *(const int *)(done + (long)r * stride);
}

// velocity DOFs of the pair in pair-DOF order: U_lo, U_hi, W_lo, W_hi
__device__ __forceinline__ void pair_dofs(const Seg &s, long lo, long hi, bool mono, int dof[12], int &nd)
{
    int il = (int)(lo - s.bead_off), ih = (int)(hi - s.bead_off);
    int tl, wl, th, wh;
    vel_dofs(s, il, tl, wl);
    vel_dofs(s, ih, th, wh);
    nd = mono ? 6 : 12;
    for (int k = 0; k < 3; k++) {
        dof[k] = tl + k; dof[3 + k] = th + k;
        if (!mono) { dof[6 + k] = wl + k; dof[9 + k] = wh + k; }
    }
}

// two-body FT far-field mobility of the pair in pair-DOF order, symmetrised
__device__ void pair_mobility(const Seg &s, const double *__restrict__ x, const double *__restrict__ chain, long lo,
                              long hi, bool mono, double *M)
{
    const int nd = mono ? 6 : 12;
    for (int k = 0; k < nd * nd; k++) M[k] = 0.0;
    double dx = x[3 * lo] - x[3 * hi], dy = x[3 * lo + 1] - x[3 * hi + 1], dz = x[3 * lo + 2] - x[3 * hi + 2];
    double r2 = dx * dx + dy * dy + dz * dz, rinv = 1.0 / sqrt(r2), r = r2 * rinv;
    double e[3] = {dx * rinv, dy * rinv, dz * rinv};
    if (mono) {
        r = ref_pair_dist(dx, dy, dz);   // the reference's distance decides the near/far branch
        rinv = 1.0 / r;
        for (int k = 0; k < 6; k++) M[k * 6 + k] = s.beta_inv;
        bool coupled = s.mm_HI && !(s.chain_HI && chain[lo] == chain[hi]);
        if (coupled) {
            double xs, ys;
            if (s.aa_mode == PS_AA_RPY) aa_scalars_rpy<double>(r, rinv, 2.0 * s.beta, xs, ys);
            else aa_scalars<double>(r, rinv, 2.0 * s.beta, xs, ys);
            for (int a = 0; a < 3; a++)
                for (int c = 0; c < 3; c++) {
                    double v = (xs - ys) * e[a] * e[c] + (a == c ? ys : 0.0);
                    M[a * 6 + 3 + c] = v;
                    M[(3 + a) * 6 + c] = v;
                }
        }
        return;
    }
    for (int k = 0; k < 3; k++) {
        M[k * 12 + k] = 1.0; M[(3 + k) * 12 + 3 + k] = 1.0;
        M[(6 + k) * 12 + 6 + k] = 0.75; M[(9 + k) * 12 + 9 + k] = 0.75;
    }
    // the partner's (F, T) column -> this bead's (U, W) rows, e = (x_lo - x_hi)/r as in the BB kernel
    for (int side = 0; side < 2; side++) {
        const bool is_lo = side == 0;
        const int rowU = is_lo ? 0 : 3, rowW = is_lo ? 6 : 9, colF = is_lo ? 3 : 0, colT = is_lo ? 9 : 6;
        for (int c = 0; c < 6; c++) {
            double in[11], out[11];
            for (int k = 0; k < 11; k++) { in[k] = 0.0; out[k] = 0.0; }
            in[c] = 1.0;
            bb_apply<double>(e, r, rinv, is_lo, in, out);
            int col = c < 3 ? colF + c : colT + (c - 3);
            for (int a = 0; a < 3; a++) { M[(rowU + a) * 12 + col] = out[a]; M[(rowW + a) * 12 + col] = out[3 + a]; }
        }
    }
    for (int a = 0; a < 12; a++)
        for (int c = a + 1; c < 12; c++) {
            double v = 0.5 * (M[a * 12 + c] + M[c * 12 + a]);
            M[a * 12 + c] = v; M[c * 12 + a] = v;
        }
}

// per pair: S = K^{1/2} and P = (I + S M_pp S)^{-1} (identity if not positive
// definite); monomer pairs in closed form as compact 6 x 6 blocks (row stride 6),
// colloid pairs by Jacobi + Cholesky as 12 x 12 blocks; each pair owns a
// 144-double slot in S and in P
__global__ void __launch_bounds__(PS_THREADS)
k_ps_setup(long npair, const int2 *__restrict__ pairs, const int *__restrict__ bead_offs, int R,
           const Seg *__restrict__ segs, const double *__restrict__ x, const double *__restrict__ chain,
           const double *__restrict__ tab, int nrow, double *__restrict__ Sout, double *__restrict__ Pout)
{
    long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= npair) return;
    const long lo = pairs[q].x, hi = pairs[q].y;
    const Seg &s = segs[rep_of_b(bead_offs, R, lo)];
    const bool mono = (lo - s.bead_off) < s.Nm;
    double *So = Sout + 144 * q, *Po = Pout + 144 * q;
    if (mono) {
        // closed form: S and the mobility share the modes of the pair block
        double d[3], lam[4], sq[4], pm[4];
        mono_pair_modes(s, x, tab, nrow, lo, hi, d, lam);
        double xs = 0.0, ys = 0.0;
        if (s.mm_HI && !(s.chain_HI && chain[lo] == chain[hi])) {
            double dx = x[3 * lo] - x[3 * hi], dy = x[3 * lo + 1] - x[3 * hi + 1], dz = x[3 * lo + 2] - x[3 * hi + 2];
            const double r = ref_pair_dist(dx, dy, dz), rinv = 1.0 / r;
            if (s.aa_mode == PS_AA_RPY) aa_scalars_rpy<double>(r, rinv, 2.0 * s.beta, xs, ys);
            else aa_scalars<double>(r, rinv, 2.0 * s.beta, xs, ys);
        }
        const double mob[4] = {s.beta_inv + xs, s.beta_inv + ys, s.beta_inv - xs, s.beta_inv - ys};
        for (int k = 0; k < 4; k++) {
            double l = lam[k] > 0 ? lam[k] : 0.0;
            sq[k] = sqrt(l);
            double t = 1.0 + l * mob[k];
            pm[k] = t > 0 ? 1.0 / t : 1.0;
        }
        // compact 6 x 6 blocks (row stride 6) at the start of the pair's slot
        mono_pair_matrix(d, sq, So, 6);
        mono_pair_matrix(d, pm, Po, 6);
        return;
    }
    const int nd = 12;
    double K[144], Q[144], S[144], M[144];
    lub_pair_block(s, x, tab, nrow, lo, hi, mono, K);
    jacobi_eig(K, nd, Q);
    for (int a = 0; a < nd; a++)
        for (int c = 0; c < nd; c++) {
            double v = 0.0;
            for (int k = 0; k < nd; k++) {
                double lam = K[k * nd + k];
                v += Q[a * nd + k] * (lam > 0 ? sqrt(lam) : 0.0) * Q[c * nd + k];
            }
            S[a * nd + c] = v;
        }
    pair_mobility(s, x, chain, lo, hi, mono, M);
    // T = I + S M S  (K <- M S, Q <- T)
    for (int a = 0; a < nd; a++)
        for (int c = 0; c < nd; c++) {
            double v = 0.0;
            for (int k = 0; k < nd; k++) v += M[a * nd + k] * S[k * nd + c];
            K[a * nd + c] = v;
        }
    for (int a = 0; a < nd; a++)
        for (int c = 0; c < nd; c++) {
            double v = (a == c) ? 1.0 : 0.0;
            for (int k = 0; k < nd; k++) v += S[a * nd + k] * K[k * nd + c];
            Q[a * nd + c] = v;
        }
    // Cholesky T = C C^T in place (lower), then P = T^{-1} column by column
    bool ok = true;
    for (int j = 0; j < nd && ok; j++) {
        double d = Q[j * nd + j];
        for (int k = 0; k < j; k++) d -= Q[j * nd + k] * Q[j * nd + k];
        if (!(d > 0)) { ok = false; break; }
        d = sqrt(d);
        Q[j * nd + j] = d;
        for (int i = j + 1; i < nd; i++) {
            double v = Q[i * nd + j];
            for (int k = 0; k < j; k++) v -= Q[i * nd + k] * Q[j * nd + k];
            Q[i * nd + j] = v / d;
        }
    }
    for (int k = 0; k < 144; k++) { So[k] = 0.0; Po[k] = 0.0; }
    for (int a = 0; a < nd; a++)
        for (int c = 0; c < nd; c++) So[a * 12 + c] = S[a * nd + c];
    if (!ok) { for (int a = 0; a < nd; a++) Po[a * 12 + a] = 1.0; return; }
    for (int c = 0; c < nd; c++) {
        double v[12];
        for (int i = 0; i < nd; i++) {
            double t = (i == c) ? 1.0 : 0.0;
            for (int k = 0; k < i; k++) t -= Q[i * nd + k] * v[k];
            v[i] = t / Q[i * nd + i];
        }
        for (int i = nd - 1; i >= 0; i--) {
            double t = v[i];
            for (int k = i + 1; k < nd; k++) t -= Q[k * nd + i] * v[k];
            v[i] = t / Q[i * nd + i];
        }
        for (int i = 0; i < nd; i++) Po[i * 12 + c] = v[i];
    }
}

// v = L y (+ add): per bead, the rows of S_q y_q that belong to it, summed over
// its near pairs in ascending partner order; optionally written into the first
// nm3nc6 entries of a mobility-layout vector and reduced into ||D^{-1} L y||^2
// per bead (constraint-row entries of D)
__global__ void k_ps_L(long ntot, const int *__restrict__ bead_offs, int R, const Seg *__restrict__ segs,
                       const int *__restrict__ sptr, const int *__restrict__ snbr, const int *__restrict__ cidx,
                       const double *__restrict__ S, const double *__restrict__ y,
                       const double *__restrict__ add, double *__restrict__ vel, double *__restrict__ top,
                       const double *__restrict__ D, double *__restrict__ bead_part, const char *__restrict__ done,
                       int dstride)
{
    long b = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= ntot) return;
    const int r = rep_of_b(bead_offs, R, b);
    if (rep_done(done, dstride, r)) return;
    const Seg &s = segs[r];
    const int i = (int)(b - s.bead_off);
    const bool mono = i < s.Nm;
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (int t = sptr[b]; t < sptr[b + 1]; t++) {
        const int qa = cidx[t];
        if (qa < 0) continue;                           // not in the canonical list (lists disagree)
        const bool low = b < (long)snbr[t];
        const double *Sq = S + 144L * qa, *yq = y + 12L * qa;
        const int ng = mono ? 1 : 2, nd = mono ? 6 : 12;    // monomer pairs: 6 x 6 block, zero elsewhere
        for (int g = 0; g < ng; g++)
            for (int k = 0; k < 3; k++) {
                const int row = 6 * g + (low ? 0 : 3) + k;
                double v = 0.0;
                for (int c = 0; c < nd; c++) v += Sq[row * nd + c] * yq[c];
                acc[3 * g + k] += v;
            }
    }
    int tb, wb;
    vel_dofs(s, i, tb, wb);
    double nrm = 0.0;
    for (int g = 0; g < (mono ? 1 : 2); g++)
        for (int k = 0; k < 3; k++) {
            const int d = (g == 0 ? tb : wb) + k;
            double v = acc[3 * g + k] + (add ? add[s.vel_off + d] : 0.0);
            if (vel) vel[s.vel_off + d] = v;
            if (top) top[s.top_off + d] = v;
            if (D) { double t = acc[3 * g + k] / D[s.vec_off + s.nm3nc11 + d]; nrm += t * t; }
        }
    if (bead_part) bead_part[b] = nrm;
}

// w_q = sign * S_q z_q (+ p_q), z gathered from the velocity rows of the Mr apply
// (y + y2 for replicas with a dense stresslet block) plus an optional velocity
// vector; part[q] = p_q . w_q
__global__ void k_ps_LT(long npair, const int2 *__restrict__ pairs, const int *__restrict__ bead_offs, int R,
                        const Seg *__restrict__ segs, const double *__restrict__ S, const double *__restrict__ y,
                        const double *__restrict__ y2, const double *__restrict__ addv, double sign,
                        const double *__restrict__ p, double *__restrict__ w, double *__restrict__ part,
                        const char *__restrict__ done, int dstride)
{
    long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= npair) return;
    const long lo = pairs[q].x, hi = pairs[q].y;
    const int r = rep_of_b(bead_offs, R, lo);
    if (rep_done(done, dstride, r)) return;
    const Seg &s = segs[r];
    const bool mono = (lo - s.bead_off) < s.Nm;
    int dof[12], nd;
    pair_dofs(s, lo, hi, mono, dof, nd);
    double z[12];
    for (int k = 0; k < 12; k++) z[k] = 0.0;
    for (int k = 0; k < nd; k++)
        z[k] = y[s.top_off + dof[k]] + (s.ss_off >= 0 ? y2[s.top_off + dof[k]] : 0.0) +
               (addv ? addv[s.vel_off + dof[k]] : 0.0);
    const double *Sq = S + 144L * q;
    double dot = 0.0;
    // monomer pairs hold a 6 x 6 block (zero elsewhere): rows and columns past nd add nothing
    for (int a = 0; a < 12; a++) {
        double v = 0.0;
        if (a < nd)
            for (int c = 0; c < nd; c++) v += Sq[a * nd + c] * z[c];
        v *= sign;
        if (p) { v += p[12 * q + a]; dot += p[12 * q + a] * v; }
        w[12 * q + a] = v;
    }
    if (part) part[q] = dot;
}

// first iterate: y = 0, r = rhs (in rv), z = P r, p = z, part = r . z
__global__ void k_ps_init(long npair, const int2 *__restrict__ pairs, const int *__restrict__ bead_offs, int R,
                          const Seg *__restrict__ segs, const double *__restrict__ P, double *__restrict__ yv,
                          const double *__restrict__ rv, double *__restrict__ zv, double *__restrict__ pv,
                          double *__restrict__ part)
{
    long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= npair) return;
    const long lo = pairs[q].x;
    const Seg &s = segs[rep_of_b(bead_offs, R, lo)];
    const int nd = (lo - s.bead_off) < s.Nm ? 6 : 12;     // monomer pairs: 6 x 6 block, zero elsewhere
    const double *Pq = P + 144L * q;
    double dot = 0.0;
    for (int a = 0; a < 12; a++) {
        double v = 0.0;
        if (a < nd)
            for (int c = 0; c < nd; c++) v += Pq[a * nd + c] * rv[12 * q + c];
        zv[12 * q + a] = v;
        pv[12 * q + a] = v;
        yv[12 * q + a] = 0.0;
        dot += rv[12 * q + a] * v;
    }
    part[q] = dot;
}

// y += alpha p ; r -= alpha Ap ; z = P r ; part = r . z
__global__ void k_ps_update(long npair, const int2 *__restrict__ pairs, const int *__restrict__ bead_offs, int R,
                            const Seg *__restrict__ segs, const PcgScal *__restrict__ pc, const double *__restrict__ P,
                            const double *__restrict__ pv, const double *__restrict__ Ap, double *__restrict__ yv,
                            double *__restrict__ rv, double *__restrict__ zv, double *__restrict__ part)
{
    long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= npair) return;
    const long lo = pairs[q].x;
    const int r = rep_of_b(bead_offs, R, lo);
    const PcgScal sc = pc[r];
    if (sc.done) return;
    // monomer pairs: 6 x 6 blocks, and entries 6..11 of every pair vector stay zero
    const int nd = (lo - segs[r].bead_off) < segs[r].Nm ? 6 : 12;
    double rq[12];
    for (int a = 0; a < nd; a++) {
        yv[12 * q + a] += sc.alpha * pv[12 * q + a];
        rq[a] = rv[12 * q + a] - sc.alpha * Ap[12 * q + a];
        rv[12 * q + a] = rq[a];
    }
    const double *Pq = P + 144L * q;
    double dot = 0.0;
    for (int a = 0; a < nd; a++) {
        double v = 0.0;
        for (int c = 0; c < nd; c++) v += Pq[a * nd + c] * rq[c];
        zv[12 * q + a] = v;
        dot += rq[a] * v;
    }
    part[q] = dot;
}

// p = z + beta p
__global__ void k_ps_dir(long npair, const int2 *__restrict__ pairs, const int *__restrict__ bead_offs, int R,
                         const PcgScal *__restrict__ pc, const double *__restrict__ zv, double *__restrict__ pv)
{
    long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= npair) return;
    const PcgScal sc = pc[rep_of_b(bead_offs, R, pairs[q].x)];
    if (sc.done) return;
    for (int a = 0; a < 12; a++) pv[12 * q + a] = zv[12 * q + a] + sc.beta * pv[12 * q + a];
}

// per-replica sums over the bead table: pair partials by lower bead plus the
// per-bead stresslet partials (add0), and the per-bead residual partials
// (bead_part + add1).
// mode 0: alpha = rz / sum(part);  mode 1: first check (rz, err);  mode 2: iteration check
__global__ void k_ps_reduce(RedTable T, const int *__restrict__ cptr, const double *__restrict__ part,
                            const double *__restrict__ bead_part, const double *__restrict__ add0,
                            const double *__restrict__ add1, PcgScal *pc, int mode, int maxit, int *nactive)
{
    __shared__ double sh[RB_THREADS / 32][2];
    const RBlk B = T.d_blk[blockIdx.x];
    if (pc[B.rep].done) return;
    double v[2] = {0.0, 0.0};
    for (int e = threadIdx.x; e < B.len; e += RB_THREADS) {
        long b = B.start + e;
        for (int q = cptr[b]; q < cptr[b + 1]; q++) v[0] += part[q];
        if (add0) v[0] += add0[b];
        if (bead_part) v[1] += bead_part[b];
        if (add1) v[1] += add1[b];
    }
    block_sum<2>(v, sh);
    double tot[2];
    if (finish_block<2>(T, B, blockIdx.x, v, tot)) {
        PcgScal p = pc[B.rep];
        if (mode == 0) {
            if (tot[0] <= 0.0) { p.done = 1; p.reason = -8; atomicSub(nactive, 1); }
            else p.alpha = p.rz / tot[0];
        } else {
            p.err = sqrt(tot[1]);
            if (mode == 2) p.it++;
            if (p.err <= p.tol) { p.done = 1; p.reason = 2; }
            else if (tot[0] <= 0.0) { p.done = 1; p.reason = -8; }
            else if (p.it >= maxit) { p.done = 1; p.reason = -3; }
            else {
                p.beta = mode == 1 ? 0.0 : tot[0] / p.rz;
                p.rz = tot[0];
            }
            if (p.done) atomicSub(nactive, 1);
        }
        pc[B.rep] = p;
    }
}

// c = -b_bot (velocity layout), u_t = b_bot
__global__ void k_ps_c(RedTable T, const Seg *__restrict__ segs, const double *__restrict__ b, double *__restrict__ c,
                       double *__restrict__ u)
{
    const RBlk B = T.d_blk[blockIdx.x];
    const Seg &s = segs[B.rep];
    for (int e = threadIdx.x; e < B.len; e += RB_THREADS) {
        long k = B.start + e;
        int j = (int)(k - s.vel_off);
        double v = b[s.vec_off + s.nm3nc11 + j];
        c[k] = -v;
        u[s.top_off + j] = v;
    }
}

// U = (y + y2)_t - g into the saddle solution
__global__ void k_ps_fin(RedTable T, const Seg *__restrict__ segs, const double *__restrict__ y,
                         const double *__restrict__ y2, const double *__restrict__ g, double *__restrict__ x)
{
    const RBlk B = T.d_blk[blockIdx.x];
    const Seg &s = segs[B.rep];
    for (int e = threadIdx.x; e < B.len; e += RB_THREADS) {
        long k = B.start + e;
        int j = (int)(k - s.vel_off);
        double v = y[s.top_off + j] + (s.ss_off >= 0 ? y2[s.top_off + j] : 0.0) - g[k];
        x[s.vec_off + s.nm3nc11 + j] = v;
    }
}

// copy F_t (velocity layout) into the force rows of the saddle solution
__global__ void k_ps_ft(RedTable T, const Seg *__restrict__ segs, const double *__restrict__ ft, double *__restrict__ x)
{
    const RBlk B = T.d_blk[blockIdx.x];
    const Seg &s = segs[B.rep];
    for (int e = threadIdx.x; e < B.len; e += RB_THREADS) {
        long k = B.start + e;
        x[s.vec_off + (k - s.vel_off)] = ft[k];
    }
}

// stresslet unknowns of the joint replicas (Nc > 0 without a dense M_SS
// inverse), one thread per bead; vectors in mobility layout (S part), with
// the inverse self block (1.8 I, 0.9 coupling of components 0 and 4) as the
// preconditioner.  mode 0 init (r = b_S + y_S), 1 Ap = y_S, 2 update, 3 direction,
// 4 finish (F_S into u and the solution).  Per-bead partials: a0 (r.z or p.Ap),
// a1 (||D^{-1} r_S||^2); zero for every other bead.
__global__ void k_ps_S(long ntot, const int *__restrict__ bead_offs, int R, const Seg *__restrict__ segs, int mode,
                       const PcgScal *__restrict__ pc, const double *__restrict__ b, const double *__restrict__ y,
                       const double *__restrict__ D, double *__restrict__ yS, double *__restrict__ rS,
                       double *__restrict__ zS, double *__restrict__ pS, double *__restrict__ ApS,
                       double *__restrict__ u, double *__restrict__ x, double *__restrict__ a0, double *__restrict__ a1)
{
    long bd = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (bd >= ntot) return;
    const int r = rep_of_b(bead_offs, R, bd);
    const Seg &s = segs[r];
    const int i = (int)(bd - s.bead_off);
    const bool joint = s.Nc > 0 && s.ss_off < 0 && i >= s.Nm;
    if (mode != 4 && pc[r].done) return;
    if (!joint) {
        if (mode <= 2) { if (a0) a0[bd] = 0.0; if (a1) a1[bd] = 0.0; }
        return;
    }
    const int c = i - s.Nm;
    const long t0 = (long)s.top_off + s.nm3nc6 + 5 * c;       // S entries in mobility layout
    const long v0 = (long)s.vec_off + s.nm3nc6 + 5 * c;       // S rows of the saddle vector
    const double det = 1.8 * 1.8 - 0.9 * 0.9;
    double dot = 0.0, nrm = 0.0;
    if (mode == 0 || mode == 2) {
        double rv[5], zv[5];
        for (int k = 0; k < 5; k++) {
            if (mode == 0) { rv[k] = b[v0 + k] + y[t0 + k]; yS[t0 + k] = 0.0; }
            else {
                const double al = pc[r].alpha;
                yS[t0 + k] += al * pS[t0 + k];
                rv[k] = rS[t0 + k] - al * ApS[t0 + k];
            }
            rS[t0 + k] = rv[k];
        }
        zv[0] = (1.8 * rv[0] - 0.9 * rv[4]) / det;
        zv[4] = (1.8 * rv[4] - 0.9 * rv[0]) / det;
        for (int k = 1; k < 4; k++) zv[k] = rv[k] / 1.8;
        for (int k = 0; k < 5; k++) {
            zS[t0 + k] = zv[k];
            dot += rv[k] * zv[k];
            double t = rv[k] / D[v0 + k];
            nrm += t * t;
            if (mode == 0) { pS[t0 + k] = zv[k]; u[t0 + k] = zv[k]; }
        }
        a0[bd] = dot;
        a1[bd] = nrm;
    } else if (mode == 1) {
        for (int k = 0; k < 5; k++) { double ap = y[t0 + k]; ApS[t0 + k] = ap; dot += pS[t0 + k] * ap; }
        a0[bd] = dot;
    } else if (mode == 3) {
        const double be = pc[r].beta;
        for (int k = 0; k < 5; k++) { double p = zS[t0 + k] + be * pS[t0 + k]; pS[t0 + k] = p; u[t0 + k] = p; }
    } else {
        for (int k = 0; k < 5; k++) { u[t0 + k] = yS[t0 + k]; x[v0 + k] = yS[t0 + k]; }
    }
}

// Mr applied to the force rows held in E.d_pu (stresslet part zero):
// d_py = M [u ; 0], d_pu2 = [0 ; -M_SS^{-1} (d_py)_S], d_py2 = M d_pu2
static void mr_apply(Engine &E, bool fp32, const void *dn, int ds, cudaStream_t st)
{
    apply_operator(E, 1, E.d_pu, E.d_py, nullptr, fp32, st, dn, ds);
    if (E.n_ss_reps) {
        ::ps_launch_count++, k_ss_apply<<<E.n_ss_reps, 64, 0, st>>>(E.d_segs, E.d_ss_reps, E.d_ssinv, E.d_py, 1, -1.0,
                                                                 nullptr, 1, 0.0, E.d_pu2, 1, (const char *)dn, ds);
        apply_operator(E, 1, E.d_pu2, E.d_py2, nullptr, fp32, st, dn, ds, true);
    }
}

// ---------------------------------------------------------------------------
// Pair-space MINRES, for replica sets whose far-field mobility may be
// indefinite (colloid pairs near contact: the far-field FTS mobility is not
// positive definite there; the reference's own monomer pair scalars).  The
// operator and preconditioner are those of the CG above; the recurrences are
// Paige & Saunders' preconditioned MINRES as in krylov.cu, with PETSc's test on
// the preconditioned residual estimate (np * prod |s_k| <= rtol * np_0).
// Vectors live in the two storages of the pair space: 12 entries per pair, and
// the stresslet entries of the joint replicas' colloids (mobility layout).
struct PMVec { double *pair; double *s; };
struct PMArgs {
    PMVec R[3], W[3], v, z, x;
    const double *Az;          // operator output, pair storage (S part: y_S of the apply)
    const double *y;           // the apply's output (mobility layout)
    double *u;                 // the apply's input (mobility layout): its S part gets z_S
    const double *P;           // pair preconditioner blocks
    double *part, *part2;      // per-pair partials
    double *sA, *sB;           // per-bead partials
};

__device__ __forceinline__ void s_precond(const double r[5], double z[5])
{
    const double det = 1.8 * 1.8 - 0.9 * 0.9;
    z[0] = (1.8 * r[0] - 0.9 * r[4]) / det;
    z[4] = (1.8 * r[4] - 0.9 * r[0]) / det;
    for (int k = 1; k < 4; k++) z[k] = r[k] / 1.8;
}

// one thread per pair (t < npair) or per bead (t - npair; stresslet entries of
// joint-replica colloids, nothing for other beads).
// mode 0 init, 1 alpha (pending w/x update, v = z/beta, Av), 2 beta (r_{k+1}, z = P r), 3 flush
__global__ void k_pm_elem(long npair, long ntot, const int2 *__restrict__ pairs, const int *__restrict__ bead_offs,
                          int R, const Seg *__restrict__ segs, const MinresScal *__restrict__ mr, int mode, int k,
                          PMArgs A)
{
    long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool is_pair = t < npair;
    if (t >= npair + ntot) return;
    long base, bead;
    int n;
    double *u_s = nullptr;
    const double *y_s = nullptr;
    int nd = 12;          // pair blocks: 6 x 6 (row stride 6) for monomer pairs
    if (is_pair) {
        base = 12 * t;
        n = 12;
        bead = pairs[t].x;
        const Seg &sp = segs[rep_of_b(bead_offs, R, bead)];
        if (bead - sp.bead_off < sp.Nm) nd = 6;
    } else {
        bead = t - npair;
        const Seg &s0 = segs[rep_of_b(bead_offs, R, bead)];
        const int i = (int)(bead - s0.bead_off);
        if (!(s0.Nc > 0 && s0.ss_off < 0 && i >= s0.Nm)) {
            if (mode <= 2) { A.sA[bead] = 0.0; A.sB[bead] = 0.0; }
            return;
        }
        base = (long)s0.top_off + s0.nm3nc6 + 5 * (i - s0.Nm);
        n = 5;
        u_s = A.u + base;
        y_s = A.y + base;
    }
    const int r = rep_of_b(bead_offs, R, bead);
    const MinresScal m = mr[r];
    auto V = [&](const PMVec &p) { return (is_pair ? p.pair : p.s) + base; };
    double dot0 = 0.0, dot1 = 0.0;
    if (mode == 0) {
        double rv[12], zv[12];
        double *rr = V(A.R[1]);
        for (int a = 0; a < n; a++) rv[a] = rr[a];
        if (is_pair) {
            const double *Pq = A.P + 144L * t;
            for (int a = 0; a < 12; a++) {
                double acc = 0.0;
                if (a < nd)
                    for (int c = 0; c < nd; c++) acc += Pq[a * nd + c] * rv[c];
                zv[a] = acc;
            }
        } else {
            s_precond(rv, zv);
        }
        double *zz = V(A.z), *xx = V(A.x), *vv = V(A.v), *w0 = V(A.W[0]), *w1 = V(A.W[1]), *w2 = V(A.W[2]);
        for (int a = 0; a < n; a++) {
            zz[a] = zv[a]; xx[a] = 0.0; vv[a] = 0.0; w0[a] = 0.0; w1[a] = 0.0; w2[a] = 0.0;
            dot0 += rv[a] * zv[a];
            dot1 += zv[a] * zv[a];
            if (u_s) u_s[a] = zv[a];
        }
    } else if (mode == 1 || mode == 3) {
        double *vv = V(A.v);
        if (m.pending) {
            double *wn = V(A.W[(k + 2) % 3]);
            const double *w1 = V(A.W[k % 3]), *w2 = V(A.W[(k + 1) % 3]);
            double *xx = V(A.x);
            for (int a = 0; a < n; a++) {
                double w = (vv[a] - m.up_oldeps * w1[a] - m.up_delta * w2[a]) * m.up_ginv;
                wn[a] = w;
                xx[a] += m.up_phi * w;
            }
        }
        if (mode == 1 && !m.done) {
            const double *zz = V(A.z);
            const double *az = is_pair ? A.Az + base : y_s;
            double *av = V(A.R[(k + 1) % 3]);
            const double *rm1 = V(A.R[(k + 2) % 3]);
            const double c1 = (k >= 2) ? m.beta / m.oldb : 0.0;
            for (int a = 0; a < n; a++) {
                double vq = zz[a] * m.sinv;
                double x = m.sinv * az[a];
                if (k >= 2) x -= c1 * rm1[a];
                vv[a] = vq;
                av[a] = x;
                dot0 += vq * x;
            }
        }
    } else if (mode == 2 && !m.done) {
        double *av = V(A.R[(k + 1) % 3]);
        const double *rk = V(A.R[k % 3]);
        const double c2 = m.alfa / m.beta;
        double rv[12], zv[12];
        for (int a = 0; a < n; a++) { rv[a] = av[a] - c2 * rk[a]; av[a] = rv[a]; }
        if (is_pair) {
            const double *Pq = A.P + 144L * t;
            for (int a = 0; a < 12; a++) {
                double acc = 0.0;
                if (a < nd)
                    for (int c = 0; c < nd; c++) acc += Pq[a * nd + c] * rv[c];
                zv[a] = acc;
            }
        } else {
            s_precond(rv, zv);
        }
        double *zz = V(A.z);
        for (int a = 0; a < n; a++) {
            zz[a] = zv[a];
            dot0 += rv[a] * zv[a];
            if (u_s) u_s[a] = zv[a];
        }
    }
    if (mode <= 2) {
        if (is_pair) { A.part[t] = dot0; A.part2[t] = dot1; }
        else { A.sA[bead] = dot0; A.sB[bead] = dot1; }
    }
}

// per-replica MINRES scalar updates over the bead table (pair partials by lower bead)
__global__ void k_pm_reduce(RedTable T, const int *__restrict__ cptr, const double *__restrict__ part,
                            const double *__restrict__ part2, const double *__restrict__ sA,
                            const double *__restrict__ sB, MinresScal *mr, int mode, int maxit, double rtol,
                            int *nactive)
{
    __shared__ double sh[RB_THREADS / 32][2];
    const RBlk B = T.d_blk[blockIdx.x];
    const MinresScal m0 = mr[B.rep];
    if (mode != 1 && m0.done) return;
    if (mode == 1 && m0.done && !m0.pending) return;
    double v[2] = {0.0, 0.0};
    for (int e = threadIdx.x; e < B.len; e += RB_THREADS) {
        long b = B.start + e;
        for (int q = cptr[b]; q < cptr[b + 1]; q++) { v[0] += part[q]; v[1] += part2[q]; }
        v[0] += sA[b];
        v[1] += sB[b];
    }
    block_sum<2>(v, sh);
    double tot[2];
    if (!finish_block<2>(T, B, blockIdx.x, v, tot)) return;
    MinresScal m = m0;
    if (mode == 0) {
        m = MinresScal{};
        double np0 = sqrt(tot[1]);
        m.np = np0;
        m.ttol = fmax(rtol * np0, 1e-50);
        if (tot[0] < 0) { m.done = 1; m.reason = -8; }
        else if (np0 <= m.ttol || tot[0] == 0.0) { m.done = 1; m.reason = 2; }
        else {
            m.beta = sqrt(tot[0]); m.phibar = m.beta; m.cs = -1; m.sn = 0; m.sinv = 1.0 / m.beta;
        }
        if (m.done) atomicSub(nactive, 1);
    } else if (mode == 1) {
        if (m.pending) m.pending = 0;
        if (!m.done) m.alfa = tot[0];
    } else {
        m.it += 1;
        double bb = tot[0];
        m.oldb = m.beta;
        if (bb < 0) {
            m.done = 1; m.reason = -8;
        } else {
            m.beta = sqrt(bb);
            double oldeps = m.epsln;
            double delta = m.cs * m.dbar + m.sn * m.alfa;
            double gbar = m.sn * m.dbar - m.cs * m.alfa;
            m.epsln = m.sn * m.beta;
            m.dbar = -m.cs * m.beta;
            double gamma = sqrt(gbar * gbar + m.beta * m.beta);
            if (gamma < 2.2250738585072014e-308) gamma = 2.2250738585072014e-308;
            m.cs = gbar / gamma;
            m.sn = m.beta / gamma;
            double phi = m.cs * m.phibar;
            m.phibar = m.sn * m.phibar;
            m.up_oldeps = oldeps; m.up_delta = delta; m.up_ginv = 1.0 / gamma; m.up_phi = phi;
            m.pending = 1;
            m.np = m.np * fabs(m.sn);
            if (m.np <= m.ttol) { m.done = 1; m.reason = 2; }
            else if (m.beta == 0.0) { m.done = 1; m.reason = 3; }
            else if (m.it >= maxit) { m.done = 1; m.reason = -3; }
            m.sinv = m.beta != 0.0 ? 1.0 / m.beta : 0.0;
        }
        if (m.done) atomicSub(nactive, 1);
    }
    mr[B.rep] = m;
}

static int ensure_pair_space(Engine &E)
{
    long need = std::max<long>(E.lub_npairs, 1);
    if (need <= E.pair_cap) return PS_OK;
    E.ps_setup_valid = false;
    cudaFree(E.d_pS); cudaFree(E.d_pP); cudaFree(E.d_ppart); cudaFree(E.d_ppart2);
    for (auto &p : E.d_py_) cudaFree(p);
    for (auto &p : E.d_pmp) cudaFree(p);
    E.pair_cap = need * 3 / 2 + 256;
    PS_CK(cudaMalloc(&E.d_pS, sizeof(double) * 144 * E.pair_cap));
    PS_CK(cudaMalloc(&E.d_pP, sizeof(double) * 144 * E.pair_cap));
    PS_CK(cudaMalloc(&E.d_ppart, sizeof(double) * E.pair_cap));
    PS_CK(cudaMalloc(&E.d_ppart2, sizeof(double) * E.pair_cap));
    for (auto &p : E.d_py_) PS_CK(cudaMalloc(&p, sizeof(double) * 12 * E.pair_cap));
    for (auto &p : E.d_pmp) PS_CK(cudaMalloc(&p, sizeof(double) * 12 * E.pair_cap));
    return PS_OK;
}

// MINRES iterations of the pair-space system; the setup (pair blocks, g, the
// u_t = b_bot apply input) has run.  Returns the solution's pair and stresslet
// storages in *ysol / *ssol.
static int pair_minres(Engine &E, const double *b, const double *g, int maxit, double rtol, bool fp32,
                       cudaStream_t st, double **ysol, double **ssol, int *iters)
{
    RedTable &TB = E.red_bead;
    const long npair = E.lub_npairs;
    const int thr = 128;
    const unsigned nbp = (unsigned)((std::max<long>(npair, 1) + PS_THREADS - 1) / PS_THREADS);
    const unsigned nbb = (unsigned)((E.ntot + thr - 1) / thr);
    const unsigned nbe = (unsigned)((npair + E.ntot + thr - 1) / thr);
    const char *dn = (const char *)&E.d_pmr[0].done;
    const int ds = (int)sizeof(MinresScal);
    PMArgs A;
    for (int k = 0; k < 3; k++) { A.R[k] = {E.d_pmp[k], E.d_pms[k]}; A.W[k] = {E.d_pmp[3 + k], E.d_pms[3 + k]}; }
    A.v = {E.d_pmp[6], E.d_pms[6]};
    A.z = {E.d_pmp[7], E.d_pms[7]};
    A.x = {E.d_pmp[8], E.d_pms[8]};
    A.Az = E.d_pmp[9];
    A.y = E.d_py;
    A.u = E.d_pu;
    A.P = E.d_pP;
    A.part = E.d_ppart; A.part2 = E.d_ppart2;
    A.sA = E.d_sbead[0]; A.sB = E.d_sbead[1];
    PS_CK(cudaMemsetAsync(E.d_pmr, 0, sizeof(MinresScal) * E.R, st));
    // rhs into R[1]: pairs L^T (g + Mr b_bot), stresslets b_S + (M b_bot)_S
    mr_apply(E, fp32, dn, ds, st);
    if (npair)
        ::ps_launch_count++, k_ps_LT<<<nbp, PS_THREADS, 0, st>>>(npair, E.d_lub_pairs, E.d_bead_offs, E.R, E.d_segs,
                                                              E.d_pS, E.d_py, E.d_py2, g, 1.0, nullptr, A.R[1].pair,
                                                              nullptr, dn, ds);
    ::ps_launch_count++, k_ps_S<<<nbb, thr, 0, st>>>(E.ntot, E.d_bead_offs, E.R, E.d_segs, 0, E.d_pcg, b, E.d_py, E.d_D,
                                                  E.d_sv[0], A.R[1].s, E.d_sv[2], E.d_sv[3], E.d_sv[4], E.d_pu,
                                                  nullptr, A.sA, A.sB);
    *E.h_nactive = E.R;
    PS_CK(cudaMemcpyAsync(E.d_nactive, E.h_nactive, sizeof(int), cudaMemcpyHostToDevice, st));
    ::ps_launch_count++, k_pm_elem<<<nbe, thr, 0, st>>>(npair, E.ntot, E.d_lub_pairs, E.d_bead_offs, E.R, E.d_segs,
                                                     E.d_pmr, 0, 0, A);
    ::ps_launch_count++, k_pm_reduce<<<TB.nblk, RB_THREADS, 0, st>>>(TB, E.d_lubc_ptr, A.part, A.part2, A.sA, A.sB,
                                                                  E.d_pmr, 0, maxit, rtol, E.d_nactive);
    PS_CK(cudaMemcpyAsync(E.h_nactive, E.d_nactive, sizeof(int), cudaMemcpyDeviceToHost, st));
    PS_CK(cudaStreamSynchronize(st));
    int nact = *E.h_nactive, k = 0;
    while (nact > 0 && k < maxit) {
        for (int j = 0; j < 8 && k < maxit; j++) {
            k++;
            // Az = A z: u = [L z_y ; z_S] (z_S already in u), apply, z_y + L^T (...)_t
            ::ps_launch_count++, k_ps_L<<<nbb, thr, 0, st>>>(E.ntot, E.d_bead_offs, E.R, E.d_segs, E.d_lub_ptr,
                                                          E.d_lub_nbr, E.d_lub_cidx, E.d_pS, A.z.pair,
                                                          nullptr, nullptr, E.d_pu, nullptr, nullptr, dn, ds);
            mr_apply(E, fp32, dn, ds, st);
            if (npair)
                ::ps_launch_count++, k_ps_LT<<<nbp, PS_THREADS, 0, st>>>(npair, E.d_lub_pairs, E.d_bead_offs, E.R,
                                                                      E.d_segs, E.d_pS, E.d_py, E.d_py2, nullptr, 1.0,
                                                                      A.z.pair, E.d_pmp[9], nullptr, dn, ds);
            ::ps_launch_count++, k_pm_elem<<<nbe, thr, 0, st>>>(npair, E.ntot, E.d_lub_pairs, E.d_bead_offs, E.R,
                                                             E.d_segs, E.d_pmr, 1, k, A);
            ::ps_launch_count++, k_pm_reduce<<<TB.nblk, RB_THREADS, 0, st>>>(TB, E.d_lubc_ptr, A.part, A.part2, A.sA,
                                                                          A.sB, E.d_pmr, 1, maxit, rtol, E.d_nactive);
            ::ps_launch_count++, k_pm_elem<<<nbe, thr, 0, st>>>(npair, E.ntot, E.d_lub_pairs, E.d_bead_offs, E.R,
                                                             E.d_segs, E.d_pmr, 2, k, A);
            ::ps_launch_count++, k_pm_reduce<<<TB.nblk, RB_THREADS, 0, st>>>(TB, E.d_lubc_ptr, A.part, A.part2, A.sA,
                                                                          A.sB, E.d_pmr, 2, maxit, rtol, E.d_nactive);
        }
        PS_CK(cudaMemcpyAsync(E.h_nactive, E.d_nactive, sizeof(int), cudaMemcpyDeviceToHost, st));
        PS_CK(cudaStreamSynchronize(st));
        nact = *E.h_nactive;
    }
    // the last pending w/x update
    ::ps_launch_count++, k_pm_elem<<<nbe, thr, 0, st>>>(npair, E.ntot, E.d_lub_pairs, E.d_bead_offs, E.R, E.d_segs,
                                                     E.d_pmr, 3, k + 1, A);
    PS_CK(cudaGetLastError());
    *ysol = A.x.pair;
    *ssol = A.x.s;
    *iters = k;
    return PS_OK;
}

static int pair_solve(Engine &E, const double *b, double *x, const ps_ksp_opts *o, ps_ksp_result *res,
                      cudaStream_t st, bool minres)
{
    RedTable &TV = E.red_vel, &TB = E.red_bead;
    const bool fp32 = E.precision == PS_PREC_MIXED;
    // CG converges in tens of iterations on positive definite far fields; a cap
    // hands the rare indefinite case to MINRES early
    const int maxit = minres ? (o->maxit > 0 ? o->maxit : 10000) : std::min(o->maxit > 0 ? o->maxit : 10000, 1000);
    const int check_every = o->check_every > 0 ? o->check_every : 8;
    const long npair = E.lub_npairs;
    const int thr = 128;
    const unsigned nbp = (unsigned)((std::max<long>(npair, 1) + PS_THREADS - 1) / PS_THREADS);
    const unsigned nbb = (unsigned)((E.ntot + thr - 1) / thr);
    int rc = diag_saddle(E, E.d_D, st);
    if (rc) return rc;
    if ((rc = ensure_pair_space(E))) return rc;
    double *yv = E.d_py_[0], *rv = E.d_py_[1], *zv = E.d_py_[2], *pv = E.d_py_[3], *Ap = E.d_py_[4];
    double *yS = E.d_sv[0], *rS = E.d_sv[1], *zS = E.d_sv[2], *pS = E.d_sv[3], *ApS = E.d_sv[4];
    double *sA = E.d_sbead[0], *sB = E.d_sbead[1];     // per-bead stresslet partials
    // d_pr (nvel >= ntot doubles) holds the per-bead partials
    double *cvel = E.d_pV, *g = E.d_pg, *tmp = E.d_tmp_vel, *bead_part = E.d_pr;
    const void *dn = &E.d_pcg[0].done;
    const int ds = (int)sizeof(PcgScal);
    // stresslet unknowns join the CG only for replicas beyond the dense stresslet
    // limit; without such replicas k_ps_S has nothing to do but keep the per-bead
    // stresslet partials at zero, which one clear at the start does
    const bool joint = E.n_ss_polish > 0;
    if (!joint) {
        PS_CK(cudaMemsetAsync(sA, 0, sizeof(double) * E.ntot, st));
        PS_CK(cudaMemsetAsync(sB, 0, sizeof(double) * E.ntot, st));
    }
    PS_CK(cudaMemsetAsync(x, 0, sizeof(double) * E.nvec, st));
    PS_CK(cudaMemsetAsync(E.d_pu, 0, sizeof(double) * E.ntop, st));
    PS_CK(cudaMemsetAsync(E.d_pu2, 0, sizeof(double) * E.ntop, st));
    PS_CK(cudaMemsetAsync(E.d_py2, 0, sizeof(double) * E.ntop, st));
    ::ps_launch_count++, k_pcg_start<<<E.red.nblk, RB_THREADS, 0, st>>>(E.red, E.d_segs, b, E.d_D, E.d_pcg, o->rtol);
    // the pair blocks depend on the staged positions and the table only: solves
    // that share a staging (the deterministic and the noise solve) set them up once
    if (npair && !E.ps_setup_valid) {
        ::ps_launch_count++, k_ps_setup<<<nbp, PS_THREADS, 0, st>>>(npair, E.d_lub_pairs, E.d_bead_offs, E.R, E.d_segs,
                                                                 E.d_x, E.d_chain, E.d_lubtab, E.lub_nrow, E.d_pS,
                                                                 E.d_pP);
        E.ps_setup_valid = true;
    }
    if (E.n_ss_reps) {
        ::ps_launch_count++, k_ss_inverse<<<E.n_ss_reps, 64, 0, st>>>(E.d_segs, E.d_ss_reps, E.d_x, E.d_delta, E.d_ssinv);
        // g: u2 = [0 ; M_SS^{-1} b_S]
        ::ps_launch_count++, k_ss_apply<<<E.n_ss_reps, 64, 0, st>>>(E.d_segs, E.d_ss_reps, E.d_ssinv, b, 0, 1.0, nullptr,
                                                                 0, 0.0, E.d_pu2, 1, nullptr, 0);
        apply_operator(E, 1, E.d_pu2, E.d_py2, nullptr, fp32, st, nullptr, 0, true);
    }
    ::ps_launch_count++, k_pcg_g<<<TV.nblk, RB_THREADS, 0, st>>>(TV, E.d_segs, b, E.d_py2, g);
    ::ps_launch_count++, k_ps_c<<<TV.nblk, RB_THREADS, 0, st>>>(TV, E.d_segs, b, cvel, E.d_pu);
    PS_CK(cudaGetLastError());
    std::vector<PcgScal> hp(E.R);
    PS_CK(cudaMemcpyAsync(hp.data(), E.d_pcg, sizeof(PcgScal) * E.R, cudaMemcpyDeviceToHost, st));
    PS_CK(cudaStreamSynchronize(st));
    int nact = 0;
    for (auto &p : hp) nact += !p.done;
    *E.h_nactive = nact;
    PS_CK(cudaMemcpyAsync(E.d_nactive, E.h_nactive, sizeof(int), cudaMemcpyHostToDevice, st));
    if (minres) {
        int nit = 0;
        rc = pair_minres(E, b, g, maxit, o->rtol, fp32, st, &yv, &yS, &nit);
        if (rc) return rc;
    } else {
        if (nact) {
            // rhs = L^T (g + Mr b_bot) (joint replicas: Mr -> M, and b_S + (M b_bot)_S) ; r = rhs ; z = P r ; p = z
            mr_apply(E, fp32, dn, ds, st);
            if (npair) {
                ::ps_launch_count++, k_ps_LT<<<nbp, PS_THREADS, 0, st>>>(npair, E.d_lub_pairs, E.d_bead_offs, E.R, E.d_segs,
                                                                      E.d_pS, E.d_py, E.d_py2, g, 1.0, nullptr, rv, nullptr,
                                                                      (const char *)dn, ds);
                ::ps_launch_count++, k_ps_init<<<nbp, PS_THREADS, 0, st>>>(npair, E.d_lub_pairs, E.d_bead_offs, E.R,
                                                                        E.d_segs, E.d_pP, yv, rv, zv, pv, E.d_ppart);
            }
        }
        if (joint)
            ::ps_launch_count++, k_ps_S<<<nbb, thr, 0, st>>>(E.ntot, E.d_bead_offs, E.R, E.d_segs, 0, E.d_pcg, b, E.d_py, E.d_D,
                                                      yS, rS, zS, pS, ApS, E.d_pu, x, sA, sB);
        // initial residual ||D^{-1} L r||^2 + ||D^{-1} r_S||^2
        ::ps_launch_count++, k_ps_L<<<nbb, thr, 0, st>>>(E.ntot, E.d_bead_offs, E.R, E.d_segs, E.d_lub_ptr, E.d_lub_nbr,
                                                      E.d_lub_cidx, E.d_pS, rv, nullptr, nullptr, nullptr,
                                                      E.d_D, bead_part, (const char *)dn, ds);
        ::ps_launch_count++, k_ps_reduce<<<TB.nblk, RB_THREADS, 0, st>>>(TB, E.d_lubc_ptr, E.d_ppart, bead_part, sA, sB,
                                                                      E.d_pcg, 1, maxit, E.d_nactive);
        PS_CK(cudaMemcpyAsync(E.h_nactive, E.d_nactive, sizeof(int), cudaMemcpyDeviceToHost, st));
        PS_CK(cudaStreamSynchronize(st));
        nact = *E.h_nactive;
        int k = 0;
        while (nact > 0 && k < maxit) {
            for (int j = 0; j < check_every && k < maxit; j++, k++) {
                // Ap = p + L^T Mr L p  (joint replicas: [p_y + L^T (M u)_t ; (M u)_S], u = [L p_y ; p_S])
                ::ps_launch_count++, k_ps_L<<<nbb, thr, 0, st>>>(E.ntot, E.d_bead_offs, E.R, E.d_segs, E.d_lub_ptr,
                                                              E.d_lub_nbr, E.d_lub_cidx, E.d_pS, pv, nullptr,
                                                              nullptr, E.d_pu, nullptr, nullptr, (const char *)dn, ds);
                mr_apply(E, fp32, dn, ds, st);
                if (npair)
                    ::ps_launch_count++, k_ps_LT<<<nbp, PS_THREADS, 0, st>>>(npair, E.d_lub_pairs, E.d_bead_offs, E.R,
                                                                          E.d_segs, E.d_pS, E.d_py, E.d_py2, nullptr, 1.0,
                                                                          pv, Ap, E.d_ppart, (const char *)dn, ds);
                if (joint)
                    ::ps_launch_count++, k_ps_S<<<nbb, thr, 0, st>>>(E.ntot, E.d_bead_offs, E.R, E.d_segs, 1, E.d_pcg, b, E.d_py,
                                                              E.d_D, yS, rS, zS, pS, ApS, E.d_pu, x, sA, nullptr);
                ::ps_launch_count++, k_ps_reduce<<<TB.nblk, RB_THREADS, 0, st>>>(TB, E.d_lubc_ptr, E.d_ppart, nullptr, sA,
                                                                              nullptr, E.d_pcg, 0, maxit, E.d_nactive);
                if (npair)
                    ::ps_launch_count++, k_ps_update<<<nbp, PS_THREADS, 0, st>>>(npair, E.d_lub_pairs, E.d_bead_offs, E.R,
                                                                              E.d_segs, E.d_pcg, E.d_pP, pv, Ap, yv, rv,
                                                                              zv, E.d_ppart);
                if (joint)
                    ::ps_launch_count++, k_ps_S<<<nbb, thr, 0, st>>>(E.ntot, E.d_bead_offs, E.R, E.d_segs, 2, E.d_pcg, b, E.d_py,
                                                              E.d_D, yS, rS, zS, pS, ApS, E.d_pu, x, sA, sB);
                ::ps_launch_count++, k_ps_L<<<nbb, thr, 0, st>>>(E.ntot, E.d_bead_offs, E.R, E.d_segs, E.d_lub_ptr,
                                                              E.d_lub_nbr, E.d_lub_cidx, E.d_pS, rv, nullptr,
                                                              nullptr, nullptr, E.d_D, bead_part, (const char *)dn, ds);
                ::ps_launch_count++, k_ps_reduce<<<TB.nblk, RB_THREADS, 0, st>>>(TB, E.d_lubc_ptr, E.d_ppart, bead_part, sA,
                                                                              sB, E.d_pcg, 2, maxit, E.d_nactive);
                if (npair)
                    ::ps_launch_count++, k_ps_dir<<<nbp, PS_THREADS, 0, st>>>(npair, E.d_lub_pairs, E.d_bead_offs, E.R,
                                                                           E.d_pcg, zv, pv);
                if (joint)
                    ::ps_launch_count++, k_ps_S<<<nbb, thr, 0, st>>>(E.ntot, E.d_bead_offs, E.R, E.d_segs, 3, E.d_pcg, b, E.d_py,
                                                              E.d_D, yS, rS, zS, pS, ApS, E.d_pu, x, nullptr, nullptr);
            }
            PS_CK(cudaMemcpyAsync(E.h_nactive, E.d_nactive, sizeof(int), cudaMemcpyDeviceToHost, st));
            PS_CK(cudaStreamSynchronize(st));
            nact = *E.h_nactive;
        }
    }
    // F_t = -b_bot + L y (into u_t and the force rows), then U = Mr F_t - g, F_S
    ::ps_launch_count++, k_ps_L<<<nbb, thr, 0, st>>>(E.ntot, E.d_bead_offs, E.R, E.d_segs, E.d_lub_ptr, E.d_lub_nbr,
                                                  E.d_lub_cidx, E.d_pS, yv, cvel, tmp, E.d_pu, nullptr,
                                                  nullptr, nullptr, 0);
    ::ps_launch_count++, k_ps_ft<<<TV.nblk, RB_THREADS, 0, st>>>(TV, E.d_segs, tmp, x);
    if (joint)
        ::ps_launch_count++, k_ps_S<<<nbb, thr, 0, st>>>(E.ntot, E.d_bead_offs, E.R, E.d_segs, 4, E.d_pcg, b, E.d_py, E.d_D,
                                                  yS, rS, zS, pS, ApS, E.d_pu, x, nullptr, nullptr);
    mr_apply(E, fp32, nullptr, 0, st);
    ::ps_launch_count++, k_ps_fin<<<TV.nblk, RB_THREADS, 0, st>>>(TV, E.d_segs, E.d_py, E.d_py2, g, x);
    if (E.n_ss_reps)
        ::ps_launch_count++, k_ss_apply<<<E.n_ss_reps, 64, 0, st>>>(E.d_segs, E.d_ss_reps, E.d_ssinv, b, 0, 1.0, E.d_py,
                                                                 1, -1.0, x, 0, nullptr, 0);
    PS_CK(cudaGetLastError());
    int worst = 1000, itmax = 0;
    long itsum = 0;
    double emax = 0;
    if (minres) {
        std::vector<MinresScal> hm(E.R);
        PS_CK(cudaMemcpyAsync(hm.data(), E.d_pmr, sizeof(MinresScal) * E.R, cudaMemcpyDeviceToHost, st));
        PS_CK(cudaStreamSynchronize(st));
        for (auto &m : hm) {
            int reason = m.done ? m.reason : -3;
            worst = std::min(worst, reason);
            itmax = std::max(itmax, m.it);
            itsum += m.it;
            emax = std::max(emax, m.np);
        }
    } else {
        PS_CK(cudaMemcpyAsync(hp.data(), E.d_pcg, sizeof(PcgScal) * E.R, cudaMemcpyDeviceToHost, st));
        PS_CK(cudaStreamSynchronize(st));
        for (auto &p : hp) {
            int reason = p.done ? p.reason : -3;
            worst = std::min(worst, reason);
            itmax = std::max(itmax, p.it);
            itsum += p.it;
            emax = std::max(emax, p.err);
        }
    }
    if (worst == 1000) worst = 2;
    if (res) { res->reason = worst; res->iters_max = itmax; res->iters_sum = itsum; res->rnorm_max = emax; }
    return PS_OK;
}

int structured_solve(Engine &E, const double *b, double *x, const ps_ksp_opts *o, ps_ksp_result *res,
                     cudaStream_t st)
{
    if (E.any_lub || E.n_ss_polish) {
        ps_ksp_result r0 = {2, 0, 0, 0.0};
        int rc = pair_solve(E, b, x, o, &r0, st, E.any_indef);
        if (rc) return rc;
        if (r0.reason < 0 && !E.any_indef) {      // CG met an indefinite far field: MINRES on the same system
            ps_ksp_result r2 = {2, 0, 0, 0.0};
            if ((rc = pair_solve(E, b, x, o, &r2, st, true))) return rc;
            r2.iters_max += r0.iters_max;
            r2.iters_sum += r0.iters_sum;
            r0 = r2;
        }
        // replicas whose CG broke down (an indefinite far-field mobility: the
        // reference's own pair scalars) finish with MINRES from the CG iterate
        if (r0.reason < 0) {
            ps_ksp_opts po = *o;
            po.warm = 1;
            po.method = PS_SOLVE_MINRES;
            ps_ksp_result r1;
            rc = minres_solve(E, b, x, &po, &r1, st);
            if (rc == PS_ERR_CUDA) return rc;
            r0.reason = r1.reason;
            r0.iters_max = std::max(r0.iters_max, r1.iters_max);
            r0.iters_sum += r1.iters_sum;
            r0.rnorm_max = std::max(r0.rnorm_max, r1.rnorm_max);
        }
        if (res) *res = r0;
        return r0.reason;
    }
    const int thr = 256;
    unsigned nb = (unsigned)((E.nvec + thr - 1) / thr);
    double *y = E.d_Rr[0];
    bool fp32 = E.precision == PS_PREC_MIXED;
    ::ps_launch_count++, k_struct_init<<<nb, thr, 0, st>>>(E.nvec, E.d_vec_offs, E.R, E.d_segs, b, x);
    if (E.n_ss_reps) {
        apply_operator(E, 0, x, y, nullptr, fp32, st);   // y_top = M [F_t ; 0]
        ::ps_launch_count++, k_struct_ss<<<E.n_ss_reps, 256, 0, st>>>(E.d_segs, E.d_ss_reps, E.d_x, E.d_delta, b, y, x);
    }
    apply_operator(E, 0, x, y, nullptr, fp32, st);       // y_top = M F
    ::ps_launch_count++, k_struct_u<<<nb, thr, 0, st>>>(E.nvec, E.d_vec_offs, E.R, E.d_segs, b, y, x);
    PS_CK(cudaGetLastError());
    ps_ksp_result r0 = {2, 0, 0, 0.0};
    if (E.n_ss_polish) {
        ps_ksp_opts po = *o;
        po.warm = 1;
        po.method = PS_SOLVE_MINRES;
        int rc = minres_solve(E, b, x, &po, &r0, st);
        if (rc == PS_ERR_CUDA) return rc;
    }
    if (res) *res = r0;
    return r0.reason;
}

}  // namespace ps
