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
#include <curand_kernel.h>
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
    pdl_enter();
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
    pdl_enter();
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
    pdl_enter();
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
    pdl_enter();
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
    pdl_enter();
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
    pdl_enter();
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
    pdl_enter();
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

// shared-memory scratch of one warp for one colloid pair
struct PsWarpSmem {
    double K[144], Q[144], S[144], M[144];
};

// One colloid pair (lo, hi) by one warp: S = K^{1/2} of the R_lub pair block in
// closed form (colloid_pair_sqrt_coeffs), M = two-body FT far-field mobility
// (symmetrised), P = (I + S M S)^{-1} by Cholesky, identity if not positive
// definite.  Every matrix-product entry sums over k in ascending order.
__device__ void ps_setup_colloid_pair(const Seg &s, long lo, long hi, const double *__restrict__ x,
                                      const double *__restrict__ tab, int nrow, double *__restrict__ So,
                                      double *__restrict__ Po, PsWarpSmem &w, int lane)
{
    double *K = w.K, *Q = w.Q, *S = w.S, *M = w.M;
    for (int t = lane; t < 144; t += 32) { S[t] = 0.0; M[t] = 0.0; }
    __syncwarp();
    {
        double d[3], f[10], kc[10], g[10];
        lub_pair_geom(s, x, tab, nrow, lo, hi, 1.0, d, f);
        lub_pair_coeffs(f, 1.0, kc);
        colloid_pair_sqrt_coeffs(kc, g);
        if (lane < 9) pair_block_entries(d, g, false, lane / 3, lane % 3, S);
    }
    if (lane < 12) {
        // the partner's (F, T) column -> this bead's (U, W) rows, e = (x_lo - x_hi)/r as in the BB kernel
        const double dx = x[3 * lo] - x[3 * hi], dy = x[3 * lo + 1] - x[3 * hi + 1], dz = x[3 * lo + 2] - x[3 * hi + 2];
        const double r2 = dx * dx + dy * dy + dz * dz, rinv = 1.0 / sqrt(r2), r = r2 * rinv;
        const double e[3] = {dx * rinv, dy * rinv, dz * rinv};
        M[lane * 12 + lane] = lane < 6 ? 1.0 : 0.75;
        const bool is_lo = lane < 6;
        const int c = lane % 6;
        const int rowU = is_lo ? 0 : 3, rowW = is_lo ? 6 : 9, colF = is_lo ? 3 : 0, colT = is_lo ? 9 : 6;
        double in[11], out[11];
        for (int k = 0; k < 11; k++) { in[k] = 0.0; out[k] = 0.0; }
        in[c] = 1.0;
        bb_apply<double>(e, r, rinv, is_lo, in, out);
        const int col = c < 3 ? colF + c : colT + (c - 3);
        for (int a = 0; a < 3; a++) { M[(rowU + a) * 12 + col] = out[a]; M[(rowW + a) * 12 + col] = out[3 + a]; }
    }
    __syncwarp();
    for (int t = lane; t < 144; t += 32) {
        const int a = t / 12, c = t % 12;
        if (c > a) {
            const double v = 0.5 * (M[a * 12 + c] + M[c * 12 + a]);
            M[a * 12 + c] = v; M[c * 12 + a] = v;
        }
    }
    __syncwarp();
    for (int t = lane; t < 144; t += 32) {          // K <- M S
        const int a = t / 12, c = t % 12;
        double v = 0.0;
        for (int k = 0; k < 12; k++) v += M[a * 12 + k] * S[k * 12 + c];
        K[t] = v;
    }
    __syncwarp();
    for (int t = lane; t < 144; t += 32) {          // Q <- I + S M S
        const int a = t / 12, c = t % 12;
        double v = (a == c) ? 1.0 : 0.0;
        for (int k = 0; k < 12; k++) v += S[a * 12 + k] * K[k * 12 + c];
        Q[t] = v;
    }
    __syncwarp();
    bool ok = true;
    for (int j = 0; j < 12; j++) {                  // Cholesky Q = C C^T in place (lower)
        double dj = Q[j * 12 + j];
        for (int k = 0; k < j; k++) dj -= Q[j * 12 + k] * Q[j * 12 + k];
        if (!(dj > 0)) { ok = false; break; }
        dj = sqrt(dj);
        const int i = j + 1 + lane;
        double v = 0.0;
        if (i < 12) {
            v = Q[i * 12 + j];
            for (int k = 0; k < j; k++) v -= Q[i * 12 + k] * Q[j * 12 + k];
        }
        __syncwarp();
        if (lane == 0) Q[j * 12 + j] = dj;
        if (i < 12) Q[i * 12 + j] = v / dj;
        __syncwarp();
    }
    for (int t = lane; t < 144; t += 32) So[t] = S[t];
    if (!ok) {
        for (int t = lane; t < 144; t += 32) Po[t] = (t / 12 == t % 12) ? 1.0 : 0.0;
        __syncwarp();
        return;
    }
    if (lane < 12) {                                // P = Q^{-1}, column `lane`
        const int c = lane;
        double v[12];
        for (int i = 0; i < 12; i++) {
            double t = (i == c) ? 1.0 : 0.0;
            for (int k = 0; k < i; k++) t -= Q[i * 12 + k] * v[k];
            v[i] = t / Q[i * 12 + i];
        }
        for (int i = 11; i >= 0; i--) {
            double t = v[i];
            for (int k = i + 1; k < 12; k++) t -= Q[k * 12 + i] * v[k];
            v[i] = t / Q[i * 12 + i];
        }
        for (int i = 0; i < 12; i++) Po[i * 12 + c] = v[i];
    }
    __syncwarp();
}

// per pair: S = K^{1/2} and P = (I + S M_pp S)^{-1} (identity if not positive
// definite); each pair owns a 144-double slot in S and in P.  Monomer pairs: one
// thread each, closed form, compact 6 x 6 blocks (row stride 6).  Colloid pairs:
// one warp per colloid in the blocks past the pair blocks, taking the canonical
// pairs for which it is the lower bead (ps_setup_colloid_pair), 12 x 12 blocks.
__global__ void __launch_bounds__(PS_THREADS)
k_ps_setup(long npair, const int2 *__restrict__ pairs, const int *__restrict__ bead_offs, int R,
           const Seg *__restrict__ segs, const double *__restrict__ x, const double *__restrict__ chain,
           const double *__restrict__ tab, int nrow, long ncoll, const int *__restrict__ coll_rep,
           const int *__restrict__ cptr, double *__restrict__ Sout, double *__restrict__ Pout)
{
    pdl_enter();
    __shared__ PsWarpSmem wsm[PS_THREADS / 32];
    const long nbp = (npair + blockDim.x - 1) / blockDim.x;
    if (blockIdx.x >= nbp) {
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        const long c = (long)(blockIdx.x - nbp) * (blockDim.x >> 5) + wid;
        if (c >= ncoll) return;
        const Seg &s = segs[coll_rep[c]];
        const long b = s.bead_off + s.Nm + (c - s.coll_off);
        for (int q = cptr[b]; q < cptr[b + 1]; q++)
            ps_setup_colloid_pair(s, b, pairs[q].y, x, tab, nrow, Sout + 144L * q, Pout + 144L * q, wsm[wid], lane);
        return;
    }
    const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= npair) return;
    const long lo = pairs[q].x, hi = pairs[q].y;
    const Seg &s = segs[rep_of_b(bead_offs, R, lo)];
    if ((lo - s.bead_off) >= s.Nm) return;            // colloid pair: its lower colloid's warp
    double *So = Sout + 144 * q, *Po = Pout + 144 * q;
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
}

static void launch_ps_setup(Engine &E, cudaStream_t st)
{
    const long npair = E.lub_npairs;
    const long nbp = (npair + PS_THREADS - 1) / PS_THREADS, nbc = (E.ncoll + PS_THREADS / 32 - 1) / (PS_THREADS / 32);
    ps_launch(k_ps_setup, (unsigned)(nbp + nbc), PS_THREADS, 0, st,
            npair, E.d_lub_pairs, E.d_bead_offs, E.R, E.d_segs, E.d_x, E.d_chain, E.d_lubtab, E.lub_nrow, E.ncoll,
            E.d_coll_rep, E.d_lubc_ptr, E.d_pS, E.d_pP);
}

// v = L y (+ add): per bead, the rows of S_q y_q that belong to it, summed over
// its near pairs; optionally written into the first nm3nc6 entries of a
// mobility-layout vector and reduced into ||D^{-1} L y||^2 per bead
// (constraint-row entries of D).  Monomer beads take one thread each and sum
// their pairs in ascending partner order.  Colloid beads, which gather the
// long lists (every near monomer and colloid), take one warp each from the
// blocks past the bead blocks: lane l sums the pairs l, l + 32, ... of the
// colloid's list and a fixed butterfly joins the lanes, so the order is fixed.
__device__ __forceinline__ void ps_L_pair(const double *__restrict__ Sq, const double *__restrict__ yq, bool low,
                                          int ng, int nd, double acc[6])
{
    double yv[12];
#pragma unroll
    for (int c = 0; c < 12; c++) yv[c] = c < nd ? yq[c] : 0.0;
    for (int g = 0; g < ng; g++)
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const double *row = Sq + (6 * g + (low ? 0 : 3) + k) * nd;
            double v = 0.0;
#pragma unroll
            for (int c = 0; c < 12; c++)
                if (c < nd) v += row[c] * yv[c];
            acc[3 * g + k] += v;
        }
}

__device__ __forceinline__ void ps_L_out(const Seg &s, int i, long b, const double acc[6], const double *__restrict__ add,
                                         double *__restrict__ vel, double *__restrict__ top,
                                         const double *__restrict__ D, double *__restrict__ bead_part)
{
    const bool mono = i < s.Nm;
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

__global__ void k_ps_L(long ntot, long ncoll, const int *__restrict__ coll_rep, const int *__restrict__ bead_offs,
                       int R, const Seg *__restrict__ segs, const int *__restrict__ sptr, const int *__restrict__ snbr,
                       const int *__restrict__ cidx, const double *__restrict__ S, const double *__restrict__ y,
                       const double *__restrict__ add, double *__restrict__ vel, double *__restrict__ top,
                       const double *__restrict__ D, double *__restrict__ bead_part, const char *__restrict__ done,
                       int dstride)
{
    pdl_enter();
    const long nbb = (ntot + blockDim.x - 1) / blockDim.x;
    double acc[6] = {0, 0, 0, 0, 0, 0};
    if (blockIdx.x >= nbb) {
        const long c = (long)(blockIdx.x - nbb) * (blockDim.x >> 5) + (threadIdx.x >> 5);
        if (c >= ncoll) return;
        const int lane = threadIdx.x & 31, r = coll_rep[c];
        if (rep_done(done, dstride, r)) return;
        const Seg &s = segs[r];
        const int i = s.Nm + (int)(c - s.coll_off);
        const long b = s.bead_off + i;
        for (int t = sptr[b] + lane; t < sptr[b + 1]; t += 32) {
            const int qa = cidx[t];
            if (qa < 0) continue;                       // not in the canonical list (lists disagree)
            ps_L_pair(S + 144L * qa, y + 12L * qa, b < (long)snbr[t], 2, 12, acc);
        }
#pragma unroll
        for (int q = 0; q < 6; q++)
            for (int o = 16; o > 0; o >>= 1) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], o);
        if (lane == 0) ps_L_out(s, i, b, acc, add, vel, top, D, bead_part);
        return;
    }
    const long b = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= ntot) return;
    const int r = rep_of_b(bead_offs, R, b);
    if (rep_done(done, dstride, r)) return;
    const Seg &s = segs[r];
    const int i = (int)(b - s.bead_off);
    if (i >= s.Nm) return;                              // colloid: one warp in the blocks past nbb
    for (int t = sptr[b]; t < sptr[b + 1]; t++) {
        const int qa = cidx[t];
        if (qa < 0) continue;
        ps_L_pair(S + 144L * qa, y + 12L * qa, b < (long)snbr[t], 1, 6, acc);   // monomer pairs: 6 x 6 blocks
    }
    ps_L_out(s, i, b, acc, add, vel, top, D, bead_part);
}

static void launch_ps_L(Engine &E, const double *y, const double *add, double *vel, double *top, const double *D,
                        double *bead_part, const char *done, int dstride, cudaStream_t st)
{
    const int thr = 128;
    const long nbb = (E.ntot + thr - 1) / thr, nbc = (E.ncoll + thr / 32 - 1) / (thr / 32);
    ps_launch(k_ps_L, (unsigned)(nbb + nbc), thr, 0, st,
            E.ntot, E.ncoll, E.d_coll_rep, E.d_bead_offs, E.R, E.d_segs, E.d_lub_ptr, E.d_lub_nbr, E.d_lub_cidx, E.d_pS,
            y, add, vel, top, D, bead_part, done, dstride);
}

// w_q = sign * S_q z_q (+ p_q), z gathered from the velocity rows of the Mr apply
// (y + y2 for replicas with a dense stresslet block) plus an optional velocity
// vector; part[q] = p_q . w_q.  Sixteen lanes per pair: lane a gathers z_a and
// forms row a (rows and columns past nd, 6 for monomer pairs, add nothing), and
// a fixed butterfly over the sixteen lanes forms the dot.
constexpr int LT_LANES = 16;

// z_a = (P_q r)_a for lane a of a pair's team (r_c held by lane c); rows and
// columns past nd (6 for monomer pairs) add nothing, columns in ascending order
__device__ __forceinline__ double pm_matvec(const double *__restrict__ Pq, int a, int nd, double ra, unsigned team)
{
    double z = 0.0;
#pragma unroll
    for (int c = 0; c < 12; c++) {
        const double rc = __shfl_sync(team, ra, c, LT_LANES);
        if (a < nd && c < nd) z += Pq[a * nd + c] * rc;
    }
    return z;
}

__global__ void k_ps_LT(long npair, const int2 *__restrict__ pairs, const int *__restrict__ bead_offs, int R,
                        const Seg *__restrict__ segs, const double *__restrict__ S, const double *__restrict__ y,
                        const double *__restrict__ y2, const double *__restrict__ addv, double sign,
                        const double *__restrict__ p, double *__restrict__ w, double *__restrict__ part,
                        const char *__restrict__ done, int dstride)
{
    pdl_enter();
    const long q = ((long)blockIdx.x * blockDim.x + threadIdx.x) / LT_LANES;
    const int a = threadIdx.x % LT_LANES;
    const unsigned team = 0xffffu << (threadIdx.x & 16);
    if (q >= npair) return;                       // whole teams leave together
    const long lo = pairs[q].x, hi = pairs[q].y;
    const int r = rep_of_b(bead_offs, R, lo);
    if (rep_done(done, dstride, r)) return;
    const Seg &s = segs[r];
    const bool mono = (lo - s.bead_off) < s.Nm;
    const int nd = mono ? 6 : 12;
    double za = 0.0;
    if (a < nd) {
        const long bd = (a % 6) < 3 ? lo : hi;
        int tb, wb;
        vel_dofs(s, (int)(bd - s.bead_off), tb, wb);
        const int d = (a < 6 ? tb : wb) + a % 3;
        za = y[s.top_off + d] + (s.ss_off >= 0 ? y2[s.top_off + d] : 0.0) + (addv ? addv[s.vel_off + d] : 0.0);
    }
    const double *Sq = S + 144L * q + a * nd;
    double v = 0.0;
#pragma unroll
    for (int c = 0; c < 12; c++) {
        const double zc = __shfl_sync(team, za, c, LT_LANES);
        if (a < nd && c < nd) v += Sq[c] * zc;
    }
    v *= sign;
    double dot = 0.0;
    if (a < 12) {
        if (p) { v += p[12 * q + a]; dot = p[12 * q + a] * v; }
        w[12 * q + a] = v;
    }
    if (part) {
#pragma unroll
        for (int o = LT_LANES / 2; o > 0; o >>= 1) dot += __shfl_xor_sync(team, dot, o, LT_LANES);
        if (a == 0) part[q] = dot;
    }
}

// first iterate: y = 0, r = rhs (in rv), z = P r, p = z, part = r . z;
// a team of LT_LANES lanes per pair, lane a owning entry a
__global__ void k_ps_init(long npair, const int2 *__restrict__ pairs, const int *__restrict__ bead_offs, int R,
                          const Seg *__restrict__ segs, const double *__restrict__ P, double *__restrict__ yv,
                          const double *__restrict__ rv, double *__restrict__ zv, double *__restrict__ pv,
                          double *__restrict__ part)
{
    pdl_enter();
    const long q = ((long)blockIdx.x * blockDim.x + threadIdx.x) / LT_LANES;
    const int a = threadIdx.x % LT_LANES;
    const unsigned team = 0xffffu << (threadIdx.x & 16);
    if (q >= npair) return;
    const long lo = pairs[q].x;
    const Seg &s = segs[rep_of_b(bead_offs, R, lo)];
    const int nd = (lo - s.bead_off) < s.Nm ? 6 : 12;     // monomer pairs: 6 x 6 block, zero elsewhere
    const long e = 12 * q + a;
    const double ra = a < 12 ? rv[e] : 0.0;
    const double v = pm_matvec(P + 144L * q, a, nd, ra, team);
    double dot = 0.0;
    if (a < 12) {
        zv[e] = v;
        pv[e] = v;
        yv[e] = 0.0;
        dot = ra * v;
    }
#pragma unroll
    for (int o = LT_LANES / 2; o > 0; o >>= 1) dot += __shfl_xor_sync(team, dot, o, LT_LANES);
    if (a == 0) part[q] = dot;
}

// y += alpha p ; r -= alpha Ap ; z = P r ; part = r . z; a team per pair as k_ps_init
__global__ void k_ps_update(long npair, const int2 *__restrict__ pairs, const int *__restrict__ bead_offs, int R,
                            const Seg *__restrict__ segs, const PcgScal *__restrict__ pc, const double *__restrict__ P,
                            const double *__restrict__ pv, const double *__restrict__ Ap, double *__restrict__ yv,
                            double *__restrict__ rv, double *__restrict__ zv, double *__restrict__ part)
{
    pdl_enter();
    const long q = ((long)blockIdx.x * blockDim.x + threadIdx.x) / LT_LANES;
    const int a = threadIdx.x % LT_LANES;
    const unsigned team = 0xffffu << (threadIdx.x & 16);
    if (q >= npair) return;
    const long lo = pairs[q].x;
    const int r = rep_of_b(bead_offs, R, lo);
    const PcgScal sc = pc[r];
    if (sc.done) return;
    // monomer pairs: 6 x 6 blocks, and entries 6..11 of every pair vector stay zero
    const int nd = (lo - segs[r].bead_off) < segs[r].Nm ? 6 : 12;
    const long e = 12 * q + a;
    double ra = 0.0;
    if (a < nd) {
        yv[e] += sc.alpha * pv[e];
        ra = rv[e] - sc.alpha * Ap[e];
        rv[e] = ra;
    }
    const double v = pm_matvec(P + 144L * q, a, nd, ra, team);
    double dot = 0.0;
    if (a < nd) {
        zv[e] = v;
        dot = ra * v;
    }
#pragma unroll
    for (int o = LT_LANES / 2; o > 0; o >>= 1) dot += __shfl_xor_sync(team, dot, o, LT_LANES);
    if (a == 0) part[q] = dot;
}

// p = z + beta p, one thread per pair-vector entry
__global__ void k_ps_dir(long npair, const int2 *__restrict__ pairs, const int *__restrict__ bead_offs, int R,
                         const PcgScal *__restrict__ pc, const double *__restrict__ zv, double *__restrict__ pv)
{
    pdl_enter();
    const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= 12 * npair) return;
    const PcgScal &sc = pc[rep_of_b(bead_offs, R, pairs[e / 12].x)];
    if (sc.done) return;
    pv[e] = zv[e] + sc.beta * pv[e];
}

// per-replica sums over the bead table: pair partials by lower bead plus the
// per-bead stresslet partials (add0), and the per-bead residual partials
// (bead_part + add1).
// mode 0: alpha = rz / sum(part);  mode 1: first check (rz, err);  mode 2: iteration check
__global__ void k_ps_reduce(RedTable T, const int *__restrict__ cptr, const double *__restrict__ part,
                            const double *__restrict__ bead_part, const double *__restrict__ add0,
                            const double *__restrict__ add1, PcgScal *pc, int mode, int maxit, int *nactive)
{
    pdl_enter();
    __shared__ double sh[RB_THREADS / 32][2];
    const RBlk B = T.d_blk[blockIdx.x];
    if (pc[B.rep].done) return;
    double v[2] = {0.0, 0.0};
    // pairs are stored by lower bead, so the block's beads own one contiguous pair range
    for (long q = cptr[B.start] + threadIdx.x; q < cptr[B.start + B.len]; q += RB_THREADS) v[0] += part[q];
    for (int e = threadIdx.x; e < B.len; e += RB_THREADS) {
        long b = B.start + e;
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
    pdl_enter();
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
    pdl_enter();
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
    pdl_enter();
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
    pdl_enter();
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
        ps_launch(k_ss_apply, E.n_ss_reps, 64, 0, st, E.d_segs, E.d_ss_reps, E.d_ssinv, E.d_py, 1, -1.0,
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
    const double *y;           // the apply's output (mobility layout; its S part is y_S)
    const double *y2;          // the dense stresslet block's share of the output (replicas with one)
    const double *S;           // pair square-root blocks (L = [B_q S_q])
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

// MINRES element work of pair t by a team of LT_LANES lanes, lane a owning entry a
// of the pair vectors (a < 12); the partial dots join over the team by a fixed
// butterfly.  mode as k_pm_elem.
__device__ __forceinline__ int pm_pair_team(long t, int a, unsigned team, const int2 *__restrict__ pairs,
                                             const int *__restrict__ bead_offs, int R, const Seg *__restrict__ segs,
                                             const MinresScal *__restrict__ mr, int mode, int k, const PMArgs &A)
{
    const long bead = pairs[t].x;
    const int r = rep_of_b(bead_offs, R, bead);
    const Seg &sp = segs[r];
    const int nd = (bead - sp.bead_off) < sp.Nm ? 6 : 12;   // monomer pairs: 6 x 6 blocks
    const MinresScal m = mr[r];
    const long e = 12 * t + a;
    const bool act = a < 12;
    double dot0 = 0.0, dot1 = 0.0;
    if (mode == 0) {
        const double rv = act ? A.R[1].pair[e] : 0.0;
        const double zv = pm_matvec(A.P + 144L * t, a, nd, rv, team);
        if (act) {
            A.z.pair[e] = zv; A.x.pair[e] = 0.0; A.v.pair[e] = 0.0;
            A.W[0].pair[e] = 0.0; A.W[1].pair[e] = 0.0; A.W[2].pair[e] = 0.0;
            dot0 = rv * zv;
            dot1 = zv * zv;
        }
    } else if (mode == 1 || mode == 3) {
        double *vv = A.v.pair;
        if (act && m.pending) {
            const double w = (vv[e] - m.up_oldeps * A.W[k % 3].pair[e] - m.up_delta * A.W[(k + 1) % 3].pair[e]) *
                             m.up_ginv;
            A.W[(k + 2) % 3].pair[e] = w;
            A.x.pair[e] += m.up_phi * w;
        }
        if (mode == 1 && !m.done) {
            // the pair rows of A z: z_q + S_q (y + y2) gathered at the pair's DOFs (the L^T of
            // the apply; lane a gathers entry a and forms row a, columns in ascending order)
            double ya = 0.0;
            if (a < nd) {
                const long bd = (a % 6) < 3 ? bead : (long)pairs[t].y;
                int tb, wb;
                vel_dofs(sp, (int)(bd - sp.bead_off), tb, wb);
                const int d = (a < 6 ? tb : wb) + a % 3;
                ya = A.y[sp.top_off + d] + (sp.ss_off >= 0 ? A.y2[sp.top_off + d] : 0.0);
            }
            const double *Sq = A.S + 144L * t + a * nd;
            double sy = 0.0;
#pragma unroll
            for (int c = 0; c < 12; c++) {
                const double yc = __shfl_sync(team, ya, c, LT_LANES);
                if (a < nd && c < nd) sy += Sq[c] * yc;
            }
            if (act) {
                const double az = sy + A.z.pair[e];
                const double vq = A.z.pair[e] * m.sinv;
                double x = m.sinv * az;
                if (k >= 2) x -= (m.beta / m.oldb) * A.R[(k + 2) % 3].pair[e];
                vv[e] = vq;
                A.R[(k + 1) % 3].pair[e] = x;
                dot0 = vq * x;
            }
        }
    } else if (mode == 2 && !m.done) {
        double rv = 0.0;
        if (act) {
            double *av = A.R[(k + 1) % 3].pair;
            rv = av[e] - (m.alfa / m.beta) * A.R[k % 3].pair[e];
            av[e] = rv;
        }
        const double zv = pm_matvec(A.P + 144L * t, a, nd, rv, team);
        if (act) {
            A.z.pair[e] = zv;
            dot0 = rv * zv;
        }
    }
    if (mode <= 2) {
#pragma unroll
        for (int o = LT_LANES / 2; o > 0; o >>= 1) {
            dot0 += __shfl_xor_sync(team, dot0, o, LT_LANES);
            dot1 += __shfl_xor_sync(team, dot1, o, LT_LANES);
        }
        if (a == 0) { A.part[t] = dot0; A.part2[t] = dot1; }
    }
    return r;
}

// Per-replica MINRES scalar recurrences from the replica's totals t0, t1 (the
// sums of the pair and bead partials of k_pm_elem); mode 0 init, 1 alpha, 2 beta.
__device__ void pm_scalars(MinresScal *mr, int r, int mode, double t0, double t1, int maxit, double rtol,
                           int *nactive)
{
    const MinresScal m0 = mr[r];
    if (mode != 1 && m0.done) return;
    if (mode == 1 && m0.done && !m0.pending) return;
    MinresScal m = m0;
    if (mode == 0) {
        m = MinresScal{};
        double np0 = sqrt(t1);
        m.np = np0;
        m.ttol = fmax(rtol * np0, 1e-50);
        if (t0 < 0) { m.done = 1; m.reason = -8; }
        else if (np0 <= m.ttol || t0 == 0.0) { m.done = 1; m.reason = 2; }
        else {
            m.beta = sqrt(t0); m.phibar = m.beta; m.cs = -1; m.sn = 0; m.sinv = 1.0 / m.beta;
        }
        if (m.done) atomicSub(nactive, 1);
    } else if (mode == 1) {
        if (m.pending) m.pending = 0;
        if (!m.done) m.alfa = t0;
    } else {
        m.it += 1;
        double bb = t0;
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
    mr[r] = m;
}

// Fixed-order sum of x[lo, hi) over the block: thread t takes lo + t, lo + t + B,
// ... into eight independent accumulators (eight loads in flight), joined in order.
__device__ __forceinline__ double block_strided_sum(const double *__restrict__ x, long lo, long hi)
{
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const long B = blockDim.x;
    for (long q = lo + threadIdx.x; q < hi; q += 8 * B) {
#pragma unroll
        for (int u = 0; u < 8; u++)
            if (q + u * B < hi) acc[u] += __ldcg(x + q + u * B);
    }
    return ((acc[0] + acc[1]) + (acc[2] + acc[3])) + ((acc[4] + acc[5]) + (acc[6] + acc[7]));
}

// In-kernel completion of the per-replica sums: every pair team and every bead
// thread counts one item of its replica (warp-aggregated atomics after a
// fence); the block whose count completes replica r sums r's pair partials (a
// contiguous range, pairs being stored by lower bead) and bead partials in a
// fixed order -- block_strided_sum, then a shuffle tree and the warps in
// order, whichever block finishes -- and runs the scalar recurrence.
struct PMRed {
    int *cnt;                  // per replica, zero between launches
    const int *cptr;           // canonical pair pointer by lower bead
    int maxit;
    double rtol;
    int *nactive;
};

__device__ void pm_count_and_finish(int myrep, const Seg *__restrict__ segs, const PMArgs &A, const PMRed &red,
                                    MinresScal *mr, int mode)
{
    __shared__ int s_n, s_list[1024];
    __shared__ double s_sum[32][2];
    if (threadIdx.x == 0) s_n = 0;
    __threadfence();
    __syncthreads();
    const unsigned valid = __ballot_sync(0xffffffffu, myrep >= 0);
    if (myrep >= 0) {
        const unsigned grp = __match_any_sync(valid, myrep);
        if ((int)(threadIdx.x & 31) == __ffs(grp) - 1) {
            const Seg &s = segs[myrep];
            const int total = red.cptr[s.bead_off + s.Np] - red.cptr[s.bead_off] + s.Np;
            const int n = __popc(grp);
            if (atomicAdd(&red.cnt[myrep], n) + n == total) s_list[atomicAdd(&s_n, 1)] = myrep;
        }
    }
    __syncthreads();
    const int nfin = s_n;
    for (int i = 0; i < nfin; i++) {
        const int r = s_list[i];
        __threadfence();
        const Seg &s = segs[r];
        const long q0 = red.cptr[s.bead_off], q1 = red.cptr[s.bead_off + s.Np];
        double v0 = block_strided_sum(A.part, q0, q1) + block_strided_sum(A.sA, s.bead_off, (long)s.bead_off + s.Np);
        double v1 = block_strided_sum(A.part2, q0, q1) + block_strided_sum(A.sB, s.bead_off, (long)s.bead_off + s.Np);
        for (int o = 16; o > 0; o >>= 1) {
            v0 += __shfl_down_sync(0xffffffffu, v0, o);
            v1 += __shfl_down_sync(0xffffffffu, v1, o);
        }
        if ((threadIdx.x & 31) == 0) { s_sum[threadIdx.x >> 5][0] = v0; s_sum[threadIdx.x >> 5][1] = v1; }
        __syncthreads();
        if (threadIdx.x == 0) {
            double t0 = 0.0, t1 = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); w++) { t0 += s_sum[w][0]; t1 += s_sum[w][1]; }
            pm_scalars(mr, r, mode, t0, t1, red.maxit, red.rtol, red.nactive);
            red.cnt[r] = 0;
        }
        __syncthreads();
    }
}

// Teams of LT_LANES lanes per pair (global thread < npair * LT_LANES), then one
// thread per bead (stresslet entries of joint-replica colloids, nothing for
// other beads); modes 0..2 finish their replica sums in the same launch
// (pm_count_and_finish).  No thread leaves early: every thread reaches the
// block barriers of the finish.
// mode 0 init, 1 alpha (pending w/x update, v = z/beta, Av), 2 beta (r_{k+1}, z = P r), 3 flush
__global__ void k_pm_elem(long npair, long ntot, const int2 *__restrict__ pairs, const int *__restrict__ bead_offs,
                          int R, const Seg *__restrict__ segs, MinresScal *mr, int mode, int k, PMArgs A, PMRed red)
{
    pdl_enter();
    const long gt = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long npt = npair * LT_LANES;
    int myrep = -1;                                   // replica of the item this thread counts
    if (gt < npt) {
        const int a = threadIdx.x % LT_LANES;
        const int r = pm_pair_team(gt / LT_LANES, a, 0xffffu << (threadIdx.x & 16), pairs, bead_offs, R, segs, mr,
                                   mode, k, A);
        if (a == 0) myrep = r;
    } else if (gt - npt < ntot) {
        const long bead = gt - npt;
        const int r = rep_of_b(bead_offs, R, bead);
        myrep = r;
        const Seg &s0 = segs[r];
        const int i = (int)(bead - s0.bead_off);
        if (!(s0.Nc > 0 && s0.ss_off < 0 && i >= s0.Nm)) {
            if (mode <= 2) { A.sA[bead] = 0.0; A.sB[bead] = 0.0; }
        } else {
            const long base = (long)s0.top_off + s0.nm3nc6 + 5 * (i - s0.Nm);
            const int n = 5;
            double *u_s = A.u + base;
            const double *y_s = A.y + base;
            const MinresScal m = mr[r];
            auto V = [&](const PMVec &p) { return p.s + base; };
            double dot0 = 0.0, dot1 = 0.0;
            if (mode == 0) {
                double rv[5], zv[5];
                double *rr = V(A.R[1]);
                for (int a = 0; a < n; a++) rv[a] = rr[a];
                s_precond(rv, zv);
                double *zz = V(A.z), *xx = V(A.x), *vv = V(A.v), *w0 = V(A.W[0]), *w1 = V(A.W[1]), *w2 = V(A.W[2]);
                for (int a = 0; a < n; a++) {
                    zz[a] = zv[a]; xx[a] = 0.0; vv[a] = 0.0; w0[a] = 0.0; w1[a] = 0.0; w2[a] = 0.0;
                    dot0 += rv[a] * zv[a];
                    dot1 += zv[a] * zv[a];
                    u_s[a] = zv[a];
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
                    double *av = V(A.R[(k + 1) % 3]);
                    const double *rm1 = V(A.R[(k + 2) % 3]);
                    const double c1 = (k >= 2) ? m.beta / m.oldb : 0.0;
                    for (int a = 0; a < n; a++) {
                        double vq = zz[a] * m.sinv;
                        double x = m.sinv * y_s[a];
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
                double rv[5], zv[5];
                for (int a = 0; a < n; a++) { rv[a] = av[a] - c2 * rk[a]; av[a] = rv[a]; }
                s_precond(rv, zv);
                double *zz = V(A.z);
                for (int a = 0; a < n; a++) {
                    zz[a] = zv[a];
                    dot0 += rv[a] * zv[a];
                    u_s[a] = zv[a];
                }
            }
            if (mode <= 2) { A.sA[bead] = dot0; A.sB[bead] = dot1; }
        }
    }
    if (mode <= 2) pm_count_and_finish(myrep, segs, A, red, mr, mode);
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
    const long npair = E.lub_npairs;
    const int thr = 128;
    const unsigned nbp = (unsigned)((std::max<long>(npair, 1) + PS_THREADS - 1) / PS_THREADS);
    const unsigned nbp_lt = (unsigned)((std::max<long>(npair, 1) * LT_LANES + PS_THREADS - 1) / PS_THREADS);
    const unsigned nbp_e = (unsigned)((std::max<long>(npair, 1) * 12 + PS_THREADS - 1) / PS_THREADS);
    const unsigned nbb = (unsigned)((E.ntot + thr - 1) / thr);
    const unsigned nbe = (unsigned)((npair * LT_LANES + E.ntot + thr - 1) / thr);
    const char *dn = (const char *)&E.d_pmr[0].done;
    const int ds = (int)sizeof(MinresScal);
    PMArgs A;
    for (int k = 0; k < 3; k++) { A.R[k] = {E.d_pmp[k], E.d_pms[k]}; A.W[k] = {E.d_pmp[3 + k], E.d_pms[3 + k]}; }
    A.v = {E.d_pmp[6], E.d_pms[6]};
    A.z = {E.d_pmp[7], E.d_pms[7]};
    A.x = {E.d_pmp[8], E.d_pms[8]};
    A.y = E.d_py;
    A.y2 = E.d_py2;
    A.S = E.d_pS;
    A.u = E.d_pu;
    A.P = E.d_pP;
    A.part = E.d_ppart; A.part2 = E.d_ppart2;
    A.sA = E.d_sbead[0]; A.sB = E.d_sbead[1];
    PS_CK(cudaMemsetAsync(E.d_pmr, 0, sizeof(MinresScal) * E.R, st));
    if (!E.d_pm_cnt) {
        PS_CK(cudaMalloc(&E.d_pm_cnt, sizeof(int) * E.R));
        PS_CK(cudaMemsetAsync(E.d_pm_cnt, 0, sizeof(int) * E.R, st));
    }
    const PMRed red = {E.d_pm_cnt, E.d_lubc_ptr, maxit, rtol, E.d_nactive};
    // rhs into R[1]: pairs L^T (g + Mr b_bot), stresslets b_S + (M b_bot)_S
    mr_apply(E, fp32, dn, ds, st);
    if (npair)
        ps_launch(k_ps_LT, nbp_lt, PS_THREADS, 0, st, npair, E.d_lub_pairs, E.d_bead_offs, E.R, E.d_segs,
                E.d_pS, E.d_py, E.d_py2, g, 1.0, nullptr, A.R[1].pair,
                nullptr, dn, ds);
    ps_launch(k_ps_S, nbb, thr, 0, st, E.ntot, E.d_bead_offs, E.R, E.d_segs, 0, E.d_pcg, b, E.d_py, E.d_D,
            E.d_sv[0], A.R[1].s, E.d_sv[2], E.d_sv[3], E.d_sv[4], E.d_pu,
            nullptr, A.sA, A.sB);
    *E.h_nactive = E.R;
    PS_CK(cudaMemcpyAsync(E.d_nactive, E.h_nactive, sizeof(int), cudaMemcpyHostToDevice, st));
    ps_launch(k_pm_elem, nbe, thr, 0, st, npair, E.ntot, E.d_lub_pairs, E.d_bead_offs, E.R, E.d_segs,
            E.d_pmr, 0, 0, A, red);
    PS_CK(cudaMemcpyAsync(E.h_nactive, E.d_nactive, sizeof(int), cudaMemcpyDeviceToHost, st));
    PS_CK(cudaStreamSynchronize(st));
    int nact = *E.h_nactive, k = 0;
    while (nact > 0 && k < maxit) {
        for (int j = 0; j < 8 && k < maxit; j++) {
            k++;
            // Az = A z: u = [L z_y ; z_S] (z_S already in u), apply; mode 1 forms z_y + L^T (...)_t itself
            launch_ps_L(E, A.z.pair, nullptr, nullptr, E.d_pu, nullptr, nullptr, dn, ds, st);
            mr_apply(E, fp32, dn, ds, st);
            ps_launch(k_pm_elem, nbe, thr, 0, st, npair, E.ntot, E.d_lub_pairs, E.d_bead_offs, E.R,
                    E.d_segs, E.d_pmr, 1, k, A, red);
            ps_launch(k_pm_elem, nbe, thr, 0, st, npair, E.ntot, E.d_lub_pairs, E.d_bead_offs, E.R,
                    E.d_segs, E.d_pmr, 2, k, A, red);
        }
        PS_CK(cudaMemcpyAsync(E.h_nactive, E.d_nactive, sizeof(int), cudaMemcpyDeviceToHost, st));
        PS_CK(cudaStreamSynchronize(st));
        nact = *E.h_nactive;
    }
    // the last pending w/x update
    ps_launch(k_pm_elem, nbe, thr, 0, st, npair, E.ntot, E.d_lub_pairs, E.d_bead_offs, E.R, E.d_segs,
            E.d_pmr, 3, k + 1, A, red);
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
    const unsigned nbp_lt = (unsigned)((std::max<long>(npair, 1) * LT_LANES + PS_THREADS - 1) / PS_THREADS);
    const unsigned nbp_e = (unsigned)((std::max<long>(npair, 1) * 12 + PS_THREADS - 1) / PS_THREADS);
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
    ps_launch(k_pcg_start, E.red.nblk, RB_THREADS, 0, st, E.red, E.d_segs, b, E.d_D, E.d_pcg, o->rtol);
    // the pair blocks depend on the staged positions and the table only: solves
    // that share a staging (the deterministic and the noise solve) set them up once
    if (npair && !E.ps_setup_valid) {
        launch_ps_setup(E, st);
        E.ps_setup_valid = true;
    }
    if (E.n_ss_reps) {
        ps_launch(k_ss_inverse, E.n_ss_reps, 64, 0, st, E.d_segs, E.d_ss_reps, E.d_x, E.d_delta, E.d_ssinv);
        // g: u2 = [0 ; M_SS^{-1} b_S]
        ps_launch(k_ss_apply, E.n_ss_reps, 64, 0, st, E.d_segs, E.d_ss_reps, E.d_ssinv, b, 0, 1.0, nullptr,
                0, 0.0, E.d_pu2, 1, nullptr, 0);
        apply_operator(E, 1, E.d_pu2, E.d_py2, nullptr, fp32, st, nullptr, 0, true);
    }
    ps_launch(k_pcg_g, TV.nblk, RB_THREADS, 0, st, TV, E.d_segs, b, E.d_py2, g);
    ps_launch(k_ps_c, TV.nblk, RB_THREADS, 0, st, TV, E.d_segs, b, cvel, E.d_pu);
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
                ps_launch(k_ps_LT, nbp_lt, PS_THREADS, 0, st, npair, E.d_lub_pairs, E.d_bead_offs, E.R, E.d_segs,
                        E.d_pS, E.d_py, E.d_py2, g, 1.0, nullptr, rv, nullptr,
                        (const char *)dn, ds);
                ps_launch(k_ps_init, nbp_lt, PS_THREADS, 0, st, npair, E.d_lub_pairs, E.d_bead_offs, E.R,
                        E.d_segs, E.d_pP, yv, rv, zv, pv, E.d_ppart);
            }
        }
        if (joint)
            ps_launch(k_ps_S, nbb, thr, 0, st, E.ntot, E.d_bead_offs, E.R, E.d_segs, 0, E.d_pcg, b, E.d_py, E.d_D,
                    yS, rS, zS, pS, ApS, E.d_pu, x, sA, sB);
        // initial residual ||D^{-1} L r||^2 + ||D^{-1} r_S||^2
        launch_ps_L(E, rv, nullptr, nullptr, nullptr, E.d_D, bead_part, (const char *)dn, ds, st);
        ps_launch(k_ps_reduce, TB.nblk, RB_THREADS, 0, st, TB, E.d_lubc_ptr, E.d_ppart, bead_part, sA, sB,
                E.d_pcg, 1, maxit, E.d_nactive);
        PS_CK(cudaMemcpyAsync(E.h_nactive, E.d_nactive, sizeof(int), cudaMemcpyDeviceToHost, st));
        PS_CK(cudaStreamSynchronize(st));
        nact = *E.h_nactive;
        int k = 0;
        while (nact > 0 && k < maxit) {
            for (int j = 0; j < check_every && k < maxit; j++, k++) {
                // Ap = p + L^T Mr L p  (joint replicas: [p_y + L^T (M u)_t ; (M u)_S], u = [L p_y ; p_S])
                launch_ps_L(E, pv, nullptr, nullptr, E.d_pu, nullptr, nullptr, (const char *)dn, ds, st);
                mr_apply(E, fp32, dn, ds, st);
                if (npair)
                    ps_launch(k_ps_LT, nbp_lt, PS_THREADS, 0, st, npair, E.d_lub_pairs, E.d_bead_offs, E.R,
                            E.d_segs, E.d_pS, E.d_py, E.d_py2, nullptr, 1.0,
                            pv, Ap, E.d_ppart, (const char *)dn, ds);
                if (joint)
                    ps_launch(k_ps_S, nbb, thr, 0, st, E.ntot, E.d_bead_offs, E.R, E.d_segs, 1, E.d_pcg, b, E.d_py,
                            E.d_D, yS, rS, zS, pS, ApS, E.d_pu, x, sA, nullptr);
                ps_launch(k_ps_reduce, TB.nblk, RB_THREADS, 0, st, TB, E.d_lubc_ptr, E.d_ppart, nullptr, sA,
                        nullptr, E.d_pcg, 0, maxit, E.d_nactive);
                if (npair)
                    ps_launch(k_ps_update, nbp_lt, PS_THREADS, 0, st, npair, E.d_lub_pairs, E.d_bead_offs, E.R,
                            E.d_segs, E.d_pcg, E.d_pP, pv, Ap, yv, rv,
                            zv, E.d_ppart);
                if (joint)
                    ps_launch(k_ps_S, nbb, thr, 0, st, E.ntot, E.d_bead_offs, E.R, E.d_segs, 2, E.d_pcg, b, E.d_py,
                            E.d_D, yS, rS, zS, pS, ApS, E.d_pu, x, sA, sB);
                launch_ps_L(E, rv, nullptr, nullptr, nullptr, E.d_D, bead_part, (const char *)dn, ds, st);
                ps_launch(k_ps_reduce, TB.nblk, RB_THREADS, 0, st, TB, E.d_lubc_ptr, E.d_ppart, bead_part, sA,
                        sB, E.d_pcg, 2, maxit, E.d_nactive);
                if (npair)
                    ps_launch(k_ps_dir, nbp_e, PS_THREADS, 0, st, npair, E.d_lub_pairs, E.d_bead_offs, E.R,
                            E.d_pcg, zv, pv);
                if (joint)
                    ps_launch(k_ps_S, nbb, thr, 0, st, E.ntot, E.d_bead_offs, E.R, E.d_segs, 3, E.d_pcg, b, E.d_py,
                            E.d_D, yS, rS, zS, pS, ApS, E.d_pu, x, nullptr, nullptr);
            }
            PS_CK(cudaMemcpyAsync(E.h_nactive, E.d_nactive, sizeof(int), cudaMemcpyDeviceToHost, st));
            PS_CK(cudaStreamSynchronize(st));
            nact = *E.h_nactive;
        }
    }
    // F_t = -b_bot + L y (into u_t and the force rows), then U = Mr F_t - g, F_S
    launch_ps_L(E, yv, cvel, tmp, E.d_pu, nullptr, nullptr, nullptr, 0, st);
    ps_launch(k_ps_ft, TV.nblk, RB_THREADS, 0, st, TV, E.d_segs, tmp, x);
    if (joint)
        ps_launch(k_ps_S, nbb, thr, 0, st, E.ntot, E.d_bead_offs, E.R, E.d_segs, 4, E.d_pcg, b, E.d_py, E.d_D,
                yS, rS, zS, pS, ApS, E.d_pu, x, nullptr, nullptr);
    mr_apply(E, fp32, nullptr, 0, st);
    ps_launch(k_ps_fin, TV.nblk, RB_THREADS, 0, st, TV, E.d_segs, E.d_py, E.d_py2, g, x);
    if (E.n_ss_reps)
        ps_launch(k_ss_apply, E.n_ss_reps, 64, 0, st, E.d_segs, E.d_ss_reps, E.d_ssinv, b, 0, 1.0, E.d_py,
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
    ps_launch(k_struct_init, nb, thr, 0, st, E.nvec, E.d_vec_offs, E.R, E.d_segs, b, x);
    if (E.n_ss_reps) {
        apply_operator(E, 0, x, y, nullptr, fp32, st);   // y_top = M [F_t ; 0]
        ps_launch(k_struct_ss, E.n_ss_reps, 256, 0, st, E.d_segs, E.d_ss_reps, E.d_x, E.d_delta, b, y, x);
    }
    apply_operator(E, 0, x, y, nullptr, fp32, st);       // y_top = M F
    ps_launch(k_struct_u, nb, thr, 0, st, E.nvec, E.d_vec_offs, E.R, E.d_segs, b, y, x);
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

// ---------------------------------------------------------------------------
// Brownian lubrication force, rhs_bot += -sqrt(2 kT / dt) sum_p B_p R_p^{1/2} z_p.
// Each canonical pair q owns 12 normals z_q (monomer pairs use the first 6):
// injected (z + 12 q) or drawn from the replica's Philox stream with
// subsequence q - (first canonical pair of the replica).  R_p^{1/2} is the
// symmetric square root that the pair-space setup stores as the pair's S block,
// so the force is the L-gather of the pair-space solve applied to z (one
// evaluation per pair; the staging's setup is shared with the solve after it).
__global__ void k_lub_z(long npair, const int2 *__restrict__ pairs, const int *__restrict__ bead_offs, int R,
                        const Seg *__restrict__ segs, const int *__restrict__ cptr, const uint64_t *__restrict__ rseed,
                        const uint64_t *__restrict__ rstep, double *__restrict__ z)
{
    pdl_enter();
    const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= npair) return;
    const int r = rep_of_b(bead_offs, R, pairs[q].x);
    curandStatePhilox4_32_10_t stt;
    curand_init(rseed[r], (unsigned long long)(q - cptr[segs[r].bead_off]), (3ull * rstep[r] + 2) * 4ull, &stt);
    for (int k = 0; k < 12; k++) z[12 * q + k] = curand_normal_double(&stt);
}

__global__ void k_lub_noise_add(long nvel, const int *__restrict__ vel_offs, int R, const Seg *__restrict__ segs,
                                const double *__restrict__ v, double *__restrict__ rhs)
{
    pdl_enter();
    const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nvel) return;
    const Seg &s = segs[rep_at(vel_offs, R, k)];
    rhs[(long)s.vec_off + s.nm3nc11 + (k - s.vel_off)] += -sqrt(2.0 * s.kT / s.dt) * v[k];
}

int lub_noise(Engine &E, const double *z, double *rhs, cudaStream_t st)
{
    const long npair = E.lub_npairs;
    if (npair <= 0) return PS_OK;
    int rc;
    if ((rc = ensure_pair_space(E))) return rc;
    const unsigned nbp = (unsigned)((npair + PS_THREADS - 1) / PS_THREADS);
    if (!E.ps_setup_valid) {
        launch_ps_setup(E, st);
        E.ps_setup_valid = true;
    }
    if (!z) {
        const long nz = 12 * npair;
        if (nz > E.zlub_cap) {
            cudaFree(E.d_zlub);
            E.zlub_cap = nz * 3 / 2 + 1024;
            PS_CK(cudaMalloc(&E.d_zlub, sizeof(double) * E.zlub_cap));
        }
        ps_launch(k_lub_z, nbp, PS_THREADS, 0, st, npair, E.d_lub_pairs, E.d_bead_offs, E.R, E.d_segs,
                E.d_lubc_ptr, E.d_rseed, E.d_rstep, E.d_zlub);
        z = E.d_zlub;
    }
    launch_ps_L(E, z, nullptr, E.d_tmp_vel, nullptr, nullptr, nullptr, nullptr, 0, st);
    const int thr = 256;
    ps_launch(k_lub_noise_add, (unsigned)((E.nvel + thr - 1) / thr), thr, 0, st,
            E.nvel, E.d_vel_offs, E.R, E.d_segs, E.d_tmp_vel, rhs);
    PS_CK(cudaGetLastError());
    return PS_OK;
}

}  // namespace ps
