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
// With lubrication the velocities solve the resistance form
//     (R + Mr^{-1}) V = R g - b_bot,   V = U + g,
//     Mr = M_tt - M_tS M_SS^{-1} M_St,  g = b_tt - M_tS M_SS^{-1} b_S,
// by conjugate gradients preconditioned with the far-field mobility Mr, which
// never needs Mr^{-1}: with p = Mr s tracked alongside, (R + Mr^{-1}) p = R p + s.
// The preconditioned operator I + Mr R has its spectrum in [1, 1 + |Mr R|], so
// the iteration count follows the stiffest lubricated gap, not the far field.
// After k iterations the saddle residual is exactly [Mr r_k ; 0 ; 0]: the
// stopping test ||D^{-1} Mr r|| <= rtol ||D^{-1} b|| (D the Jacobi diagonal) is
// the MINRES test of the same system.
//
// Replicas with more than 12 colloids (M_SS not solved densely), and replicas
// whose PCG breaks down because Mr is not positive definite (the reference's
// own monomer pair scalars make M indefinite), take the result as the warm
// start of a MINRES polish.
#include <cmath>
#include <vector>
#include "ps_internal.h"
#include "ps_kernels.h"
#include "ps_reduce.cuh"

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
                           double cb, double *__restrict__ out, int lo, const PcgScal *__restrict__ pc)
{
    __shared__ double in[SS_MAX];
    const int r = reps[blockIdx.x];
    if (pc && pc[r].done) return;
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
        // replicas whose stresslet block is not dense-solved are left to the MINRES polish
        p.done = (s.Nc > 0 && s.ss_off < 0) ? 1 : 0;
        p.reason = p.done ? -1 : 0;
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

// c = R g - b_bot; V = 0; r = s = c; u_t = r
__global__ void k_pcg_init(RedTable T, const Seg *__restrict__ segs, const double *__restrict__ b,
                           const double *__restrict__ Rg, double *__restrict__ V, double *__restrict__ r,
                           double *__restrict__ sv, double *__restrict__ u)
{
    const RBlk B = T.d_blk[blockIdx.x];
    const Seg &s = segs[B.rep];
    for (int e = threadIdx.x; e < B.len; e += RB_THREADS) {
        long k = B.start + e;
        int j = (int)(k - s.vel_off);
        double c = Rg[k] - b[s.vec_off + s.nm3nc11 + j];
        V[k] = 0.0; r[k] = c; sv[k] = c;
        u[s.top_off + j] = c;
    }
}

// z = (M [r ; F_S])_t split over the two applies; err = ||D_t^{-1} z||, rz = r.z
__global__ void k_pcg_z(RedTable T, const Seg *__restrict__ segs, const double *__restrict__ y,
                        const double *__restrict__ y2, const double *__restrict__ D, const double *__restrict__ r,
                        double *__restrict__ z, PcgScal *pc, int first, int maxit, int *nactive)
{
    __shared__ double sh[RB_THREADS / 32][2];
    const RBlk B = T.d_blk[blockIdx.x];
    if (pc[B.rep].done) return;
    const Seg &s = segs[B.rep];
    double v[2] = {0.0, 0.0};
    for (int e = threadIdx.x; e < B.len; e += RB_THREADS) {
        long k = B.start + e;
        int j = (int)(k - s.vel_off);
        double zk = y[s.top_off + j] + (s.ss_off >= 0 ? y2[s.top_off + j] : 0.0);
        z[k] = zk;
        double t = zk / D[s.vec_off + j];
        v[0] += t * t;
        v[1] += r[k] * zk;
    }
    block_sum<2>(v, sh);
    double tot[2];
    if (finish_block<2>(T, B, blockIdx.x, v, tot)) {
        PcgScal p = pc[B.rep];
        p.err = sqrt(tot[0]);
        if (!first) p.it++;
        if (p.err <= p.tol) { p.done = 1; p.reason = 2; }
        else if (tot[1] <= 0.0) { p.done = 1; p.reason = -8; }          // preconditioner not positive
        else if (p.it >= maxit) { p.done = 1; p.reason = -3; }
        else {
            p.beta = first ? 0.0 : tot[1] / p.rz;
            p.rz = tot[1];
        }
        if (p.done) atomicSub(nactive, 1);
        pc[B.rep] = p;
    }
}

// p = z + beta p ; s = r + beta s
__global__ void k_pcg_dir(RedTable T, const PcgScal *__restrict__ pc, const double *__restrict__ z,
                          const double *__restrict__ r, double *__restrict__ p, double *__restrict__ sv, int first)
{
    const RBlk B = T.d_blk[blockIdx.x];
    const PcgScal q = pc[B.rep];
    if (q.done) return;
    for (int e = threadIdx.x; e < B.len; e += RB_THREADS) {
        long k = B.start + e;
        if (first) { p[k] = z[k]; sv[k] = r[k]; }
        else { p[k] = z[k] + q.beta * p[k]; sv[k] = r[k] + q.beta * sv[k]; }
    }
}

// Ap = R p + s ; alpha = rz / p.Ap
__global__ void k_pcg_alpha(RedTable T, const double *__restrict__ Rp, const double *__restrict__ sv,
                            const double *__restrict__ p, double *__restrict__ Ap, PcgScal *pc, int *nactive)
{
    __shared__ double sh[RB_THREADS / 32][1];
    const RBlk B = T.d_blk[blockIdx.x];
    if (pc[B.rep].done) return;
    double v[1] = {0.0};
    for (int e = threadIdx.x; e < B.len; e += RB_THREADS) {
        long k = B.start + e;
        double a = Rp[k] + sv[k];
        Ap[k] = a;
        v[0] += p[k] * a;
    }
    block_sum<1>(v, sh);
    double tot[1];
    if (finish_block<1>(T, B, blockIdx.x, v, tot)) {
        PcgScal q = pc[B.rep];
        if (tot[0] <= 0.0) { q.done = 1; q.reason = -8; atomicSub(nactive, 1); }
        else q.alpha = q.rz / tot[0];
        pc[B.rep] = q;
    }
}

// V += alpha p ; r -= alpha Ap ; u_t = r
__global__ void k_pcg_update(RedTable T, const Seg *__restrict__ segs, const PcgScal *__restrict__ pc,
                             const double *__restrict__ p, const double *__restrict__ Ap, double *__restrict__ V,
                             double *__restrict__ r, double *__restrict__ u)
{
    const RBlk B = T.d_blk[blockIdx.x];
    const PcgScal q = pc[B.rep];
    if (q.done) return;
    const Seg &s = segs[B.rep];
    for (int e = threadIdx.x; e < B.len; e += RB_THREADS) {
        long k = B.start + e;
        V[k] += q.alpha * p[k];
        double rk = r[k] - q.alpha * Ap[k];
        r[k] = rk;
        u[s.top_off + (k - s.vel_off)] = rk;
    }
}

// U = V - g into the saddle solution
__global__ void k_pcg_fin1(RedTable T, const Seg *__restrict__ segs, const double *__restrict__ V,
                           const double *__restrict__ g, double *__restrict__ x)
{
    const RBlk B = T.d_blk[blockIdx.x];
    const Seg &s = segs[B.rep];
    for (int e = threadIdx.x; e < B.len; e += RB_THREADS) {
        long k = B.start + e;
        x[s.vec_off + s.nm3nc11 + (k - s.vel_off)] = V[k] - g[k];
    }
}

// F_t = -b_bot - R U into the saddle solution and into u_t
__global__ void k_pcg_fin2(RedTable T, const Seg *__restrict__ segs, const double *__restrict__ b,
                           const double *__restrict__ RU, double *__restrict__ x, double *__restrict__ u)
{
    const RBlk B = T.d_blk[blockIdx.x];
    const Seg &s = segs[B.rep];
    for (int e = threadIdx.x; e < B.len; e += RB_THREADS) {
        long k = B.start + e;
        int j = (int)(k - s.vel_off);
        double f = -b[s.vec_off + s.nm3nc11 + j] - RU[k];
        x[s.vec_off + j] = f;
        u[s.top_off + j] = f;
    }
}

// Mr r_t -> z (two applies: M [r;0], then M [0; -M_SS^{-1} (M [r;0])_S])
static void pcg_precond(Engine &E, bool fp32, int first, int maxit, cudaStream_t st)
{
    RedTable &TV = E.red_vel;
    const void *dn = &E.d_pcg[0].done;
    const int ds = (int)sizeof(PcgScal);
    apply_operator(E, 1, E.d_pu, E.d_py, nullptr, fp32, st, dn, ds);
    if (E.n_ss_reps) {
        ::ps_launch_count++, k_ss_apply<<<E.n_ss_reps, 64, 0, st>>>(E.d_segs, E.d_ss_reps, E.d_ssinv, E.d_py, 1, -1.0,
                                                                 nullptr, 1, 0.0, E.d_pu2, 1, E.d_pcg);
        apply_operator(E, 1, E.d_pu2, E.d_py2, nullptr, fp32, st, dn, ds, true);
    }
    ::ps_launch_count++, k_pcg_z<<<TV.nblk, RB_THREADS, 0, st>>>(TV, E.d_segs, E.d_py, E.d_py2, E.d_D, E.d_pr, E.d_pz,
                                                              E.d_pcg, first, maxit, E.d_nactive);
    ::ps_launch_count++, k_pcg_dir<<<TV.nblk, RB_THREADS, 0, st>>>(TV, E.d_pcg, E.d_pz, E.d_pr, E.d_pp, E.d_ps, first);
}

static int pcg_lub_solve(Engine &E, const double *b, double *x, const ps_ksp_opts *o, ps_ksp_result *res,
                         cudaStream_t st)
{
    RedTable &TV = E.red_vel;
    const bool fp32 = E.precision == PS_PREC_MIXED;
    const int maxit = o->maxit > 0 ? o->maxit : 10000;
    const int check_every = o->check_every > 0 ? o->check_every : 8;
    int rc = diag_saddle(E, E.d_D, st);
    if (rc) return rc;
    PS_CK(cudaMemsetAsync(x, 0, sizeof(double) * E.nvec, st));
    PS_CK(cudaMemsetAsync(E.d_pu, 0, sizeof(double) * E.ntop, st));
    PS_CK(cudaMemsetAsync(E.d_pu2, 0, sizeof(double) * E.ntop, st));
    PS_CK(cudaMemsetAsync(E.d_py2, 0, sizeof(double) * E.ntop, st));
    ::ps_launch_count++, k_pcg_start<<<E.red.nblk, RB_THREADS, 0, st>>>(E.red, E.d_segs, b, E.d_D, E.d_pcg, o->rtol);
    if (E.n_ss_reps) {
        ::ps_launch_count++, k_ss_inverse<<<E.n_ss_reps, 64, 0, st>>>(E.d_segs, E.d_ss_reps, E.d_x, E.d_delta, E.d_ssinv);
        // g: u2 = [0 ; M_SS^{-1} b_S]
        ::ps_launch_count++, k_ss_apply<<<E.n_ss_reps, 64, 0, st>>>(E.d_segs, E.d_ss_reps, E.d_ssinv, b, 0, 1.0, nullptr,
                                                                 0, 0.0, E.d_pu2, 1, nullptr);
        apply_operator(E, 1, E.d_pu2, E.d_py2, nullptr, fp32, st, nullptr, 0, true);
    }
    ::ps_launch_count++, k_pcg_g<<<TV.nblk, RB_THREADS, 0, st>>>(TV, E.d_segs, b, E.d_py2, E.d_pg);
    lub_apply_vel(E, E.d_pg, E.d_tmp_vel, st);
    ::ps_launch_count++, k_pcg_init<<<TV.nblk, RB_THREADS, 0, st>>>(TV, E.d_segs, b, E.d_tmp_vel, E.d_pV, E.d_pr, E.d_ps,
                                                                 E.d_pu);
    PS_CK(cudaGetLastError());
    std::vector<PcgScal> hp(E.R);
    PS_CK(cudaMemcpyAsync(hp.data(), E.d_pcg, sizeof(PcgScal) * E.R, cudaMemcpyDeviceToHost, st));
    PS_CK(cudaStreamSynchronize(st));
    int nact = 0;
    for (auto &p : hp) nact += !p.done;
    *E.h_nactive = nact;
    PS_CK(cudaMemcpyAsync(E.d_nactive, E.h_nactive, sizeof(int), cudaMemcpyHostToDevice, st));
    if (nact > 0) pcg_precond(E, fp32, 1, maxit, st);
    int k = 0;
    while (nact > 0 && k < maxit) {
        for (int j = 0; j < check_every && k < maxit; j++, k++) {
            lub_apply_vel(E, E.d_pp, E.d_tmp_vel, st);
            ::ps_launch_count++, k_pcg_alpha<<<TV.nblk, RB_THREADS, 0, st>>>(TV, E.d_tmp_vel, E.d_ps, E.d_pp, E.d_pAp,
                                                                          E.d_pcg, E.d_nactive);
            ::ps_launch_count++, k_pcg_update<<<TV.nblk, RB_THREADS, 0, st>>>(TV, E.d_segs, E.d_pcg, E.d_pp, E.d_pAp,
                                                                           E.d_pV, E.d_pr, E.d_pu);
            pcg_precond(E, fp32, 0, maxit, st);
        }
        PS_CK(cudaMemcpyAsync(E.h_nactive, E.d_nactive, sizeof(int), cudaMemcpyDeviceToHost, st));
        PS_CK(cudaStreamSynchronize(st));
        nact = *E.h_nactive;
    }
    // reconstruct [F_t ; F_S ; U]
    ::ps_launch_count++, k_pcg_fin1<<<TV.nblk, RB_THREADS, 0, st>>>(TV, E.d_segs, E.d_pV, E.d_pg, x);
    lub_apply(E, x, E.d_tmp_vel, st);
    ::ps_launch_count++, k_pcg_fin2<<<TV.nblk, RB_THREADS, 0, st>>>(TV, E.d_segs, b, E.d_tmp_vel, x, E.d_pu);
    if (E.n_ss_reps) {
        apply_operator(E, 1, E.d_pu, E.d_py, nullptr, fp32, st, nullptr, 0, true);   // colloid rows: M_St F_t
        ::ps_launch_count++, k_ss_apply<<<E.n_ss_reps, 64, 0, st>>>(E.d_segs, E.d_ss_reps, E.d_ssinv, b, 0, 1.0, E.d_py,
                                                                 1, -1.0, x, 0, nullptr);
    }
    PS_CK(cudaGetLastError());
    PS_CK(cudaMemcpyAsync(hp.data(), E.d_pcg, sizeof(PcgScal) * E.R, cudaMemcpyDeviceToHost, st));
    PS_CK(cudaStreamSynchronize(st));
    int worst = 1000, itmax = 0;
    long itsum = 0;
    double emax = 0;
    for (auto &p : hp) {
        if (p.reason == -1) continue;               // left to the polish
        int reason = p.done ? p.reason : -3;
        worst = std::min(worst, reason);
        itmax = std::max(itmax, p.it);
        itsum += p.it;
        emax = std::max(emax, p.err);
    }
    if (worst == 1000) worst = 2;
    if (res) { res->reason = worst; res->iters_max = itmax; res->iters_sum = itsum; res->rnorm_max = emax; }
    return PS_OK;
}

int structured_solve(Engine &E, const double *b, double *x, const ps_ksp_opts *o, ps_ksp_result *res,
                     cudaStream_t st)
{
    if (E.any_lub) {
        ps_ksp_result r0 = {2, 0, 0, 0.0};
        int rc = pcg_lub_solve(E, b, x, o, &r0, st);
        if (rc) return rc;
        // replicas beyond the dense stresslet limit, and any whose PCG broke down
        // (an indefinite far-field mobility: the reference's own pair scalars),
        // finish with MINRES from the PCG iterate
        if (E.n_ss_polish || r0.reason < 0) {
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
