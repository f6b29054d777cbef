// krylov.cu -- batched preconditioned MINRES (KSPSolve stand-in) and the
// Lanczos square root M^{1/2} z, with device-side per-replica scalars and
// convergence flags.
//
// MINRES follows the preconditioned Paige & Saunders (1975) recurrences with
// PETSc KSPMINRES semantics (src/ksp/ksp/impls/minres of PETSc 3.22+; called
// from src/vel.cpp:41-43 of the reference with PCJACOBI fix-diagonal,
// src/init.cpp:217-241): convergence when ||B r0||_2 * prod|s_k| <= rtol * ref,
// ref = ||B r0|| for a zero guess and ||B b|| for a nonzero guess.
//
// Reductions are segmented per replica: each block covers a contiguous range of
// one replica; the last block of a replica to arrive (atomic counter) sums the
// partials in fixed order and runs that replica's scalar update, so the result
// never depends on other replicas or on block scheduling.
#include <cmath>
#include <cstdio>
#include <vector>
#include <cooperative_groups.h>
#include "ps_internal.h"
#include "ps_kernels.h"
#include "ps_reduce.cuh"

namespace ps {

// layout 0: saddle vectors, 1: mobility (top) vectors, 2: velocity vectors, 3: beads
int build_red_table(Engine &E, RedTable &T, int layout)
{
    std::vector<RBlk> blk;
    std::vector<int> first(E.R), cnt(E.R);
    for (int r = 0; r < E.R; r++) {
        const Seg &s = E.segs[r];
        int n = layout == 1 ? s.nm3nc11 : (layout == 2 ? s.nm3nc6 : (layout == 3 ? s.Np : s.n));
        int off = layout == 1 ? s.top_off : (layout == 2 ? s.vel_off : (layout == 3 ? s.bead_off : s.vec_off));
        first[r] = (int)blk.size();
        int nb = (n + RB_SPAN - 1) / RB_SPAN;
        if (nb == 0) nb = 1;
        for (int b = 0; b < nb; b++) {
            int st = b * RB_SPAN, len = std::min(RB_SPAN, n - st);
            if (len < 0) len = 0;
            blk.push_back({r, off + st, len});
        }
        cnt[r] = nb;
    }
    T.nblk = (int)blk.size();
    PS_CK(cudaMalloc(&T.d_blk, sizeof(RBlk) * T.nblk));
    PS_CK(cudaMalloc(&T.d_first, sizeof(int) * E.R));
    PS_CK(cudaMalloc(&T.d_count, sizeof(int) * E.R));
    PS_CK(cudaMalloc(&T.d_counter, sizeof(int) * E.R));
    PS_CK(cudaMalloc(&T.d_part, sizeof(double) * 65 * T.nblk));   // 4 for scalar sums, 65 for Lanczos dots
    PS_CK(cudaMemcpy(T.d_blk, blk.data(), sizeof(RBlk) * T.nblk, cudaMemcpyHostToDevice));
    PS_CK(cudaMemcpy(T.d_first, first.data(), sizeof(int) * E.R, cudaMemcpyHostToDevice));
    PS_CK(cudaMemcpy(T.d_count, cnt.data(), sizeof(int) * E.R, cudaMemcpyHostToDevice));
    PS_CK(cudaMemset(T.d_counter, 0, sizeof(int) * E.R));
    return PS_OK;
}

void free_red_table(RedTable &T)
{
    cudaFree(T.d_blk); cudaFree(T.d_first); cudaFree(T.d_count); cudaFree(T.d_counter); cudaFree(T.d_part);
    T = RedTable();
}

// ---------------------------------------------------------------------------
// generic segmented dot: out[rep] = a.b
__global__ void k_seg_dot(RedTable T, const double *__restrict__ a, const double *__restrict__ b, double *out)
{
    pdl_enter();
    __shared__ double sh[RB_THREADS / 32][1];
    const RBlk B = T.d_blk[blockIdx.x];
    double v[1] = {0.0};
    for (int e = threadIdx.x; e < B.len; e += RB_THREADS) v[0] += a[B.start + e] * b[B.start + e];
    block_sum<1>(v, sh);
    double tot[1];
    if (finish_block<1>(T, B, blockIdx.x, v, tot)) out[B.rep] = tot[0];
}

void seg_dot(Engine &E, RedTable &T, const double *a, const double *b, double *out, cudaStream_t st)
{
    ps_launch(k_seg_dot, T.nblk, RB_THREADS, 0, st, T, a, b, out);
}

// ---------------------------------------------------------------------------
// MINRES
__global__ void k_mr_init(RedTable T, const Seg *segs, const double *__restrict__ b, const double *__restrict__ Ax,
                          const double *__restrict__ D, double *__restrict__ r, double *__restrict__ z,
                          double *__restrict__ x, MinresScal *mr, int warm, double rtol, int maxit,
                          double *__restrict__ v, double *__restrict__ w0, double *__restrict__ w1,
                          double *__restrict__ w2, double *__restrict__ sinv)
{
    pdl_enter();
    __shared__ double sh[RB_THREADS / 32][3];
    const RBlk B = T.d_blk[blockIdx.x];
    double s[3] = {0.0, 0.0, 0.0};
    for (int e = threadIdx.x; e < B.len; e += RB_THREADS) {
        long k = B.start + e;
        double bk = b[k], rk, dk = D[k];
        if (warm) rk = bk - Ax[k];
        else { rk = bk; x[k] = 0.0; }
        double zk = rk / dk;
        r[k] = rk; z[k] = zk;
        v[k] = 0.0; w0[k] = 0.0; w1[k] = 0.0; w2[k] = 0.0;
        s[0] += zk * zk;
        s[1] += rk * zk;
        double bz = bk / dk;
        s[2] += bz * bz;
    }
    block_sum<3>(s, sh);
    double tot[3];
    if (finish_block<3>(T, B, blockIdx.x, s, tot)) {
        MinresScal m = {};
        double np0 = sqrt(tot[0]);
        double ref = warm ? sqrt(tot[2]) : np0;
        double ttol = rtol * ref;
        if (ttol < 1e-50) ttol = 1e-50;
        m.np = np0; m.ttol = ttol; m.it = 0; m.pending = 0;
        (void)maxit;
        if (tot[1] < 0) { m.done = 1; m.reason = -8; }
        else if (np0 <= ttol || tot[1] == 0.0) { m.done = 1; m.reason = 2; }
        else {
            m.done = 0; m.reason = 0;
            m.beta = sqrt(tot[1]); m.oldb = 0; m.dbar = 0; m.epsln = 0; m.phibar = m.beta;
            m.cs = -1; m.sn = 0; m.sinv = 1.0 / m.beta;
        }
        mr[B.rep] = m;
        sinv[B.rep] = m.sinv;
    }
}

// (b) of iteration k: pending w/x update of iteration k-1, v = z/beta,
// Av -= (beta/oldb) r_{k-1}, alfa = v.Av
__global__ void k_mr_alpha(RedTable T, const double *__restrict__ z, double *__restrict__ v,
                           double *__restrict__ Av, const double *__restrict__ rkm1, double *__restrict__ wnew,
                           const double *__restrict__ w1, const double *__restrict__ w2, double *__restrict__ x,
                           MinresScal *mr, int k)
{
    pdl_enter();
    __shared__ double sh[RB_THREADS / 32][1];
    const RBlk B = T.d_blk[blockIdx.x];
    const MinresScal m = mr[B.rep];
    double s[1] = {0.0};
    const bool upd = m.pending != 0;
    const bool act = !m.done;
    const double c1 = (k >= 2) ? m.beta / m.oldb : 0.0;
    for (int e = threadIdx.x; e < B.len; e += RB_THREADS) {
        long q = B.start + e;
        if (upd) {
            double wn = (v[q] - m.up_oldeps * w1[q] - m.up_delta * w2[q]) * m.up_ginv;
            wnew[q] = wn;
            x[q] += m.up_phi * wn;
        }
        if (act) {
            double vq = z[q] * m.sinv;
            double a = Av[q];
            if (k >= 2) a -= c1 * rkm1[q];
            v[q] = vq;
            Av[q] = a;
            s[0] += vq * a;
        }
    }
    block_sum<1>(s, sh);
    double tot[1];
    if (finish_block<1>(T, B, blockIdx.x, s, tot)) {
        if (upd) mr[B.rep].pending = 0;
        if (act) mr[B.rep].alfa = tot[0];
    }
}

// (c) of iteration k: r_{k+1} = Av - (alfa/beta) r_k, z = r_{k+1}/D,
// beta_{k+1} = sqrt(r_{k+1}.z), Givens rotation, convergence test.
__global__ void k_mr_beta(RedTable T, double *__restrict__ Av, const double *__restrict__ rk,
                          const double *__restrict__ D, double *__restrict__ z, MinresScal *mr, int maxit,
                          int *nactive, double *__restrict__ sinv)
{
    pdl_enter();
    __shared__ double sh[RB_THREADS / 32][1];
    const RBlk B = T.d_blk[blockIdx.x];
    const MinresScal m0 = mr[B.rep];
    double s[1] = {0.0};
    const bool act = !m0.done;
    if (act) {
        const double c2 = m0.alfa / m0.beta;
        for (int e = threadIdx.x; e < B.len; e += RB_THREADS) {
            long q = B.start + e;
            double a = Av[q] - c2 * rk[q];
            double zq = a / D[q];
            Av[q] = a;
            z[q] = zq;
            s[0] += a * zq;
        }
    }
    block_sum<1>(s, sh);
    double tot[1];
    if (finish_block<1>(T, B, blockIdx.x, s, tot)) {
        if (!act) return;
        MinresScal m = m0;
        m.it += 1;
        double bb = tot[0];
        m.oldb = m.beta;
        if (bb < 0) { m.done = 1; m.reason = -8; mr[B.rep] = m; atomicSub(nactive, 1); return; }
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
        mr[B.rep] = m;
        sinv[B.rep] = m.sinv;
        if (m.done) atomicSub(nactive, 1);
    }
}

// final pending update (after the last iteration)
__global__ void k_mr_flush(RedTable T, const double *__restrict__ v, double *__restrict__ wnew,
                           const double *__restrict__ w1, const double *__restrict__ w2, double *__restrict__ x,
                           MinresScal *mr)
{
    pdl_enter();
    __shared__ double sh[RB_THREADS / 32][1];
    const RBlk B = T.d_blk[blockIdx.x];
    const MinresScal m = mr[B.rep];
    if (m.pending) {
        for (int e = threadIdx.x; e < B.len; e += RB_THREADS) {
            long q = B.start + e;
            double wn = (v[q] - m.up_oldeps * w1[q] - m.up_delta * w2[q]) * m.up_ginv;
            wnew[q] = wn;
            x[q] += m.up_phi * wn;
        }
    }
    double s[1] = {0.0};
    block_sum<1>(s, sh);
    double tot[1];
    if (finish_block<1>(T, B, blockIdx.x, s, tot)) mr[B.rep].pending = 0;
}

int minres_solve(Engine &E, const double *b, double *x, const ps_ksp_opts *o, ps_ksp_result *res, cudaStream_t st)
{
    ps_ksp_opts opt = {1e-6, 10000, 0, 8, PS_SOLVE_MINRES};
    if (o) opt = *o;
    if (opt.check_every <= 0) opt.check_every = 8;
    if (opt.maxit <= 0) opt.maxit = 10000;
    RedTable &T = E.red;
    int rc = diag_saddle(E, E.d_D, st);
    if (rc) return rc;
    const double *Ax = nullptr;
    if (opt.warm) {
        apply_operator(E, 0, x, E.d_Rr[2], nullptr, false, st);
        Ax = E.d_Rr[2];
    }
    // r_1 in slot 1 (slot k % 3 holds r_k)
    ps_launch(k_mr_init, T.nblk, RB_THREADS, 0, st, T, E.d_segs, b, Ax, E.d_D, E.d_Rr[1], E.d_z, x, E.d_mr, opt.warm,
            opt.rtol, opt.maxit, E.d_v, E.d_W[0], E.d_W[1], E.d_W[2],
            E.d_sinv);
    PS_CK(cudaGetLastError());
    // count active replicas
    std::vector<MinresScal> hm(E.R);
    PS_CK(cudaMemcpyAsync(hm.data(), E.d_mr, sizeof(MinresScal) * E.R, cudaMemcpyDeviceToHost, st));
    PS_CK(cudaStreamSynchronize(st));
    int nact = 0;
    for (auto &m : hm) nact += !m.done;
    *E.h_nactive = nact;
    PS_CK(cudaMemcpyAsync(E.d_nactive, E.h_nactive, sizeof(int), cudaMemcpyHostToDevice, st));
    int k = 0;
    while (nact > 0 && k < opt.maxit) {
        for (int j = 0; j < opt.check_every && k < opt.maxit; j++) {
            k++;
            double *Av = E.d_Rr[(k + 1) % 3];
            const double *rk = E.d_Rr[k % 3];
            const double *rkm1 = E.d_Rr[(k + 2) % 3];
            // iteration k-1's update writes w_{k-1} into slot (k-1)%3; w_{k-2}, w_{k-3}... in the others
            double *wnew = E.d_W[(k + 2) % 3];
            const double *w1 = E.d_W[(k + 0) % 3];   // w_{k-3}
            const double *w2 = E.d_W[(k + 1) % 3];   // w_{k-2}
            // A v_k = (1/beta_k) A z_k: the operator applies the per-replica scale
            apply_operator(E, 0, E.d_z, Av, E.d_sinv, E.precision == PS_PREC_MIXED, st, &E.d_mr[0].done,
                           (int)sizeof(MinresScal));
            ps_launch(k_mr_alpha, T.nblk, RB_THREADS, 0, st, T, E.d_z, E.d_v, Av, rkm1, wnew, w1, w2, x, E.d_mr, k);
            ps_launch(k_mr_beta, T.nblk, RB_THREADS, 0, st, T, Av, rk, E.d_D, E.d_z, E.d_mr, opt.maxit, E.d_nactive,
                    E.d_sinv);
        }
        PS_CK(cudaMemcpyAsync(E.h_nactive, E.d_nactive, sizeof(int), cudaMemcpyDeviceToHost, st));
        PS_CK(cudaStreamSynchronize(st));
        nact = *E.h_nactive;
    }
    // the last iteration's pending update: w_k into slot (k+3)%3 == k%3 ... uses w_{k-1}, w_{k-2}
    {
        int kk = k + 1;
        double *wnew = E.d_W[(kk + 2) % 3];
        const double *w1 = E.d_W[(kk + 0) % 3];
        const double *w2 = E.d_W[(kk + 1) % 3];
        ps_launch(k_mr_flush, T.nblk, RB_THREADS, 0, st, T, E.d_v, wnew, w1, w2, x, E.d_mr);
    }
    PS_CK(cudaMemcpyAsync(hm.data(), E.d_mr, sizeof(MinresScal) * E.R, cudaMemcpyDeviceToHost, st));
    PS_CK(cudaStreamSynchronize(st));
    PS_CK(cudaGetLastError());
    int worst = 1000, itmax = 0;
    long itsum = 0;
    double rmax = 0;
    for (auto &m : hm) {
        int reason = m.done ? m.reason : -3;
        if (reason < worst) worst = reason;
        itmax = std::max(itmax, m.it);
        itsum += m.it;
        rmax = std::max(rmax, m.np);
    }
    if (res) { res->reason = worst; res->iters_max = itmax; res->iters_sum = itsum; res->rnorm_max = rmax; }
    return worst;
}


// ---------------------------------------------------------------------------
// Lanczos square root w = M^{1/2} z on the mobility vectors (top layout), full
// two-pass Gram-Schmidt reorthogonalisation, projected spectrum floored at 0
// (the policy of schur_sqrt_lanczos, slip_vel.cpp:351-477, applied to the full
// grand mobility instead of SLEPc MFN/FNSQRT, slip_vel.cpp:27-49).
struct LzScal {
    double b0;
    int m, done, nneg;
};
constexpr int LZ_KMAX = 64;

// Partial dots of q (held by the block's threads in qv) against V_0..V_j, one
// block of the table; the last block of the replica sums the partials in block
// order into h[].  An inactive block contributes zeros.
__device__ __forceinline__ void lz_dots_block(const RedTable &T, const RBlk &B, const double *__restrict__ V, long ldv,
                                              const double (&qv)[RB_EPT], bool act, int j, double *__restrict__ h)
{
    __shared__ double sh[RB_THREADS / 32][LZ_KMAX + 1];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    // eight basis vectors per pass keep 8 x RB_EPT loads in flight.  Each dot is
    // summed in element order and reduced by the same shuffle tree as one at a time.
    for (int i0 = 0; i0 <= j; i0 += 8) {
        double v[8];
#pragma unroll
        for (int c = 0; c < 8; c++) {
            v[c] = 0.0;
            if (act && i0 + c <= j) {
                const double *Vi = V + (long)(i0 + c) * ldv + B.start;
#pragma unroll
                for (int k = 0; k < RB_EPT; k++) {
                    const int e = threadIdx.x + k * RB_THREADS;
                    if (e < B.len) v[c] += Vi[e] * qv[k];
                }
            }
        }
#pragma unroll
        for (int c = 0; c < 8; c++) {
            double t = v[c];
            for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
            if (lane == 0 && i0 + c <= j) sh[wid][i0 + c] = t;
        }
    }
    __syncthreads();
    // block partial for i stored at d_part[(LZ_KMAX+1) * blk + i]
    if (threadIdx.x <= j) {
        double t = 0;
        for (int w = 0; w < RB_THREADS / 32; w++) t += sh[w][threadIdx.x];
        T.d_part[(long)(LZ_KMAX + 1) * blockIdx.x + threadIdx.x] = t;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = atomicAdd(&T.d_counter[B.rep], 1);
        last = (t == T.d_count[B.rep] - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    int f = T.d_first[B.rep], c = T.d_count[B.rep];
    if (threadIdx.x <= j) {
        double t = 0;
        for (int k = 0; k < c; k++) t += ((volatile double *)T.d_part)[(long)(LZ_KMAX + 1) * (f + k) + threadIdx.x];
        h[(long)(LZ_KMAX + 1) * B.rep + threadIdx.x] = t;
    }
    __syncthreads();
    if (threadIdx.x == 0) T.d_counter[B.rep] = 0;
}

// h = V_0..V_j dotted with q (first pass of the Gram-Schmidt step)
__global__ void k_lz_dots(RedTable T, const double *__restrict__ V, long ldv, const double *__restrict__ q, int j,
                          const LzScal *__restrict__ lz, double *__restrict__ h)
{
    pdl_enter();
    const RBlk B = T.d_blk[blockIdx.x];
    const bool act = !lz[B.rep].done;
    // q held in registers (a block spans at most RB_EPT elements per thread)
    double qv[RB_EPT];
#pragma unroll
    for (int k = 0; k < RB_EPT; k++) {
        const int e = threadIdx.x + k * RB_THREADS;
        qv[k] = (act && e < B.len) ? q[B.start + e] : 0.0;
    }
    lz_dots_block(T, B, V, ldv, qv, act, j, h);
}

// The first pass's subtraction and the second pass's dots in one sweep:
// q -= sum_i h_i V_i (per element in the order i = 0..j), alpha_j = h_j, then
// h2 = V_0..V_j dotted with the new q, which the block still holds in registers.
// The block's slices of V are read twice, the second time from cache.  Same
// arithmetic, in the same order, as the subtraction and dots kernels one after
// the other.
__global__ void k_lz_sub_dots(RedTable T, const double *__restrict__ V, long ldv, double *__restrict__ q, int j,
                              const LzScal *__restrict__ lz, const double *__restrict__ h, double *__restrict__ alpha,
                              double *__restrict__ h2)
{
    pdl_enter();
    const RBlk B = T.d_blk[blockIdx.x];
    const bool act = !lz[B.rep].done;
    double acc[RB_EPT];
    if (act) {
        const double *hr = h + (long)(LZ_KMAX + 1) * B.rep;
#pragma unroll
        for (int k = 0; k < RB_EPT; k++) {
            const int e = threadIdx.x + k * RB_THREADS;
            acc[k] = e < B.len ? q[B.start + e] : 0.0;
        }
#pragma unroll 4
        for (int i = 0; i <= j; i++) {
            const double hi = hr[i];
            const double *Vi = V + (long)i * ldv + B.start;
#pragma unroll
            for (int k = 0; k < RB_EPT; k++) {
                const int e = threadIdx.x + k * RB_THREADS;
                if (e < B.len) acc[k] -= hi * Vi[e];
            }
        }
#pragma unroll
        for (int k = 0; k < RB_EPT; k++) {
            const int e = threadIdx.x + k * RB_THREADS;
            if (e < B.len) q[B.start + e] = acc[k];
            else acc[k] = 0.0;
        }
        if (threadIdx.x == 0 && (B.start == T.d_blk[T.d_first[B.rep]].start))
            alpha[(long)LZ_KMAX * B.rep + j] = 0.0 + hr[j];
    } else {
#pragma unroll
        for (int k = 0; k < RB_EPT; k++) acc[k] = 0.0;
    }
    lz_dots_block(T, B, V, ldv, acc, act, j, h2);
}

// The second pass's subtraction, the norm and the breakdown test in one sweep:
// q -= sum_i h2_i V_i, alpha_j += h2_j, nrm2 = q.q summed as the segmented dot
// sums it (the same elements per thread, shuffle tree and block order), and the
// replica's last block records m = j + 1 and stops the replica on an invariant
// subspace.  A done replica's blocks only take part in the norm, of its
// unchanged q, as the segmented dot would.
__global__ void k_lz_sub_norm(RedTable T, const double *__restrict__ V, long ldv, double *__restrict__ q, int j,
                              LzScal *__restrict__ lz, const double *__restrict__ h2, double *__restrict__ alpha,
                              double *__restrict__ nrm2)
{
    pdl_enter();
    __shared__ double sh[RB_THREADS / 32][1];
    const RBlk B = T.d_blk[blockIdx.x];
    const bool act = !lz[B.rep].done;
    double acc[RB_EPT];
#pragma unroll
    for (int k = 0; k < RB_EPT; k++) {
        const int e = threadIdx.x + k * RB_THREADS;
        acc[k] = e < B.len ? q[B.start + e] : 0.0;
    }
    if (act) {
        const double *hr = h2 + (long)(LZ_KMAX + 1) * B.rep;
#pragma unroll 4
        for (int i = 0; i <= j; i++) {
            const double hi = hr[i];
            const double *Vi = V + (long)i * ldv + B.start;
#pragma unroll
            for (int k = 0; k < RB_EPT; k++) {
                const int e = threadIdx.x + k * RB_THREADS;
                if (e < B.len) acc[k] -= hi * Vi[e];
            }
        }
#pragma unroll
        for (int k = 0; k < RB_EPT; k++) {
            const int e = threadIdx.x + k * RB_THREADS;
            if (e < B.len) q[B.start + e] = acc[k];
        }
        if (threadIdx.x == 0 && (B.start == T.d_blk[T.d_first[B.rep]].start))
            alpha[(long)LZ_KMAX * B.rep + j] = alpha[(long)LZ_KMAX * B.rep + j] + hr[j];
    }
    double v[1] = {0.0};
#pragma unroll
    for (int k = 0; k < RB_EPT; k++) {
        const int e = threadIdx.x + k * RB_THREADS;
        if (e < B.len) v[0] += acc[k] * acc[k];
    }
    block_sum<1>(v, sh);
    double tot[1];
    if (finish_block<1>(T, B, blockIdx.x, v, tot)) {
        nrm2[B.rep] = tot[0];
        LzScal &l = lz[B.rep];
        if (!l.done) {
            l.m = j + 1;
            if (sqrt(tot[0]) <= 1e-12 * l.b0) l.done = 2;   // 2: finalise with m = j+1
        }
    }
}

// V_{j+1} = q / ||q||; beta_j = ||q||  (norm from nrm[rep])
__global__ void k_lz_next(RedTable T, double *__restrict__ V, long ldv, const double *__restrict__ q, int j,
                          LzScal *__restrict__ lz, const double *__restrict__ nrm2, double *__restrict__ betad)
{
    pdl_enter();
    const RBlk B = T.d_blk[blockIdx.x];
    if (lz[B.rep].done) return;
    double bj = sqrt(nrm2[B.rep]);
    double inv = bj > 0 ? 1.0 / bj : 0.0;
    for (int e = threadIdx.x; e < B.len; e += RB_THREADS) V[(long)(j + 1) * ldv + B.start + e] = q[B.start + e] * inv;
    if (threadIdx.x == 0 && (B.start == T.d_blk[T.d_first[B.rep]].start)) betad[(long)LZ_KMAX * B.rep + j] = bj;
}

__global__ void k_lz_init(RedTable T, const Seg *__restrict__ segs, double *__restrict__ V,
                          const double *__restrict__ z, LzScal *__restrict__ lz, const double *__restrict__ nrm2)
{
    pdl_enter();
    const RBlk B = T.d_blk[blockIdx.x];
    // shell replicas take the block-Cholesky noise path instead
    const bool skip = !segs[B.rep].mm_HI;
    double b0 = sqrt(nrm2[B.rep]);
    double inv = b0 > 0 ? 1.0 / b0 : 0.0;
    for (int e = threadIdx.x; e < B.len; e += RB_THREADS) V[B.start + e] = z[B.start + e] * inv;
    if (threadIdx.x == 0 && (B.start == T.d_blk[T.d_first[B.rep]].start)) {
        lz[B.rep].b0 = skip ? 0.0 : b0; lz[B.rep].m = 0; lz[B.rep].done = (b0 == 0.0 || skip); lz[B.rep].nneg = 0;
    }
}

// Implicit QL (symmetric tridiagonal, Wilkinson shift) on one warp.  Lane 0
// runs each QL iteration's scalar recurrence on the shared d, e and records
// the iteration's rotations (c, s) in rot; then every lane applies them, in the
// recurrence's order, to its own rows of Z.  A row sees the same rotations in
// the same order as when each rotation is applied to all rows at once, so Z is
// the same, without a warp barrier per rotation.  rot holds 2 n doubles;
// n <= 64 (two rows of Z per lane).  The warp's lanes search for the split
// point together.  Every lane of the warp takes part.
__device__ void warp_tql(double *d, double *e, double *Z, double *rot, int n)
{
    const int lane = threadIdx.x & 31;
    for (int k = lane; k < n * n; k += 32) Z[k] = (k / n == k % n) ? 1.0 : 0.0;
    __syncwarp();
    for (int l = 0; l < n; l++) {
        int iter = 0;
        while (true) {
            // the first m >= l with a negligible e[m] (n - 1 if none), tested 32 at a time
            int m = n - 1, iend = l;
            for (int m0 = l; m0 < n - 1; m0 += 32) {
                const int mm = m0 + lane;
                bool hit = false;
                if (mm < n - 1) {
                    const double dd = fabs(d[mm]) + fabs(d[mm + 1]);
                    hit = fabs(e[mm]) <= 1e-16 * dd;
                }
                const unsigned b = __ballot_sync(0xffffffffu, hit);
                if (b) { m = m0 + __ffs(b) - 1; break; }
            }
            const bool go = (m != l) && (iter < 60);
            if (lane == 0) {
                if (go) {
                    double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
                    double r = hypot(g, 1.0);
                    g = d[m] - d[l] + e[l] / (g + copysign(r, g));
                    double s = 1, c = 1, p = 0;
                    bool brk = false;
                    for (int i = m - 1; i >= l; i--) {
                        const double ei = e[i], di = d[i], di1 = d[i + 1];
                        double f = s * ei, b = c * ei;
                        // rotation from one reciprocal square root (the chain of dependent
                        // divisions is this loop's latency; f, g are O(|T|), far from overflow)
                        const double r2 = f * f + g * g, ri = r2 > 0.0 ? rsqrt(r2) : 0.0;
                        const double rr = r2 * ri;
                        if (rr == 0.0) {
                            e[i + 1] = rr; d[i + 1] = di1 - p; e[m] = 0.0;
                            brk = true;
                            iend = i + 1;
                            break;
                        }
                        s = f * ri; c = g * ri;
                        g = di1 - p;
                        r = (di - g) * s + 2.0 * c * b;
                        p = s * r;
                        e[i + 1] = rr; d[i + 1] = g + p;
                        g = c * r - b;
                        rot[2 * i] = c; rot[2 * i + 1] = s;
                    }
                    if (!brk) { d[l] -= p; e[l] = g; e[m] = 0.0; }
                }
            }
            iter++;
            iend = __shfl_sync(0xffffffffu, iend, 0);
            if (!go) break;
            __syncwarp();                       // rot, d, e written by lane 0 are visible
            // rows lane and lane + 32 (n <= 64) advance together, each in the order i = m-1 .. iend
            const int k0 = lane, k1 = lane + 32;
            if (k0 < n) {
                double *Z0 = Z + k0 * n, *Z1 = Z + (k1 < n ? k1 : k0) * n;
                const bool two = k1 < n;
                for (int i = m - 1; i >= iend; i--) {
                    const double c = rot[2 * i], sn = rot[2 * i + 1];
                    const double f0 = Z0[i + 1], g0 = Z0[i];
                    double f1 = 0.0, g1 = 0.0;
                    if (two) { f1 = Z1[i + 1]; g1 = Z1[i]; }
                    Z0[i + 1] = sn * g0 + c * f0;
                    Z0[i] = c * g0 - sn * f0;
                    if (two) {
                        Z1[i + 1] = sn * g1 + c * f1;
                        Z1[i] = c * g1 - sn * f1;
                    }
                }
            }
            __syncwarp();
        }
    }
}

// A check's outcome for one replica, written by the speculative checks.
struct LzSpec {
    int conv;      // converged at m
    int m;
    int fin;       // converged, or already done when the check started
    int pad;
};

// one warp per replica: eig of T_m, g = b0 U sqrt(max(theta,0)) U^T e1,
// convergence ||g - g_prev|| <= tol ||g|| (the Lanczos basis is orthonormal).
// final_ = 1: the final estimate, on the replica's own m when it is done, into lz.
// final_ = 0: a speculative check beside the next basis vectors: it reads the
// snapshot `snap` of lz taken when it was launched (the vectors that follow
// move lz on) and writes its outcome into spec; the host applies it later
// (k_lz_spec_apply).  g_prev is the previous check's g in both cases.
__global__ void k_lz_check(int R, LzScal *__restrict__ lz, const LzScal *__restrict__ snap, LzSpec *__restrict__ spec,
                           const double *__restrict__ alpha, const double *__restrict__ betad, double *__restrict__ gbuf,
                           int m, double tol, int final_)
{
    pdl_enter();
    extern __shared__ double sm[];
    const int r = blockIdx.x;
    const LzScal L = final_ ? lz[r] : snap[r];
    const int lane = threadIdx.x;
    if (!final_ && L.done) {
        if (lane == 0) spec[r] = LzSpec{0, L.m, 1, 0};
        return;
    }
    int mr = L.done ? L.m : m;
    if (mr <= 0) {
        if (!final_ && lane == 0) spec[r] = LzSpec{0, 0, 0, 0};
        return;
    }
    double *d = sm, *e = sm + LZ_KMAX, *Z = sm + 2 * LZ_KMAX, *rot = Z + LZ_KMAX * LZ_KMAX;
    for (int i = lane; i < mr; i += 32) {
        d[i] = alpha[(long)LZ_KMAX * r + i];
        e[i] = (i < mr - 1) ? betad[(long)LZ_KMAX * r + i] : 0.0;
    }
    __syncwarp();
    warp_tql(d, e, Z, rot, mr);
    __syncwarp();
    double *g = gbuf + (long)(LZ_KMAX + 1) * r;   // g[0..m-1], g[LZ_KMAX] = |g|^2 of previous
    double diff2 = 0, nrm2 = 0;
    int nneg = 0;
    for (int i = lane; i < LZ_KMAX; i += 32) {
        double gi = 0;
        if (i < mr) {
            for (int j = 0; j < mr; j++) {
                double th = d[j];
                double sq = th > 0 ? sqrt(th) : 0.0;
                gi += Z[i * mr + j] * sq * Z[0 * mr + j];
            }
            gi *= L.b0;
        }
        double old = g[i];
        diff2 += (gi - old) * (gi - old);
        nrm2 += gi * gi;
        if (i < mr) g[i] = gi;
    }
    for (int j = lane; j < mr; j += 32) nneg += d[j] < 0.0;
    for (int o = 16; o > 0; o >>= 1) {
        diff2 += __shfl_down_sync(0xffffffffu, diff2, o);
        nrm2 += __shfl_down_sync(0xffffffffu, nrm2, o);
        nneg += __shfl_down_sync(0xffffffffu, nneg, o);
    }
    if (lane == 0) {
        const int conv = sqrt(diff2) <= tol * sqrt(nrm2);
        if (final_) {
            lz[r].nneg = nneg;
            if (!lz[r].done) {
                lz[r].m = mr;
                lz[r].done = 1;
            }
        } else {
            spec[r] = LzSpec{conv, mr, conv, 0};
        }
    }
}

// a speculative check's outcome, applied in stream order after the vectors that
// ran beside it: a replica that had converged at m stops there (done, m), as if
// the check had held the vectors back; the vectors it took meanwhile are unused
__global__ void k_lz_spec_apply(int R, LzScal *__restrict__ lz, const LzSpec *__restrict__ spec)
{
    pdl_enter();
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= R) return;
    if (spec[r].conv) { lz[r].done = 1; lz[r].m = spec[r].m; }
}

// w = V g (top layout)
__global__ void k_lz_combine(RedTable T, const double *__restrict__ V, long ldv, const LzScal *__restrict__ lz,
                             const double *__restrict__ gbuf, double *__restrict__ w)
{
    pdl_enter();
    const RBlk B = T.d_blk[blockIdx.x];
    const int m = lz[B.rep].m;
    const double *g = gbuf + (long)(LZ_KMAX + 1) * B.rep;
    for (int e = threadIdx.x; e < B.len; e += RB_THREADS) {
        double acc = 0;
        for (int i = 0; i < m; i++) acc += g[i] * V[(long)i * ldv + B.start + e];
        w[B.start + e] = (lz[B.rep].b0 == 0.0) ? 0.0 : acc;
    }
}

// One Lanczos iteration's orthogonalisation for small batches, in one launch:
// one cluster of LZC_CTAS blocks per replica.  Both passes of the
// reorthogonalisation (dots against V_0..V_j, then q -= V h), the norm, the
// breakdown test and the next basis vector, with cluster barriers between the
// phases and the cross-block sums read through distributed shared memory.
// The arithmetic is bit for bit that of the launch sequence it replaces
// (k_lz_dots, k_lz_sub_dots, k_lz_sub_norm, k_lz_next): the replica's
// vector is cut into the reduction table's RB_SPAN blocks, each half of a
// block (RB_THREADS threads) forms an RB block's partials with the same
// thread-to-element map, shuffle tree and warp order, and every sum over RB
// blocks runs in block order.  So a replica's noise does not depend on which
// path its batch takes.  Used when the batch fits one wave of clusters and each
// replica at most LZC_SLOTS RB blocks per half-block; a replica that is done
// leaves with its whole cluster (the flag is read before any block writes it).
namespace cgr = cooperative_groups;
constexpr int LZC_CTAS = 8, LZC_HALVES = 2, LZC_THREADS = RB_THREADS * LZC_HALVES, LZC_SLOTS = 4;
constexpr int LZC_VB = LZC_CTAS * LZC_HALVES;         // virtual RB-table blocks per cluster

__global__ void __cluster_dims__(LZC_CTAS, 1, 1) __launch_bounds__(LZC_THREADS)
k_lz_orth_cluster(const Seg *__restrict__ segs, double *__restrict__ V, long ldv, double *__restrict__ q, int j,
                  int kmax, LzScal *__restrict__ lz, double *__restrict__ alpha, double *__restrict__ betad)
{
    pdl_enter();
    cgr::cluster_group cl = cgr::this_cluster();
    const int rank = (int)cl.block_rank();
    const int r = blockIdx.x / LZC_CTAS;
    const int half = threadIdx.x / RB_THREADS, t = threadIdx.x % RB_THREADS;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    constexpr int HW = RB_THREADS / 32;                   // warps per half
    __shared__ double part[2][LZC_HALVES][LZC_SLOTS][LZ_KMAX + 1];   // per pass: RB-block partial dots
    __shared__ double npart[LZC_HALVES][LZC_SLOTS];       // RB-block partial norms
    __shared__ double sh[LZC_THREADS / 32][8];
    __shared__ double hsh[LZ_KMAX + 1];
    if (lz[r].done) return;                     // the whole cluster: no block has written lz yet
    const Seg &s = segs[r];
    const int n = s.nm3nc11;
    const long base = s.top_off;
    const int nb = (n + RB_SPAN - 1) / RB_SPAN, nslot = (nb + LZC_VB - 1) / LZC_VB;
    const int vb = rank * LZC_HALVES + half;
    double alpha_j = 0.0;
    for (int pass = 0; pass < 2; pass++) {
        for (int sl = 0; sl < nslot; sl++) {
            const int rb = vb + LZC_VB * sl;
            const long st = (long)rb * RB_SPAN;
            const int len = rb < nb ? min(RB_SPAN, n - rb * RB_SPAN) : 0;
            double qv[RB_EPT];
#pragma unroll
            for (int k = 0; k < RB_EPT; k++) {
                const int e = t + k * RB_THREADS;
                qv[k] = e < len ? q[base + st + e] : 0.0;
            }
            for (int i0 = 0; i0 <= j; i0 += 8) {
                double v[8];
#pragma unroll
                for (int c = 0; c < 8; c++) {
                    v[c] = 0.0;
                    if (i0 + c <= j) {
                        const double *Vi = V + (long)(i0 + c) * ldv + base + st;
#pragma unroll
                        for (int k = 0; k < RB_EPT; k++) {
                            const int e = t + k * RB_THREADS;
                            if (e < len) v[c] += Vi[e] * qv[k];
                        }
                    }
                }
#pragma unroll
                for (int c = 0; c < 8; c++) {
                    double x = v[c];
                    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
                    if (lane == 0) sh[wid][c] = x;
                }
                __syncthreads();
                if (t < 8 && i0 + t <= j) {
                    double x = 0.0;
                    for (int w = 0; w < HW; w++) x += sh[half * HW + w][t];
                    part[pass][half][sl][i0 + t] = x;
                }
                __syncthreads();
            }
        }
        cl.sync();
        for (int i = threadIdx.x; i <= j; i += LZC_THREADS) {   // h_i over the RB blocks in block order
            double h = 0.0;
            for (int rb = 0; rb < nb; rb++) {
                const int v2 = rb % LZC_VB;
                h += cl.map_shared_rank(&part[pass][v2 % LZC_HALVES][rb / LZC_VB][0], v2 / LZC_HALVES)[i];
            }
            hsh[i] = h;
        }
        __syncthreads();
        for (int sl = 0; sl < nslot; sl++) {                   // q -= sum_i h_i V_i, i = 0..j per element
            const int rb = vb + LZC_VB * sl;
            if (rb >= nb) break;
            const long st = (long)rb * RB_SPAN;
            const int len = min(RB_SPAN, n - rb * RB_SPAN);
            for (int k = 0; k < RB_EPT; k++) {
                const int e = t + k * RB_THREADS;
                if (e >= len) break;
                double acc = q[base + st + e];
                for (int i = 0; i <= j; i++) acc -= hsh[i] * V[(long)i * ldv + base + st + e];
                q[base + st + e] = acc;
            }
        }
        alpha_j += hsh[j];
        __syncthreads();
    }
    for (int sl = 0; sl < nslot; sl++) {                       // RB-block norms, as seg_dot
        const int rb = vb + LZC_VB * sl;
        const long st = (long)rb * RB_SPAN;
        const int len = rb < nb ? min(RB_SPAN, n - rb * RB_SPAN) : 0;
        double x = 0.0;
        for (int e = t; e < len; e += RB_THREADS) x += q[base + st + e] * q[base + st + e];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) sh[wid][0] = x;
        __syncthreads();
        if (t == 0) {
            double y = 0.0;
            for (int w = 0; w < HW; w++) y += sh[half * HW + w][0];
            npart[half][sl] = y;
        }
        __syncthreads();
    }
    cl.sync();
    double nrm2 = 0.0;
    for (int rb = 0; rb < nb; rb++) {
        const int v2 = rb % LZC_VB;
        nrm2 += cl.map_shared_rank(&npart[v2 % LZC_HALVES][rb / LZC_VB], v2 / LZC_HALVES)[0];
    }
    cl.sync();                                  // no block leaves while others read its shared memory
    const double bj = sqrt(nrm2);
    const bool broken = bj <= 1e-12 * lz[r].b0;
    if (rank == 0 && threadIdx.x == 0) {
        alpha[(long)LZ_KMAX * r + j] = alpha_j;
        lz[r].m = j + 1;
        if (broken) lz[r].done = 2;             // invariant subspace: finalise with m = j + 1
        else if (j + 1 < kmax) betad[(long)LZ_KMAX * r + j] = bj;
    }
    if (!broken && j + 1 < kmax) {
        const double inv = bj > 0 ? 1.0 / bj : 0.0;
        for (int sl = 0; sl < nslot; sl++) {
            const int rb = vb + LZC_VB * sl;
            if (rb >= nb) break;
            const long st = (long)rb * RB_SPAN;
            const int len = min(RB_SPAN, n - rb * RB_SPAN);
            for (int e = t; e < len; e += RB_THREADS) V[(long)(j + 1) * ldv + base + st + e] = q[base + st + e] * inv;
        }
    }
}

int lanczos_sqrt(Engine &E, const double *z, double *w, const ps_sqrt_opts *o, ps_sqrt_result *res, cudaStream_t st)
{
    int kmax = o && o->kmax > 0 ? o->kmax : 40;
    double tol = o && o->tol > 0 ? o->tol : 1e-6;
    if (kmax > LZ_KMAX) kmax = LZ_KMAX;
    RedTable &T = E.red_top;
    long ldv = E.ntop;
    double *V = E.d_lzV, *q = E.d_lzq;
    LzScal *lz = (LzScal *)E.d_lzs;
    double *h = E.d_lzT;                                    // [R][LZ_KMAX+1]
    double *alpha = h + (long)(LZ_KMAX + 1) * E.R;          // [R][LZ_KMAX]
    double *betad = alpha + (long)LZ_KMAX * E.R;            // [R][LZ_KMAX]
    double *gbuf = betad + (long)LZ_KMAX * E.R;             // [R][LZ_KMAX+1]
    double *nrm2 = gbuf + (long)(LZ_KMAX + 1) * E.R;        // [R]
    double *h2 = nrm2 + E.R;                                // [R][LZ_KMAX+1]: the second pass's dots
    seg_dot(E, T, z, z, nrm2, st);
    ps_launch(k_lz_init, T.nblk, RB_THREADS, 0, st, T, E.d_segs, V, z, lz, nrm2);
    PS_CK(cudaMemsetAsync(gbuf, 0, sizeof(double) * (LZ_KMAX + 1) * E.R, st));
    const int check = 8;   // convergence test every 8 vectors; the cap is handled after the loop
    // batches that fit one wave of clusters orthogonalise in one cluster launch per vector
    bool small = (long)E.R * LZC_CTAS <= 128;
    for (const Seg &sg : E.segs)
        small = small && (sg.nm3nc11 + RB_SPAN - 1) / RB_SPAN <= LZC_VB * LZC_SLOTS;
    size_t smem = sizeof(double) * (4 * LZ_KMAX + LZ_KMAX * LZ_KMAX);
    std::vector<LzScal> hl(E.R);
    LzScal *snap = lz + E.R;                                 // the scalars when a check was launched
    LzSpec *spec = (LzSpec *)(snap + E.R);                   // the checks' outcomes
    LzSpec *hspec = (LzSpec *)E.h_spec;
    bool pending = false;
    int j = 0;
    for (j = 0; j < kmax; j++) {
        apply_operator(E, 1, V + (long)j * ldv, q, nullptr, E.precision == PS_PREC_MIXED, st, &lz[0].done,
                       (int)sizeof(LzScal));
        if (small) {
            ::ps_launch_count++, k_lz_orth_cluster<<<E.R * LZC_CTAS, LZC_THREADS, 0, st>>>(E.d_segs, V, ldv, q, j, kmax, lz,
                                                                                       alpha, betad);
        } else {
            // two-pass classical Gram-Schmidt in three sweeps over the basis, then the next vector
            ps_launch(k_lz_dots, T.nblk, RB_THREADS, 0, st, T, V, ldv, q, j, lz, h);
            ps_launch(k_lz_sub_dots, T.nblk, RB_THREADS, 0, st, T, V, ldv, q, j, lz, h, alpha, h2);
            ps_launch(k_lz_sub_norm, T.nblk, RB_THREADS, 0, st, T, V, ldv, q, j, lz, h2, alpha, nrm2);
            if (j + 1 < kmax)
                ps_launch(k_lz_next, T.nblk, RB_THREADS, 0, st, T, V, ldv, q, j, lz, nrm2, betad);
        }
        if ((j + 1) % check == 0 && j + 1 < kmax) {
            if (pending) {
                // the previous check (normally finished long before): apply its outcomes
                PS_CK(cudaEventSynchronize(E.ev_chk));
                pending = false;
                ps_launch(k_lz_spec_apply, (E.R + 127) / 128, 128, 0, st, E.R, lz, spec);
                bool all = true;
                for (int r = 0; r < E.R; r++) all &= hspec[r].fin != 0;
                if (all) break;
            }
            // check at m = j + 1 beside the next vectors, on a snapshot of the scalars
            PS_CK(cudaMemcpyAsync(snap, lz, sizeof(LzScal) * E.R, cudaMemcpyDeviceToDevice, st));
            PS_CK(cudaEventRecord(E.ev_fork2, st));
            PS_CK(cudaStreamWaitEvent(E.side2, E.ev_fork2, 0));
            ps_launch(k_lz_check, E.R, 32, smem, E.side2, E.R, lz, snap, spec, alpha, betad, gbuf, j + 1,
                    tol, 0);
            PS_CK(cudaMemcpyAsync(hspec, spec, sizeof(LzSpec) * E.R, cudaMemcpyDeviceToHost, E.side2));
            PS_CK(cudaEventRecord(E.ev_chk, E.side2));
            pending = true;
        }
    }
    if (pending) {
        // the last check's outcomes, and its g, ahead of the final estimate
        PS_CK(cudaStreamWaitEvent(st, E.ev_chk, 0));
        ps_launch(k_lz_spec_apply, (E.R + 127) / 128, 128, 0, st, E.R, lz, spec);
    }
    // final estimate: replicas at the cap, replicas stopped by breakdown, and the converged ones on their own m
    ps_launch(k_lz_check, E.R, 32, smem, st, E.R, lz, snap, spec, alpha, betad, gbuf,
            std::min(j + 1, kmax), tol, 1);
    ps_launch(k_lz_combine, T.nblk, RB_THREADS, 0, st, T, V, ldv, lz, gbuf, w);
    PS_CK(cudaMemcpyAsync(hl.data(), lz, sizeof(LzScal) * E.R, cudaMemcpyDeviceToHost, st));
    PS_CK(cudaStreamSynchronize(st));
    PS_CK(cudaGetLastError());
    if (res) {
        res->iters_max = 0; res->nneg = 0;
        for (auto &l : hl) { res->iters_max = std::max(res->iters_max, l.m); res->nneg += l.nneg; }
    }
    return PS_OK;
}

// ---------------------------------------------------------------------------
// Schur Lanczos noise of the shell (arrowhead) path above the dense Schur limit,
// schur_sqrt_lanczos (slip_vel.cpp:351-477): sqrt(S) xi_c with
// S q = Mcc q - beta Mcm (Mcm^T q) applied matrix-free through two mobility
// applies per vector ([0; q] gives Mcm^T q in the monomer rows and Mcc q in the
// colloid rows; [Mcm^T q; 0] gives Mcm Mcm^T q in the colloid rows), at most
// min(40, nc11) vectors, two-pass reorthogonalisation against the whole basis,
// stop on an invariant subspace (||w|| <= 1e-12 ||xi_c||) or the cap, then the
// square root of the projected tridiagonal with negative eigenvalues floored at
// 0.  One block per such replica for the short vectors (length nc11).
struct SlScal {
    double b0;
    int m, done, nneg, pad;
};
constexpr int SL_THREADS = 256;

// sum over the block in a fixed order (thread-strided partials, shuffle tree, warp order)
__device__ double sl_block_sum(double v)
{
    __shared__ double ws[SL_THREADS / 32];
    __shared__ double tot;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) ws[wid] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        for (int w = 0; w < SL_THREADS / 32; w++) t += ws[w];
        tot = t;
    }
    __syncthreads();
    double r = tot;
    __syncthreads();
    return r;
}

__device__ double sl_dot(const double *a, const double *b, int n)
{
    double acc = 0;
    for (int i = threadIdx.x; i < n; i += SL_THREADS) acc += a[i] * b[i];
    return sl_block_sum(acc);
}

// V_0 = xi_c / ||xi_c||
__global__ void k_sl_init(const Seg *__restrict__ segs, const int *__restrict__ reps, const double *__restrict__ fb,
                          double *__restrict__ V, SlScal *__restrict__ sc, int *__restrict__ skip)
{
    pdl_enter();
    const int slot = blockIdx.x, r = reps[slot];
    const Seg &s = segs[r];
    const int n = s.nc11;
    const double *b = fb + s.top_off + s.nm3;
    const double b0 = sqrt(sl_dot(b, b, n));
    double *V0 = V + s.sl_off;
    const double inv = b0 > 0 ? 1.0 / b0 : 0.0;
    for (int i = threadIdx.x; i < n; i += SL_THREADS) V0[i] = b[i] * inv;
    if (threadIdx.x == 0) {
        sc[slot].b0 = b0; sc[slot].m = 0; sc[slot].nneg = 0; sc[slot].done = (b0 == 0.0);
        skip[r] = (b0 == 0.0);
    }
}

// u = [0 ; V_j] (stage 0) or u = [y_m ; 0] (stage 1) on the Lanczos replicas, 0 elsewhere
__global__ void k_sl_load(long ntop, const int *__restrict__ top_offs, int R, const Seg *__restrict__ segs,
                          const double *__restrict__ V, const SlScal *__restrict__ sc, int j, int stage,
                          const double *__restrict__ y, double *__restrict__ u)
{
    pdl_enter();
    long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= ntop) return;
    int lo = 0, hi = R;
    while (hi - lo > 1) { int mid = (lo + hi) >> 1; if (top_offs[mid] <= k) lo = mid; else hi = mid; }
    const Seg &s = segs[lo];
    const int i = (int)(k - s.top_off);
    double v = 0.0;
    if (s.sl_slot >= 0 && !sc[s.sl_slot].done) {
        if (stage == 0) { if (i >= s.nm3) v = V[s.sl_off + (long)j * s.nc11 + (i - s.nm3)]; }
        else if (i < s.nm3) v = y[k];
    }
    u[k] = v;
}

// one Lanczos vector: w = S V_j - beta_{j-1} V_{j-1}, alpha_j, two reorthogonalisation passes,
// beta_j and V_{j+1} (row j+1 of the basis holds w while it is formed)
__global__ void k_sl_iter(const Seg *__restrict__ segs, const int *__restrict__ reps, double *__restrict__ V,
                          double *__restrict__ ab, SlScal *__restrict__ sc, int *__restrict__ skip,
                          const double *__restrict__ y, const double *__restrict__ y2, int j)
{
    pdl_enter();
    const int slot = blockIdx.x, r = reps[slot];
    if (sc[slot].done) return;
    const Seg &s = segs[r];
    const int n = s.nc11;
    double *Vb = V + s.sl_off;
    double *w = Vb + (long)(j + 1) * n;
    double *alpha = ab + (long)2 * SL_KMAX * slot, *betad = alpha + SL_KMAX;
    const double *yc = y + s.top_off + s.nm3, *y2c = y2 + s.top_off + s.nm3;
    for (int i = threadIdx.x; i < n; i += SL_THREADS) {
        double v = yc[i] - s.beta * y2c[i];
        if (j > 0) v -= betad[j - 1] * Vb[(long)(j - 1) * n + i];
        w[i] = v;
    }
    __syncthreads();
    const double *Vj = Vb + (long)j * n;
    const double aj = sl_dot(Vj, w, n);
    for (int i = threadIdx.x; i < n; i += SL_THREADS) w[i] -= aj * Vj[i];
    __syncthreads();
    for (int pass = 0; pass < 2; pass++)
        for (int l = 0; l <= j; l++) {
            const double *Vl = Vb + (long)l * n;
            const double h = sl_dot(Vl, w, n);
            for (int i = threadIdx.x; i < n; i += SL_THREADS) w[i] -= h * Vl[i];
            __syncthreads();
        }
    const double bj = sqrt(sl_dot(w, w, n));
    const int kmax = n < SL_KMAX ? n : SL_KMAX;
    const bool stop = (bj <= 1e-12 * sc[slot].b0) || (j == kmax - 1);
    if (!stop) {
        const double inv = 1.0 / bj;
        for (int i = threadIdx.x; i < n; i += SL_THREADS) w[i] *= inv;
    }
    if (threadIdx.x == 0) {
        alpha[j] = aj;
        sc[slot].m = j + 1;
        if (stop) { sc[slot].done = 1; skip[r] = 1; }
        else betad[j] = bj;
    }
}

// W_m = sqrt(beta_inv) xi_m; W_c = sqrt(beta) (Mcm xi_m) + b0 V U sqrt(max(theta, 0)) U^T e1
__global__ void k_sl_finish(const Seg *__restrict__ segs, const int *__restrict__ reps, const double *__restrict__ V,
                            const double *__restrict__ ab, SlScal *__restrict__ sc, const double *__restrict__ fb,
                            const double *__restrict__ ymcm, double *__restrict__ W)
{
    pdl_enter();
    __shared__ double d[SL_KMAX], e[SL_KMAX], Z[SL_KMAX * SL_KMAX], g[SL_KMAX], rot[2 * SL_KMAX];
    const int slot = blockIdx.x, r = reps[slot];
    const Seg &s = segs[r];
    const int n = s.nc11, m = sc[slot].m;
    const double b0 = sc[slot].b0;
    for (int i = threadIdx.x; i < s.nm3; i += blockDim.x) W[s.top_off + i] = sqrt(s.beta_inv) * fb[s.top_off + i];
    const double *alpha = ab + (long)2 * SL_KMAX * slot, *betad = alpha + SL_KMAX;
    if (m > 0 && threadIdx.x < 32) {
        for (int i = threadIdx.x; i < m; i += 32) { d[i] = alpha[i]; e[i] = (i < m - 1) ? betad[i] : 0.0; }
        __syncwarp();
        warp_tql(d, e, Z, rot, m);
        __syncwarp();
        int nneg = 0;
        for (int i = threadIdx.x; i < m; i += 32) {
            double gi = 0;
            for (int c = 0; c < m; c++) gi += Z[i * m + c] * (d[c] > 0 ? sqrt(d[c]) : 0.0) * Z[c];
            g[i] = b0 * gi;
            nneg += d[i] < 0.0;
        }
        for (int o = 16; o > 0; o >>= 1) nneg += __shfl_down_sync(0xffffffffu, nneg, o);
        if (threadIdx.x == 0) sc[slot].nneg = nneg;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        double acc = sqrt(s.beta) * ymcm[s.top_off + s.nm3 + i];
        for (int c = 0; c < m; c++) acc += g[c] * V[s.sl_off + (long)c * n + i];
        W[s.top_off + s.nm3 + i] = acc;
    }
}

int schur_lanczos_noise(Engine &E, const double *fb, const double *ymcm, double *W, int *nneg, cudaStream_t st)
{
    if (!E.n_sl_reps) return PS_OK;
    SlScal *sc = (SlScal *)E.d_sl_sc;
    const int ns = E.n_sl_reps;
    int kmax = 0;
    for (auto &s : E.segs)
        if (s.sl_slot >= 0) kmax = std::max(kmax, std::min(s.nc11, SL_KMAX));
    ps_launch(k_sl_init, ns, SL_THREADS, 0, st, E.d_segs, E.d_sl_reps, fb, E.d_slV, sc, E.d_sl_skip);
    const int thr = 256;
    const unsigned gb = (unsigned)((E.ntop + thr - 1) / thr);
    for (int j = 0; j < kmax; j++) {
        ps_launch(k_sl_load, gb, thr, 0, st, E.ntop, E.d_top_offs, E.R, E.d_segs, E.d_slV, sc, j, 0,
                nullptr, E.d_sl_u);
        apply_operator(E, 1, E.d_sl_u, E.d_sl_y, nullptr, false, st, E.d_sl_skip, (int)sizeof(int));
        ps_launch(k_sl_load, gb, thr, 0, st, E.ntop, E.d_top_offs, E.R, E.d_segs, E.d_slV, sc, j, 1,
                E.d_sl_y, E.d_sl_u);
        apply_operator(E, 1, E.d_sl_u, E.d_sl_y2, nullptr, false, st, E.d_sl_skip, (int)sizeof(int));
        ps_launch(k_sl_iter, ns, SL_THREADS, 0, st, E.d_segs, E.d_sl_reps, E.d_slV, E.d_slT, sc,
                E.d_sl_skip, E.d_sl_y, E.d_sl_y2, j);
    }
    ps_launch(k_sl_finish, ns, SL_THREADS, 0, st, E.d_segs, E.d_sl_reps, E.d_slV, E.d_slT, sc, fb, ymcm, W);
    // the operator applies of the next noise draw start from the Lanczos set again
    std::vector<int> skip(E.R, 1);
    for (auto &s : E.segs)
        if (s.sl_slot >= 0) skip[&s - &E.segs[0]] = 0;
    PS_CK(cudaMemcpyAsync(E.d_sl_skip, skip.data(), sizeof(int) * E.R, cudaMemcpyHostToDevice, st));
    std::vector<SlScal> hs(ns);
    PS_CK(cudaMemcpyAsync(hs.data(), sc, sizeof(SlScal) * ns, cudaMemcpyDeviceToHost, st));
    PS_CK(cudaStreamSynchronize(st));
    PS_CK(cudaGetLastError());
    if (nneg) { *nneg = 0; for (auto &h : hs) *nneg += h.nneg; }
    return PS_OK;
}
}  // namespace ps
