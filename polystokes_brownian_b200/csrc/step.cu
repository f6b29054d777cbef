// step.cu -- Brownian noise assembly and the predictor-corrector step of every
// replica (run.cpp:70-162, slip_vel.cpp:19-79/205-349, drift.cpp:9-62,
// traj.cpp:9-94, quat.cpp:7-54).  Compiled with --fmad=false so position
// updates round like the reference's C++.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>
#include <curand_kernel.h>
#include "ps_internal.h"
#include "ps_kernels.h"

namespace ps {

__device__ __forceinline__ int rep_lookup(const int *__restrict__ offs, int R, long k)
{
    int lo = 0, hi = R;
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (offs[mid] <= k) lo = mid; else hi = mid;
    }
    return lo;
}

// ---------------------------------------------------------------------------
// noise: shell (block-Cholesky) path.  u = [fb_m ; 0] is applied through the
// mobility operator so that y_c = Mcm fb_m; then W_m = sqrt(beta_inv) fb_m,
// W_c = sqrt(beta) y_c + Q diag(sqrt(lambda_floored)) Q^T fb_c.
__global__ void k_zero_colloid_dofs(long ntop, const int *__restrict__ top_offs, int R, const Seg *__restrict__ segs,
                                    const double *__restrict__ fb, double *__restrict__ u)
{
    pdl_enter();
    long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= ntop) return;
    int r = rep_lookup(top_offs, R, k);
    const Seg &s = segs[r];
    int i = (int)(k - s.top_off);
    u[k] = (i < s.nm3) ? fb[k] : 0.0;
}

__global__ void k_shell_noise(const Seg *__restrict__ segs, const int *__restrict__ reps, const double *__restrict__ fb,
                              const double *__restrict__ ymcm, const double *__restrict__ schurQ,
                              const double *__restrict__ schurL, double *__restrict__ W)
{
    pdl_enter();
    __shared__ double yv[PS_MAX_NC11_SCHUR];
    const int r = reps[blockIdx.x];
    const Seg &s = segs[r];
    const int n = s.nc11;
    const double *Q = schurQ + s.schur_off, *L = schurL + s.schur_off;
    const double *fc = fb + s.top_off + s.nm3;
    for (int i = threadIdx.x; i < s.nm3; i += blockDim.x) W[s.top_off + i] = sqrt(s.beta_inv) * fb[s.top_off + i];
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        double acc = 0.0;
        for (int i = 0; i < n; i++) acc += Q[i * n + j] * fc[i];
        yv[j] = sqrt(L[j]) * acc;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        double acc = 0.0;
        for (int j = 0; j < n; j++) acc += Q[i * n + j] * yv[j];
        W[s.top_off + s.nm3 + i] = ymcm[s.top_off + s.nm3 + i] * sqrt(s.beta) + acc;
    }
}

int slip_noise(Engine &E, const double *fb, double *W, const ps_sqrt_opts *o, ps_sqrt_result *res, cudaStream_t st)
{
    ps_sqrt_result r0 = {0, 0};
    if (E.any_mmhi) {
        int rc = lanczos_sqrt(E, fb, W, o, &r0, st);
        if (rc) return rc;
    }
    if (E.n_schur_reps || E.n_sl_reps) {
        int thr = 256;
        ps_launch(k_zero_colloid_dofs, (unsigned)((E.ntop + thr - 1) / thr), thr, 0, st, E.ntop, E.d_top_offs, E.R, E.d_segs,
                fb, E.d_tmp_top);
        apply_operator(E, 1, E.d_tmp_top, E.d_tmp_top2, nullptr, false, st);
        if (E.n_schur_reps)
            ps_launch(k_shell_noise, E.n_schur_reps, 128, 0, st, E.d_segs, E.d_schur_reps, fb, E.d_tmp_top2,
                    E.d_schurQ, E.d_schurL, W);
        if (E.n_sl_reps) {
            // above the dense Schur limit: Lanczos on the colloid Schur complement
            int nneg = 0;
            int rc = schur_lanczos_noise(E, fb, E.d_tmp_top2, W, &nneg, st);
            if (rc) return rc;
            r0.nneg += nneg;
        }
    }
    PS_CK(cudaGetLastError());
    if (res) *res = r0;
    return PS_OK;
}

// ---------------------------------------------------------------------------
// device RNG (Philox) for runs without injected noise
// element k of a layout (offs: per-replica offsets) draws from replica r's key
// with subsequence = its index within the replica and offset (3 step + which)
__global__ void k_normals(long n, const int *__restrict__ offs, int R, const uint64_t *__restrict__ rseed,
                          const uint64_t *__restrict__ rstep, int which, double *__restrict__ out)
{
    pdl_enter();
    long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    int r = rep_lookup(offs, R, k);
    curandStatePhilox4_32_10_t stt;
    curand_init(rseed[r], (unsigned long long)(k - offs[r]), (3ull * rstep[r] + which) * 4ull, &stt);
    out[k] = curand_normal_double(&stt);
}

// ---------------------------------------------------------------------------
// elementwise step kernels.  Index spaces: "vel" (nm3nc6 per replica, first
// 3 Np entries are the bead translational DOFs), "top", "vec" (saddle).
__global__ void k_extract_vel(long nvel, const int *__restrict__ vel_offs, int R, const Seg *__restrict__ segs,
                              const double *__restrict__ X, double *__restrict__ out, int from)
{
    pdl_enter();
    long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nvel) return;
    int r = rep_lookup(vel_offs, R, k);
    const Seg &s = segs[r];
    int j = (int)(k - s.vel_off);
    // from = 0: velocity block X[nm3nc11 + j]; from = 1: force block X[j]
    out[k] = X[s.vec_off + (from == 0 ? s.nm3nc11 : 0) + j];
}

__global__ void k_add_noise(long ntop, const int *__restrict__ top_offs, int R, const Seg *__restrict__ segs,
                            const double *__restrict__ W, double *__restrict__ rhs)
{
    pdl_enter();
    long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= ntop) return;
    int r = rep_lookup(top_offs, R, k);
    const Seg &s = segs[r];
    int i = (int)(k - s.top_off);
    double sc = sqrt(2 * s.kT / s.dt);
    rhs[s.vec_off + i] += W[k] * sc;
}

// bead-coordinate kernels: k over 3*ntot position entries
__global__ void k_probe(long n3, const int *__restrict__ bead_offs, int R, const Seg *__restrict__ segs,
                        double *__restrict__ x, const double *__restrict__ fext, double mult)
{
    pdl_enter();
    long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n3) return;
    long b = k / 3;
    int r = rep_lookup(bead_offs, R, b);
    const Seg &s = segs[r];
    long local = k - 3L * s.bead_off;
    const double eps = 1.0e-3;
    x[k] += (mult * eps) * fext[s.vel_off + local];
}

__device__ __forceinline__ double wrap1(double v, double L) { return v - L * nearbyint(v * (1.0 / L)); }

__global__ void k_step_pred(long n3, const int *__restrict__ bead_offs, int R, const Seg *__restrict__ segs,
                            double *__restrict__ x, const double *__restrict__ fext, const double *__restrict__ ud,
                            const double *__restrict__ up)
{
    pdl_enter();
    long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n3) return;
    long b = k / 3;
    int r = rep_lookup(bead_offs, R, b);
    const Seg &s = segs[r];
    long local = k - 3L * s.bead_off;
    const double eps = 1.0e-3;
    double v = x[k];
    if (s.kT > 0) {
        double ds = s.kT / (2.0 * eps);
        v += eps * fext[s.vel_off + local];
        v += ds * ud[s.vel_off + local] * s.dt;
    }
    v += up[s.vel_off + local] * s.dt;
    if (s.box_on) v = wrap1(v, s.L[local % 3]);
    x[k] = v;
}

__global__ void k_step_corr(long n3, const int *__restrict__ bead_offs, int R, const Seg *__restrict__ segs,
                            double *__restrict__ x, const double *__restrict__ xn, const double *__restrict__ ud,
                            double *__restrict__ up, const double *__restrict__ vdn, const double *__restrict__ vdc,
                            const double *__restrict__ vb)
{
    pdl_enter();
    long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n3) return;
    long b = k / 3;
    int r = rep_lookup(bead_offs, R, b);
    const Seg &s = segs[r];
    long local = k - 3L * s.bead_off;
    long q = s.vel_off + local;
    double u = 0.5 * (vdn[q] + vdc[q]) + vb[q];
    up[q] = u;
    double v;
    if (s.kT > 0) {
        double ds = s.kT / (2.0 * 1.0e-3);
        v = xn[k] + ds * ud[q] * s.dt + u * s.dt;
    } else {
        v = xn[k] + u * s.dt;
    }
    if (s.box_on) v = wrap1(v, s.L[local % 3]);
    x[k] = v;
}

// the rotational part of up (not covered by k_step_corr) and the quaternions
__global__ void k_step_rot(long ncoll, const Seg *__restrict__ segs, const int *__restrict__ coll_rep,
                           double *__restrict__ up, const double *__restrict__ vdn, const double *__restrict__ vdc,
                           const double *__restrict__ vb, double *__restrict__ q)
{
    pdl_enter();
    long c = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncoll) return;
    int r = coll_rep[c];
    const Seg &s = segs[r];
    int cl = (int)(c - s.coll_off);
    long o = s.vel_off + s.nm3nc3 + 3 * cl;
    double om[3];
    for (int a = 0; a < 3; a++) {
        om[a] = 0.5 * (vdn[o + a] + vdc[o + a]) + vb[o + a];
        up[o + a] = om[a];
    }
    double *qq = q + 4 * c;
    double w1 = qq[0], x1 = qq[1], y1 = qq[2], z1 = qq[3];
    double w2 = 0.0, x2 = om[0], y2 = om[1], z2 = om[2];
    double d[4] = {w1 * w2 - x1 * x2 - y1 * y2 - z1 * z2, w1 * x2 + x1 * w2 + y1 * z2 - z1 * y2,
                   w1 * y2 - x1 * z2 + y1 * w2 + z1 * x2, w1 * z2 + x1 * y2 - y1 * x2 + z1 * w2};
    double qn[4];
    for (int a = 0; a < 4; a++) qn[a] = qq[a] + 0.5 * d[a] * s.dt;
    double nr = sqrt(qn[0] * qn[0] + qn[1] * qn[1] + qn[2] * qn[2] + qn[3] * qn[3]);
    for (int a = 0; a < 4; a++) qq[a] = qn[a] / nr;
}

// v_brown = up - v_det_n
__global__ void k_sub(long n, const double *__restrict__ a, const double *__restrict__ b, double *__restrict__ out)
{
    pdl_enter();
    long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    out[k] = a[k] - b[k];
}

// udiff = U(x - eps W) - U(x + eps W); sb = (S(+) - S(-)) / (2 eps)
__global__ void k_drift_fin(long nvel, const int *__restrict__ vel_offs, int R, const Seg *__restrict__ segs,
                            const double *__restrict__ Xd, const double *__restrict__ drift, double *__restrict__ ud,
                            double *__restrict__ sb, const double *__restrict__ sbp)
{
    pdl_enter();
    long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nvel) return;
    int r = rep_lookup(vel_offs, R, k);
    const Seg &s = segs[r];
    int j = (int)(k - s.vel_off);
    ud[k] = Xd[s.vec_off + s.nm3nc11 + j] - drift[k];
    if (j < s.nc5) sb[k] = (sbp[s.vec_off + s.nm3nc6 + j] - Xd[s.vec_off + s.nm3nc6 + j]) / (2 * 1.0e-3);
}
__global__ void k_time(int R, const Seg *__restrict__ segs, double *__restrict__ t)
{
    pdl_enter();
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < R) t[r] += segs[r].dt;
}

__global__ void k_step_count(int R, uint64_t *__restrict__ rstep)
{
    pdl_enter();
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < R) rstep[r]++;
}

bool is_host_ptr(const void *p)
{
    if (!p) return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) { cudaGetLastError(); return true; }
    return a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged;
}

static inline unsigned nb(long n, int thr) { return (unsigned)((n + thr - 1) / thr); }

static int stage(Engine &E, double *rhs, cudaStream_t st)
{
    int rc;
    if ((rc = stage_pairs(E, st))) return rc;
    if ((rc = stage_rhs(E, 0, nullptr, rhs, st))) return rc;
    if ((rc = stage_assemble(E, st))) return rc;
    return stage_schur(E, st);
}

// r = b - y
__global__ void k_resid(long n, const double *__restrict__ b, const double *__restrict__ y, double *__restrict__ r)
{
    pdl_enter();
    long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) r[k] = b[k] - y[k];
}

// x += d
__global__ void k_add(long n, const double *__restrict__ d, double *__restrict__ x)
{
    pdl_enter();
    long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) x[k] += d[k];
}

static int solve(Engine &E, const double *b, double *x, int warm, const ps_step_inputs *in, ps_step_result *res,
                 int slot, cudaStream_t st)
{
    ps_ksp_opts o = {in ? in->rtol : 1e-6, in && in->maxit > 0 ? in->maxit : 10000, warm, 8,
                     in ? in->solver : PS_SOLVE_MINRES};
    if (o.rtol <= 0) o.rtol = 1e-6;
    ps_ksp_result kr;
    auto run = [&](const double *rhs, double *sol, ps_ksp_opts &oo) {
        return (oo.method == PS_SOLVE_STRUCTURED) ? structured_solve(E, rhs, sol, &oo, &kr, st)
                                                  : minres_solve(E, rhs, sol, &oo, &kr, st);
    };
    int reason = run(b, x, o);
    if (reason == PS_ERR_CUDA) return reason;
    int its = kr.iters_max, worst = kr.reason;
    // FP64 iterative refinement of the mixed-precision solve: the residual with the FP64
    // operator, a mixed-precision correction, x += d
    const int sweeps = (in && E.precision == PS_PREC_MIXED) ? in->refine : 0;
    if (sweeps > 0) {
        if (!E.d_ref_r) {
            PS_CK(cudaMalloc(&E.d_ref_r, sizeof(double) * E.nvec));
            PS_CK(cudaMalloc(&E.d_ref_d, sizeof(double) * E.nvec));
        }
        const int thr = 256;
        const unsigned g = (unsigned)((E.nvec + thr - 1) / thr);
        for (int k = 0; k < sweeps; k++) {
            apply_operator(E, 0, x, E.d_ref_d, nullptr, false, st);
            ps_launch(k_resid, g, thr, 0, st, E.nvec, b, E.d_ref_d, E.d_ref_r);
            ps_ksp_opts oc = o;
            oc.warm = 0;
            reason = run(E.d_ref_r, E.d_ref_d, oc);
            if (reason == PS_ERR_CUDA) return reason;
            ps_launch(k_add, g, thr, 0, st, E.nvec, E.d_ref_d, x);
            its += kr.iters_max;
            worst = std::min(worst, kr.reason);
        }
        PS_CK(cudaGetLastError());
    }
    if (res) {
        res->iters[slot] = its;
        if (worst < res->reason) res->reason = worst;
    }
    return PS_OK;
}

int step_all(Engine &E, const ps_step_inputs *in, ps_step_result *res, cudaStream_t st)
{
    const int thr = 256;
    int rc;
    if (res) { for (int k = 0; k < 5; k++) res->iters[k] = 0; res->reason = 1000; res->lanczos_iters = 0; res->lanczos_nneg = 0; }
    ps_launch(k_time, (E.R + 127) / 128, 128, 0, st, E.R, E.d_segs, E.d_time);
    PS_CK(cudaMemcpyAsync(E.d_xn, E.d_x, sizeof(double) * 3 * E.ntot, cudaMemcpyDeviceToDevice, st));
    // predictor stage at x_n
    if ((rc = stage(E, E.d_rhs, st))) return rc;
    if ((rc = solve(E, E.d_rhs, E.d_Xdet, 0, in, res, 0, st))) return rc;
    ps_launch(k_extract_vel, nb(E.nvel, thr), thr, 0, st, E.nvel, E.d_vel_offs, E.R, E.d_segs, E.d_Xdet, E.d_vdn, 0);
    if (E.any_kT) {
        const double *fb = in ? in->fb : nullptr;
        const double *wr = in ? in->wrfd : nullptr;
        if (fb && is_host_ptr(fb)) {
            PS_CK(cudaMemcpyAsync(E.d_fb, fb, sizeof(double) * E.ntop, cudaMemcpyHostToDevice, st));
            fb = E.d_fb;
        }
        if (wr && is_host_ptr(wr)) {
            PS_CK(cudaMemcpyAsync(E.d_wr, wr, sizeof(double) * E.nvel, cudaMemcpyHostToDevice, st));
            wr = E.d_wr;
        }
        if (!fb) {
            ps_launch(k_normals, nb(E.ntop, thr), thr, 0, st, E.ntop, E.d_top_offs, E.R, E.d_rseed, E.d_rstep, 0, E.d_fb);
            fb = E.d_fb;
        }
        if (!wr) {
            ps_launch(k_normals, nb(E.nvel, thr), thr, 0, st, E.nvel, E.d_vel_offs, E.R, E.d_rseed, E.d_rstep, 1, E.d_wr);
            wr = E.d_wr;
        }
        ps_sqrt_opts so = {in && in->sqrt_kmax > 0 ? in->sqrt_kmax : 40, in && in->sqrt_tol > 0 ? in->sqrt_tol : 1e-6};
        ps_sqrt_result sr = {0, 0};
        if ((rc = slip_noise(E, fb, E.d_Wn, &so, &sr, st))) return rc;
        if (res) { res->lanczos_iters = sr.iters_max; res->lanczos_nneg = sr.nneg; }
        ps_launch(k_add_noise, nb(E.ntop, thr), thr, 0, st, E.ntop, E.d_top_offs, E.R, E.d_segs, E.d_Wn, E.d_rhs);
        if (E.any_lub && E.lub_npairs > 0) {
            // Brownian lubrication force: 12 normals per canonical pair, injected
            // or drawn from the replica's Philox stream
            const double *zl = in ? in->zlub : nullptr;
            if (zl && is_host_ptr(zl)) {
                long nz = 12 * E.lub_npairs;
                if (nz > E.zlub_cap) {
                    cudaFree(E.d_zlub);
                    E.zlub_cap = nz * 3 / 2 + 1024;
                    PS_CK(cudaMalloc(&E.d_zlub, sizeof(double) * E.zlub_cap));
                }
                PS_CK(cudaMemcpyAsync(E.d_zlub, zl, sizeof(double) * nz, cudaMemcpyHostToDevice, st));
                zl = E.d_zlub;
            }
            if ((rc = lub_noise(E, zl, E.d_rhs, st))) return rc;
        }
        if ((rc = solve(E, E.d_rhs, E.d_X, 0, in, res, 1, st))) return rc;
        ps_launch(k_extract_vel, nb(E.nvel, thr), thr, 0, st, E.nvel, E.d_vel_offs, E.R, E.d_segs, E.d_X, E.d_up, 0);
        ps_launch(k_sub, nb(E.nvel, thr), thr, 0, st, E.nvel, E.d_up, E.d_vdn, E.d_vb);
        // drift(): fext <- W (the quirk of drift.cpp:13 overwrites the recorded forces)
        PS_CK(cudaMemcpyAsync(E.d_fext, wr, sizeof(double) * E.nvel, cudaMemcpyDeviceToDevice, st));
        long n3 = 3 * E.ntot;
        ps_launch(k_probe, nb(n3, thr), thr, 0, st, n3, E.d_bead_offs, E.R, E.d_segs, E.d_x, E.d_fext, 1.0);
        if ((rc = E.any_lub ? stage_pairs(E, st) : stage_pack(E, st))) return rc;
        if ((rc = stage_assemble(E, st))) return rc;
        if ((rc = stage_rhs(E, 1, E.d_fext, E.d_rhs, st))) return rc;
        if ((rc = solve(E, E.d_rhs, E.d_Xd, 0, in, res, 2, st))) return rc;
        ps_launch(k_extract_vel, nb(E.nvel, thr), thr, 0, st, E.nvel, E.d_vel_offs, E.R, E.d_segs, E.d_Xd, E.d_drift, 0);
        PS_CK(cudaMemcpyAsync(E.d_X, E.d_Xd, sizeof(double) * E.nvec, cudaMemcpyDeviceToDevice, st));  // keep S(+)
        ps_launch(k_probe, nb(n3, thr), thr, 0, st, n3, E.d_bead_offs, E.R, E.d_segs, E.d_x, E.d_fext, -2.0);
        if ((rc = E.any_lub ? stage_pairs(E, st) : stage_pack(E, st))) return rc;
        if ((rc = stage_assemble(E, st))) return rc;
        if ((rc = stage_rhs(E, 1, E.d_fext, E.d_rhs, st))) return rc;
        if ((rc = solve(E, E.d_rhs, E.d_Xd, 1, in, res, 3, st))) return rc;
        ps_launch(k_drift_fin, nb(E.nvel, thr), thr, 0, st, E.nvel, E.d_vel_offs, E.R, E.d_segs, E.d_Xd, E.d_drift, E.d_ud,
                E.d_sb, E.d_X);
    } else {
        if ((rc = solve(E, E.d_rhs, E.d_X, 0, in, res, 1, st))) return rc;
        ps_launch(k_extract_vel, nb(E.nvel, thr), thr, 0, st, E.nvel, E.d_vel_offs, E.R, E.d_segs, E.d_X, E.d_up, 0);
        ps_launch(k_extract_vel, nb(E.nvel, thr), thr, 0, st, E.nvel, E.d_vel_offs, E.R, E.d_segs, E.d_X, E.d_fext, 1);
        PS_CK(cudaMemsetAsync(E.d_vb, 0, sizeof(double) * E.nvel, st));
        PS_CK(cudaMemsetAsync(E.d_ud, 0, sizeof(double) * E.nvel, st));
    }
    long n3 = 3 * E.ntot;
    ps_launch(k_step_pred, nb(n3, thr), thr, 0, st, n3, E.d_bead_offs, E.R, E.d_segs, E.d_x, E.d_fext, E.d_ud, E.d_up);
    // corrector stage at x_pred
    if ((rc = stage(E, E.d_rhs, st))) return rc;
    if ((rc = solve(E, E.d_rhs, E.d_Xdet, 0, in, res, 4, st))) return rc;
    ps_launch(k_extract_vel, nb(E.nvel, thr), thr, 0, st, E.nvel, E.d_vel_offs, E.R, E.d_segs, E.d_Xdet, E.d_vdc, 0);
    ps_launch(k_step_corr, nb(n3, thr), thr, 0, st, n3, E.d_bead_offs, E.R, E.d_segs, E.d_x, E.d_xn, E.d_ud, E.d_up, E.d_vdn,
            E.d_vdc, E.d_vb);
    if (E.ncoll)
        ps_launch(k_step_rot, nb(E.ncoll, 128), 128, 0, st, E.ncoll, E.d_segs, E.d_coll_rep, E.d_up, E.d_vdn, E.d_vdc, E.d_vb,
                E.d_q);
    E.step_counter++;
    ps_launch(k_step_count, (E.R + 127) / 128, 128, 0, st, E.R, E.d_rstep);
    PS_CK(cudaGetLastError());
    return PS_OK;
}

}  // namespace ps
