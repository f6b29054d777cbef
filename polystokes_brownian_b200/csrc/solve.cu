// solve.cu -- structured saddle solve (PS_SOLVE_STRUCTURED).
//
// The saddle system of the reference (arrays.cpp:349-408, matfree_A.cpp:38-80)
//     [ M    B ] [F]   [b_top]        B = [-I_{nm3nc6} ; 0]
//     [ B^T  0 ] [U] = [b_bot]
// splits F = [F_t ; F_S] (forces/torques of every bead, then colloid stresslets)
// and is solved exactly by block elimination:
//     F_t = -b_bot                          (constraint rows)
//     M_SS F_S = b_S - M_St F_t             (dense nc5 x nc5 colloid-stresslet solve)
//     U = (M F)_t - b_t                     (velocity rows)
// which costs two operator applies instead of a Krylov iteration.  The solution
// is the same one MINRES converges to (it is the unique solution of the system).
// Where the elimination is not exact -- the lubrication block in the lower
// right, or a replica with more than 12 colloids whose M_SS is not solved
// densely -- the result is the warm start of a MINRES polish.
#include <cmath>
#include <vector>
#include "ps_internal.h"
#include "ps_kernels.h"

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

// one block per replica with colloids: assemble M_SS (self + colloid pair
// stresslet blocks + the Schur correction of the shell path), solve
// M_SS F_S = b_S - y_S by Gaussian elimination with partial pivoting.
__global__ void k_struct_ss(const Seg *__restrict__ segs, const int *__restrict__ reps, const double *__restrict__ pos_x,
                            const double *__restrict__ delta, const double *__restrict__ b,
                            const double *__restrict__ y, double *__restrict__ x)
{
    __shared__ double A[SS_MAX][SS_MAX + 1];
    __shared__ int piv;
    const int r = reps[blockIdx.x];
    const Seg &s = segs[r];
    const int n = s.nc5, Nc = s.Nc;
    for (int t = threadIdx.x; t < n * (n + 1); t += blockDim.x) {
        int i = t / (n + 1), j = t % (n + 1);
        double v = 0.0;
        if (j == n) {
            v = b[s.vec_off + s.nm3nc6 + i] - y[s.vec_off + s.nm3nc6 + i];
        } else {
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
        }
        A[i][j] = v;
    }
    __syncthreads();
    (void)Nc;
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

int structured_solve(Engine &E, const double *b, double *x, const ps_ksp_opts *o, ps_ksp_result *res,
                     cudaStream_t st)
{
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
    if (E.any_lub || E.n_ss_polish) {
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
