// lub.cu -- near-field lubrication on the device (absent from the reference,
// whose lubdat/*.dat tables are never read; hooks at check_dist.cpp:73-85 and
// saddle.cpp:53).  Formulation (Fiore & Swan, J. Fluid Mech. 878 (2019) 544):
// the saddle's lower-right block is -R_lub, R_lub the sum over near pairs of the
// two-body resistance minus the inverted far-field two-body mobility, which is
// what the tables hold.
//
// Pairs: equal-radius pairs (monomer pairs of radius beta, colloid pairs of
// radius 1) with gap r - 2a < lub_gap * a.  Table r2babc.dat columns (r/a, X11A
// X12A Y11A Y12A Y11B Y12B X11C X12C Y11C Y12C), normalised by 6 pi mu a (A),
// 4 pi mu a^2 (B) and 8 pi mu a^3 (C); in the reference's units (6 pi mu = 1)
// the prefactors are a, (2/3) a^2 and (4/3) a^3.  Below the first row
// (xi = r/a - 2 < 0.1) the leading singular terms of Jeffrey & Onishi (1984)
// are added to the first row's value; xi is clamped at 1e-4.  Monomers carry
// only the A (force-velocity) blocks.
//
// Seen from bead b with partner j and d = (x_j - x_b)/r:
//   F_b = a [A11 U_b + A12 U_j] + (2/3)a^2 [B11^T W_b + B21^T W_j]
//   T_b = (2/3)a^2 [B11 U_b + B12 U_j] + (4/3)a^3 [C11 W_b + C12 W_j]
// with B11 = Y11B eps.d, B12 = Y12B eps.d, B21 = -Y12B eps.d.
// Compiled with --fmad=false (pair membership must round like the oracle).
#include <cmath>
#include <curand_kernel.h>
#include <vector>
#include "ps_internal.h"
#include "ps_kernels.h"

namespace ps {

int build_list(Engine &E, int which, long *npairs, cudaStream_t st);

__device__ __forceinline__ int rep_of_b(const int *__restrict__ offs, int R, long k)
{
    int lo = 0, hi = R;
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (offs[mid] <= k) lo = mid; else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ double lub_sing(int col, double xi)
{
    double l = log(xi);
    switch (col) {
    case 0: return 1.0 / (4.0 * xi) - (9.0 / 40.0) * l;
    case 1: return -(1.0 / (4.0 * xi) - (9.0 / 40.0) * l);
    case 2: return -(1.0 / 6.0) * l;
    case 3: return (1.0 / 6.0) * l;
    case 4: return (1.0 / 4.0) * l;
    case 5: return -(1.0 / 4.0) * l;
    case 8: return -(1.0 / 5.0) * l;
    case 9: return -(1.0 / 20.0) * l;
    default: return 0.0;
    }
}

// ten scalar functions at rr = r / a
__device__ void lub_scalars(const double *__restrict__ T, int nr, double rr, double f[10])
{
    double r0 = T[0], rl = T[(nr - 1) * 11];
    if (rr >= rl) { for (int c = 0; c < 10; c++) f[c] = 0.0; return; }
    if (rr <= r0) {
        double xi = rr - 2.0;
        if (xi < 1e-4) xi = 1e-4;
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

__device__ __forceinline__ void mimg_l(const Seg &s, double &dx, double &dy, double &dz)
{
    if (!s.box_on) return;
    dx -= s.L[0] * nearbyint(dx * (1.0 / s.L[0]));
    dy -= s.L[1] * nearbyint(dy * (1.0 / s.L[1]));
    dz -= s.L[2] * nearbyint(dz * (1.0 / s.L[2]));
}

// velocity-vector DOFs of bead b (local index i): translation, rotation (-1 for monomers)
__device__ __forceinline__ void vel_dofs(const Seg &s, int i, int &t, int &w)
{
    if (i < s.Nm) { t = 3 * i; w = -1; }
    else { int c = i - s.Nm; t = s.nm3 + 3 * c; w = s.nm3nc3 + 3 * c; }
}

// y_vel = R_lub u_vel, u read from the velocity block of a saddle vector
// (u_off_kind 0) or from a velocity-layout vector (1); gather over the
// symmetric lubrication partner list.  diag (optional) receives |diag R|.
__global__ void k_lub_apply(long ntot, const int *__restrict__ bead_offs, int R, const Seg *__restrict__ segs,
                            const double *__restrict__ x, const double *__restrict__ tab, int nrow,
                            const int *__restrict__ ptr, const int *__restrict__ nbr, const double *__restrict__ u,
                            int u_saddle, double *__restrict__ y, double *__restrict__ diag)
{
    long b = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= ntot) return;
    int r = rep_of_b(bead_offs, R, b);
    const Seg &s = segs[r];
    int i = (int)(b - s.bead_off);
    int tb, wb;
    vel_dofs(s, i, tb, wb);
    const long uo = u_saddle ? (long)s.vec_off + s.nm3nc11 : (long)s.vel_off;
    double F[3] = {0, 0, 0}, Tq[3] = {0, 0, 0}, dF[3] = {0, 0, 0}, dT[3] = {0, 0, 0};
    const bool mono = i < s.Nm;
    const double a = mono ? s.beta : 1.0, sa = a, sb = (2.0 / 3.0) * a * a, sc = (4.0 / 3.0) * a * a * a;
    for (int q = ptr[b]; q < ptr[b + 1]; q++) {
        long j = nbr[q];
        int jl = (int)(j - s.bead_off);
        int tj, wj;
        vel_dofs(s, jl, tj, wj);
        double dx = x[3 * j] - x[3 * b], dy = x[3 * j + 1] - x[3 * b + 1], dz = x[3 * j + 2] - x[3 * b + 2];
        mimg_l(s, dx, dy, dz);
        double rr = sqrt(dx * dx + dy * dy + dz * dz);
        double d[3] = {dx / rr, dy / rr, dz / rr};
        double f[10];
        lub_scalars(tab, nrow, rr / a, f);
        double Ub[3], Uj[3], Wb[3] = {0, 0, 0}, Wj[3] = {0, 0, 0};
        for (int k = 0; k < 3; k++) { Ub[k] = u[uo + tb + k]; Uj[k] = u[uo + tj + k]; }
        if (!mono) for (int k = 0; k < 3; k++) { Wb[k] = u[uo + wb + k]; Wj[k] = u[uo + wj + k]; }
        double dUb = d[0] * Ub[0] + d[1] * Ub[1] + d[2] * Ub[2], dUj = d[0] * Uj[0] + d[1] * Uj[1] + d[2] * Uj[2];
        for (int k = 0; k < 3; k++) {
            // A v = X dd v + Y (I - dd) v
            F[k] += sa * (f[0] * dUb * d[k] + f[2] * (Ub[k] - dUb * d[k]) + f[1] * dUj * d[k] + f[3] * (Uj[k] - dUj * d[k]));
            dF[k] += sa * (f[0] * d[k] * d[k] + f[2] * (1.0 - d[k] * d[k]));
        }
        if (!mono) {
            // (eps.d) v = d x v ... (eps.d)_{pq} v_q = eps_{pqk} d_k v_q = (v x d)_p ; its transpose gives (d x v)
            double vWb[3] = {Wb[1] * d[2] - Wb[2] * d[1], Wb[2] * d[0] - Wb[0] * d[2], Wb[0] * d[1] - Wb[1] * d[0]};
            double vWj[3] = {Wj[1] * d[2] - Wj[2] * d[1], Wj[2] * d[0] - Wj[0] * d[2], Wj[0] * d[1] - Wj[1] * d[0]};
            double vUb[3] = {Ub[1] * d[2] - Ub[2] * d[1], Ub[2] * d[0] - Ub[0] * d[2], Ub[0] * d[1] - Ub[1] * d[0]};
            double vUj[3] = {Uj[1] * d[2] - Uj[2] * d[1], Uj[2] * d[0] - Uj[0] * d[2], Uj[0] * d[1] - Uj[1] * d[0]};
            double dWb = d[0] * Wb[0] + d[1] * Wb[1] + d[2] * Wb[2], dWj = d[0] * Wj[0] + d[1] * Wj[1] + d[2] * Wj[2];
            for (int k = 0; k < 3; k++) {
                // F_b += sb [B11^T W_b + B21^T W_j], B^T v = -(v x d)
                F[k] += sb * (-f[4] * vWb[k] + f[5] * vWj[k]);
                // T_b += sb [B11 U_b + B12 U_j] + sc [C11 W_b + C12 W_j]
                Tq[k] += sb * (f[4] * vUb[k] + f[5] * vUj[k]);
                Tq[k] += sc * (f[6] * dWb * d[k] + f[8] * (Wb[k] - dWb * d[k]) + f[7] * dWj * d[k] + f[9] * (Wj[k] - dWj * d[k]));
                dT[k] += sc * (f[6] * d[k] * d[k] + f[8] * (1.0 - d[k] * d[k]));
            }
        }
    }
    for (int k = 0; k < 3; k++) y[s.vel_off + tb + k] = F[k];
    if (!mono) for (int k = 0; k < 3; k++) y[s.vel_off + wb + k] = Tq[k];
    if (diag) {
        for (int k = 0; k < 3; k++) diag[s.vel_off + tb + k] = dF[k];
        if (!mono) for (int k = 0; k < 3; k++) diag[s.vel_off + wb + k] = dT[k];
    }
}

// 12x12 (or 6x6) symmetric square root by cyclic Jacobi, negative eigenvalues floored at 0
__device__ void small_sqrt_apply(double *A, int n, const double *z, double *out)
{
    double Q[144];
    for (int k = 0; k < n * n; k++) Q[k] = (k / n == k % n) ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 40; sweep++) {
        double off = 0, tot = 0;
        for (int p = 0; p < n; p++) for (int q = 0; q < n; q++) { double v = A[p * n + q] * A[p * n + q]; tot += v; if (p != q) off += v; }
        if (off <= 1e-30 * tot || off == 0.0) break;
        for (int p = 0; p < n - 1; p++)
            for (int q = p + 1; q < n; q++) {
                double apq = A[p * n + q];
                if (fabs(apq) < 1e-300) continue;
                double theta = (A[q * n + q] - A[p * n + p]) / (2 * apq);
                double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1));
                double c = 1 / sqrt(t * t + 1), sn = t * c;
                for (int k = 0; k < n; k++) {
                    double akp = A[k * n + p], akq = A[k * n + q];
                    A[k * n + p] = c * akp - sn * akq; A[k * n + q] = sn * akp + c * akq;
                }
                for (int k = 0; k < n; k++) {
                    double apk = A[p * n + k], aqk = A[q * n + k];
                    A[p * n + k] = c * apk - sn * aqk; A[q * n + k] = sn * apk + c * aqk;
                    double qkp = Q[k * n + p], qkq = Q[k * n + q];
                    Q[k * n + p] = c * qkp - sn * qkq; Q[k * n + q] = sn * qkp + c * qkq;
                }
            }
    }
    double t[12];
    for (int jj = 0; jj < n; jj++) {
        double acc = 0;
        for (int ii = 0; ii < n; ii++) acc += Q[ii * n + jj] * z[ii];
        double lam = A[jj * n + jj];
        t[jj] = (lam > 0 ? sqrt(lam) : 0.0) * acc;
    }
    for (int ii = 0; ii < n; ii++) {
        double acc = 0;
        for (int jj = 0; jj < n; jj++) acc += Q[ii * n + jj] * t[jj];
        out[ii] = acc;
    }
}

// 12x12 (or 6x6) pair block R_p in the canonical orientation d = (x_hi - x_lo)/r
__device__ void lub_pair_block(const Seg &s, const double *__restrict__ x, const double *__restrict__ tab, int nrow,
                               long lo, long hi, bool mono, double *Rm)
{
    const double a = mono ? s.beta : 1.0, sa = a, sb = (2.0 / 3.0) * a * a, sc = (4.0 / 3.0) * a * a * a;
    double dx = x[3 * hi] - x[3 * lo], dy = x[3 * hi + 1] - x[3 * lo + 1], dz = x[3 * hi + 2] - x[3 * lo + 2];
    mimg_l(s, dx, dy, dz);
    double rr = sqrt(dx * dx + dy * dy + dz * dz);
    double d[3] = {dx / rr, dy / rr, dz / rr};
    double f[10];
    lub_scalars(tab, nrow, rr / a, f);
    const int nd = mono ? 6 : 12;
    for (int k = 0; k < nd * nd; k++) Rm[k] = 0.0;
    for (int p = 0; p < 3; p++)
        for (int qq = 0; qq < 3; qq++) {
            double dd = d[p] * d[qq], id = (p == qq) - dd;
            double a11 = sa * (f[0] * dd + f[2] * id), a12 = sa * (f[1] * dd + f[3] * id);
            Rm[(0 + p) * nd + 0 + qq] = a11; Rm[(3 + p) * nd + 3 + qq] = a11;
            Rm[(0 + p) * nd + 3 + qq] = a12; Rm[(3 + p) * nd + 0 + qq] = a12;
        }
    if (mono) return;
    for (int p = 0; p < 3; p++)
        for (int qq = 0; qq < 3; qq++) {
            int k3 = 3 - p - qq;
            double ed = 0.0;
            if (p != qq && k3 >= 0 && k3 < 3) ed = (((p - qq + 3) % 3) == 2 ? 1.0 : -1.0) * d[k3];
            double b11 = sb * f[4] * ed, b12 = sb * f[5] * ed, b21 = -b12, b22 = -b11;
            Rm[(6 + p) * nd + 0 + qq] = b11; Rm[(6 + p) * nd + 3 + qq] = b12;
            Rm[(9 + p) * nd + 0 + qq] = b21; Rm[(9 + p) * nd + 3 + qq] = b22;
            Rm[(0 + qq) * nd + 6 + p] = b11; Rm[(3 + qq) * nd + 6 + p] = b12;
            Rm[(0 + qq) * nd + 9 + p] = b21; Rm[(3 + qq) * nd + 9 + p] = b22;
            double dd = d[p] * d[qq], id = (p == qq) - dd;
            double c11 = sc * (f[6] * dd + f[8] * id), c12 = sc * (f[7] * dd + f[9] * id);
            Rm[(6 + p) * nd + 6 + qq] = c11; Rm[(9 + p) * nd + 9 + qq] = c11;
            Rm[(6 + p) * nd + 9 + qq] = c12; Rm[(9 + p) * nd + 6 + qq] = c12;
        }
}

// Brownian lubrication force, gathered per bead (no atomics: the sum over a
// bead's pairs runs in ascending partner order, so the result is bit-exact and
// independent of the rest of the batch).  Each canonical pair p = (lo < hi) with
// index q in the canonical CSR list owns 12 normals z_p (monomer pairs use the
// first 6): injected (z + 12 q) or drawn from the replica's Philox stream with
// subsequence = q - (first canonical pair of the replica).  Both beads of a pair
// compute w_p = R_p^{1/2} z_p identically and take their own rows;
// rhs_bot += -sqrt(2 kT / dt) w.
__global__ void k_lub_noise(long ntot, const int *__restrict__ bead_offs, int R, const Seg *__restrict__ segs,
                            const double *__restrict__ x, const double *__restrict__ tab, int nrow,
                            const int *__restrict__ sptr, const int *__restrict__ snbr,
                            const int *__restrict__ cptr, const int *__restrict__ cnbr, const double *__restrict__ z,
                            const uint64_t *__restrict__ rseed, const uint64_t *__restrict__ rstep,
                            double *__restrict__ rhs)
{
    long b = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= ntot) return;
    int r = rep_of_b(bead_offs, R, b);
    const Seg &s = segs[r];
    int i = (int)(b - s.bead_off);
    const bool mono = i < s.Nm;
    const int nd = mono ? 6 : 12;
    const double scale = -sqrt(2 * s.kT / s.dt);
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (int t = sptr[b]; t < sptr[b + 1]; t++) {
        long j = snbr[t];
        const bool low = b < j;
        long lo = low ? b : j, hi = low ? j : b;
        // canonical index of (lo, hi): binary search in lo's ascending list
        int qa = cptr[lo], qb = cptr[lo + 1];
        while (qb - qa > 1) {
            int mid = (qa + qb) >> 1;
            if (cnbr[mid] <= hi) qa = mid; else qb = mid;
        }
        const long q = qa;
        double zp[12];
        if (z) {
            for (int k = 0; k < 12; k++) zp[k] = z[12 * q + k];
        } else {
            curandStatePhilox4_32_10_t stt;
            curand_init(rseed[r], (unsigned long long)(q - cptr[s.bead_off]), (3ull * rstep[r] + 2) * 4ull, &stt);
            for (int k = 0; k < 12; k++) zp[k] = curand_normal_double(&stt);
        }
        double Rm[144], w[12];
        lub_pair_block(s, x, tab, nrow, lo, hi, mono, Rm);
        small_sqrt_apply(Rm, nd, zp, w);
        const int o = low ? 0 : 3;
        for (int k = 0; k < 3; k++) acc[k] += w[o + k];
        if (!mono) for (int k = 0; k < 3; k++) acc[3 + k] += w[6 + o + k];
    }
    int tb, wb;
    vel_dofs(s, i, tb, wb);
    long base = (long)s.vec_off + s.nm3nc11;
    for (int k = 0; k < 3; k++) rhs[base + tb + k] += scale * acc[k];
    if (!mono) for (int k = 0; k < 3; k++) rhs[base + wb + k] += scale * acc[3 + k];
}

// build the symmetric partner list (which 3) and the canonical i<j list (which 2)
int lub_build(Engine &E, cudaStream_t st)
{
    long np = 0;
    int rc = build_list(E, 3, &np, st);
    if (rc) return rc;
    // keep the symmetric list in the lubrication buffers
    if (np + 1 > E.lub_cap) {
        cudaFree(E.d_lub_nbr);
        E.lub_cap = np * 3 / 2 + 1024;
        PS_CK(cudaMalloc(&E.d_lub_nbr, sizeof(int) * E.lub_cap));
    }
    PS_CK(cudaMemcpyAsync(E.d_lub_ptr, E.d_nbr_ptr, sizeof(int) * (E.ntot + 1), cudaMemcpyDeviceToDevice, st));
    if (np) PS_CK(cudaMemcpyAsync(E.d_lub_nbr, E.d_nbr, sizeof(int) * np, cudaMemcpyDeviceToDevice, st));
    // canonical list stays in d_nbr_ptr / d_nbr
    long nc = 0;
    rc = build_list(E, 2, &nc, st);
    E.lub_npairs = nc;
    return rc;
}

void lub_apply(Engine &E, const double *x_saddle, double *y_vel, cudaStream_t st)
{
    int thr = 128;
    ::ps_launch_count++, k_lub_apply<<<(unsigned)((E.ntot + thr - 1) / thr), thr, 0, st>>>(
        E.ntot, E.d_bead_offs, E.R, E.d_segs, E.d_x, E.d_lubtab, E.lub_nrow, E.d_lub_ptr, E.d_lub_nbr, x_saddle, 1,
        y_vel, nullptr);
}

void lub_apply_vel(Engine &E, const double *u_vel, double *y_vel, cudaStream_t st)
{
    int thr = 128;
    ::ps_launch_count++, k_lub_apply<<<(unsigned)((E.ntot + thr - 1) / thr), thr, 0, st>>>(
        E.ntot, E.d_bead_offs, E.R, E.d_segs, E.d_x, E.d_lubtab, E.lub_nrow, E.d_lub_ptr, E.d_lub_nbr, u_vel, 0,
        y_vel, nullptr);
}

int lub_diag(Engine &E, cudaStream_t st)
{
    int thr = 128;
    PS_CK(cudaMemsetAsync(E.d_lub_diag, 0, sizeof(double) * E.nvel, st));
    PS_CK(cudaMemsetAsync(E.d_tmp_vel, 0, sizeof(double) * E.nvel, st));
    ::ps_launch_count++, k_lub_apply<<<(unsigned)((E.ntot + thr - 1) / thr), thr, 0, st>>>(
        E.ntot, E.d_bead_offs, E.R, E.d_segs, E.d_x, E.d_lubtab, E.lub_nrow, E.d_lub_ptr, E.d_lub_nbr, E.d_tmp_vel, 0,
        E.d_tmp_vel2, E.d_lub_diag);
    PS_CK(cudaGetLastError());
    return PS_OK;
}

int lub_noise(Engine &E, const double *z, double *rhs, cudaStream_t st)
{
    int thr = 64;
    ::ps_launch_count++, k_lub_noise<<<(unsigned)((E.ntot + thr - 1) / thr), thr, 0, st>>>(
        E.ntot, E.d_bead_offs, E.R, E.d_segs, E.d_x, E.d_lubtab, E.lub_nrow, E.d_lub_ptr, E.d_lub_nbr, E.d_nbr_ptr,
        E.d_nbr, z, E.d_rseed, E.d_rstep, rhs);
    PS_CK(cudaGetLastError());
    return PS_OK;
}

}  // namespace ps
