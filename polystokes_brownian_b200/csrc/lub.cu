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
#include <vector>
#include "ps_internal.h"
#include "ps_kernels.h"
#include "lub_dev.cuh"

namespace ps {

int build_list(Engine &E, int which, long *npairs, cudaStream_t st);

// y_vel = R_lub u_vel, u read from the velocity block of a saddle vector
// (u_off_kind 0) or from a velocity-layout vector (1); gather over the
// symmetric lubrication partner list.  diag (optional) receives |diag R|.
__global__ void k_lub_apply(long ntot, const int *__restrict__ bead_offs, int R, const Seg *__restrict__ segs,
                            const double *__restrict__ x, const double *__restrict__ tab, int nrow,
                            const int *__restrict__ ptr, const int *__restrict__ nbr, const double *__restrict__ u,
                            int u_saddle, double *__restrict__ y, double *__restrict__ diag)
{
    pdl_enter();
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

__global__ void k_canon_count(long ntot, const int *__restrict__ sptr, const int *__restrict__ snbr, int *__restrict__ cnt)
{
    pdl_enter();
    long b = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= ntot) return;
    int n = 0;
    for (int t = sptr[b]; t < sptr[b + 1]; t++) n += snbr[t] > b;
    cnt[b] = n;
}

__global__ void k_canon_fill(long ntot, const int *__restrict__ sptr, const int *__restrict__ snbr,
                             const int *__restrict__ cptr, int *__restrict__ cnbr, int2 *__restrict__ pairs)
{
    pdl_enter();
    long b = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= ntot) return;
    int q = cptr[b];
    for (int t = sptr[b]; t < sptr[b + 1]; t++)
        if (snbr[t] > b) { cnbr[q] = snbr[t]; pairs[q] = make_int2((int)b, snbr[t]); q++; }
}

// build the symmetric partner list (which 3) and from it the canonical i<j list
// canonical index of every symmetric-list entry (b, j): the position of
// (min, max) in min's ascending canonical list, found once per list build so
// the per-iteration gathers need no search; -1 if absent (lists disagree)
__global__ void k_canon_map(long ntot, const int *__restrict__ sptr, const int *__restrict__ snbr,
                            const int *__restrict__ cptr, const int *__restrict__ cnbr, int *__restrict__ cidx)
{
    pdl_enter();
    long b = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= ntot) return;
    for (int t = sptr[b]; t < sptr[b + 1]; t++) {
        const long j = snbr[t];
        const long lo = b < j ? b : j, hi = b < j ? j : b;
        int qa = cptr[lo], qb = cptr[lo + 1];
        const int qend = qb;
        while (qb - qa > 1) {
            int mid = (qa + qb) >> 1;
            if (cnbr[mid] <= hi) qa = mid; else qb = mid;
        }
        cidx[t] = (qa < qend && cnbr[qa] == hi) ? qa : -1;
    }
}

int lub_build(Engine &E, cudaStream_t st)
{
    E.ps_setup_valid = false;     // new pair list
    long np = 0;
    int rc = build_list(E, 3, &np, st);
    if (rc) return rc;
    // keep the symmetric list in the lubrication buffers
    if (np + 1 > E.lub_cap) {
        cudaFree(E.d_lub_nbr);
        cudaFree(E.d_lub_cidx);
        E.lub_cap = np * 3 / 2 + 1024;
        PS_CK(cudaMalloc(&E.d_lub_nbr, sizeof(int) * E.lub_cap));
        PS_CK(cudaMalloc(&E.d_lub_cidx, sizeof(int) * E.lub_cap));
    }
    PS_CK(cudaMemcpyAsync(E.d_lub_ptr, E.d_nbr_ptr, sizeof(int) * (E.ntot + 1), cudaMemcpyDeviceToDevice, st));
    if (np) PS_CK(cudaMemcpyAsync(E.d_lub_nbr, E.d_nbr, sizeof(int) * np, cudaMemcpyDeviceToDevice, st));
    // canonical list (lo < hi, ascending): the partners j > b of the symmetric
    // list, which holds every pair twice (the membership test is symmetric)
    // (capacity for np entries: a bound whatever the list holds)
    const long nc = np / 2;
    if (np + 1 > E.lubc_cap) {
        cudaFree(E.d_lubc_nbr);
        cudaFree(E.d_lub_pairs);
        E.lubc_cap = np * 3 / 2 + 1024;
        PS_CK(cudaMalloc(&E.d_lubc_nbr, sizeof(int) * E.lubc_cap));
        PS_CK(cudaMalloc(&E.d_lub_pairs, sizeof(int2) * E.lubc_cap));
    }
    int thr = 128;
    unsigned nb = (unsigned)((E.ntot + thr - 1) / thr);
    ps_launch(k_canon_count, nb, thr, 0, st, E.ntot, E.d_lub_ptr, E.d_lub_nbr, E.d_nbr_count);
    if ((rc = exclusive_scan(E, E.d_nbr_count, E.d_lubc_ptr, E.ntot, st))) return rc;
    ps_launch(k_canon_fill, nb, thr, 0, st, E.ntot, E.d_lub_ptr, E.d_lub_nbr, E.d_lubc_ptr, E.d_lubc_nbr,
            E.d_lub_pairs);
    ps_launch(k_canon_map, nb, thr, 0, st, E.ntot, E.d_lub_ptr, E.d_lub_nbr, E.d_lubc_ptr, E.d_lubc_nbr,
            E.d_lub_cidx);
    E.lub_npairs = nc;
    PS_CK(cudaGetLastError());
    return PS_OK;
}

void lub_apply(Engine &E, const double *x_saddle, double *y_vel, cudaStream_t st)
{
    int thr = 128;
    ps_launch(k_lub_apply, (unsigned)((E.ntot + thr - 1) / thr), thr, 0, st,
            E.ntot, E.d_bead_offs, E.R, E.d_segs, E.d_x, E.d_lubtab, E.lub_nrow, E.d_lub_ptr, E.d_lub_nbr, x_saddle, 1,
            y_vel, nullptr);
}

void lub_apply_vel(Engine &E, const double *u_vel, double *y_vel, cudaStream_t st)
{
    int thr = 128;
    ps_launch(k_lub_apply, (unsigned)((E.ntot + thr - 1) / thr), thr, 0, st,
            E.ntot, E.d_bead_offs, E.R, E.d_segs, E.d_x, E.d_lubtab, E.lub_nrow, E.d_lub_ptr, E.d_lub_nbr, u_vel, 0,
            y_vel, nullptr);
}

int lub_diag(Engine &E, cudaStream_t st)
{
    int thr = 128;
    PS_CK(cudaMemsetAsync(E.d_lub_diag, 0, sizeof(double) * E.nvel, st));
    PS_CK(cudaMemsetAsync(E.d_tmp_vel, 0, sizeof(double) * E.nvel, st));
    ps_launch(k_lub_apply, (unsigned)((E.ntot + thr - 1) / thr), thr, 0, st,
            E.ntot, E.d_bead_offs, E.R, E.d_segs, E.d_x, E.d_lubtab, E.lub_nrow, E.d_lub_ptr, E.d_lub_nbr, E.d_tmp_vel, 0,
            E.d_tmp_vel2, E.d_lub_diag);
    PS_CK(cudaGetLastError());
    return PS_OK;
}

}  // namespace ps
