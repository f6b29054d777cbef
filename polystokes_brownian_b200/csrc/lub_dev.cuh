// lub_dev.cuh -- device helpers of the lubrication path: table interpolation
// with the Jeffrey-Onishi near-contact extrapolation, pair resistance blocks,
// and small dense symmetric eigen-decompositions (cyclic Jacobi).
#pragma once
#include <cmath>
#include "ps_internal.h"

namespace ps {

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
__device__ inline void lub_scalars(const double *__restrict__ T, int nr, double rr, double f[10])
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

// 12x12 (or 6x6) pair block R_p in the canonical orientation d = (x_hi - x_lo)/r
// separation direction d and the ten table scalars of the pair; a = bead radius
__device__ inline void lub_pair_geom(const Seg &s, const double *__restrict__ x, const double *__restrict__ tab,
                                     int nrow, long lo, long hi, double a, double d[3], double f[10])
{
    double dx = x[3 * hi] - x[3 * lo], dy = x[3 * hi + 1] - x[3 * lo + 1], dz = x[3 * hi + 2] - x[3 * lo + 2];
    mimg_l(s, dx, dy, dz);
    double rr = sqrt(dx * dx + dy * dy + dz * dz);
    d[0] = dx / rr; d[1] = dy / rr; d[2] = dz / rr;
    lub_scalars(tab, nrow, rr / a, f);
}

// the entries of a pair block that depend on the component pair (p, qq), from
// its ten coefficients g (A11 along/across d, A12 along/across, the rotation-
// translation couplings B11 = g4 E and B12 = g5 E with E v = v x d, C11 and
// C12 along/across); the block is zero elsewhere (nd = 6 for monomer pairs:
// A blocks only)
__device__ __forceinline__ void pair_block_entries(const double d[3], const double g[10], bool mono, int p, int qq,
                                                   double *Rm)
{
    const int nd = mono ? 6 : 12;
    {
        double dd = d[p] * d[qq], id = (p == qq) - dd;
        double a11 = g[0] * dd + g[2] * id, a12 = g[1] * dd + g[3] * id;
        Rm[(0 + p) * nd + 0 + qq] = a11; Rm[(3 + p) * nd + 3 + qq] = a11;
        Rm[(0 + p) * nd + 3 + qq] = a12; Rm[(3 + p) * nd + 0 + qq] = a12;
    }
    if (mono) return;
    int k3 = 3 - p - qq;
    double ed = 0.0;
    if (p != qq && k3 >= 0 && k3 < 3) ed = (((p - qq + 3) % 3) == 2 ? 1.0 : -1.0) * d[k3];
    double b11 = g[4] * ed, b12 = g[5] * ed, b21 = -b12, b22 = -b11;
    Rm[(6 + p) * nd + 0 + qq] = b11; Rm[(6 + p) * nd + 3 + qq] = b12;
    Rm[(9 + p) * nd + 0 + qq] = b21; Rm[(9 + p) * nd + 3 + qq] = b22;
    Rm[(0 + qq) * nd + 6 + p] = b11; Rm[(3 + qq) * nd + 6 + p] = b12;
    Rm[(0 + qq) * nd + 9 + p] = b21; Rm[(3 + qq) * nd + 9 + p] = b22;
    double dd = d[p] * d[qq], id = (p == qq) - dd;
    double c11 = g[6] * dd + g[8] * id, c12 = g[7] * dd + g[9] * id;
    Rm[(6 + p) * nd + 6 + qq] = c11; Rm[(9 + p) * nd + 9 + qq] = c11;
    Rm[(6 + p) * nd + 9 + qq] = c12; Rm[(9 + p) * nd + 6 + qq] = c12;
}

// the lubrication pair block's coefficients: the table scalars with the
// prefactors a (A), (2/3) a^2 (B) and (4/3) a^3 (C)
__device__ __forceinline__ void lub_pair_coeffs(const double f[10], double a, double g[10])
{
    const double sa = a, sb = (2.0 / 3.0) * a * a, sc = (4.0 / 3.0) * a * a * a;
    for (int k = 0; k < 4; k++) g[k] = sa * f[k];
    g[4] = sb * f[4]; g[5] = sb * f[5];
    for (int k = 6; k < 10; k++) g[k] = sc * f[k];
}

__device__ __forceinline__ void lub_pair_entries(const double d[3], const double f[10], double a, bool mono, int p,
                                                 int qq, double *Rm)
{
    double g[10];
    lub_pair_coeffs(f, a, g);
    pair_block_entries(d, g, mono, p, qq, Rm);
}

// square root (eigenvalues floored at 0) of the symmetric 2 x 2 [[a, b], [b, c]]
// by one Jacobi rotation: returns its entries tt, tr, rr
__device__ __forceinline__ void sqrt_sym2(double a, double b, double c, double &tt, double &tr, double &rr)
{
    if (fabs(b) < 1e-300) { tt = a > 0 ? sqrt(a) : 0.0; tr = 0.0; rr = c > 0 ? sqrt(c) : 0.0; return; }
    const double theta = (c - a) / (2 * b);
    const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1));
    const double co = 1 / sqrt(t * t + 1), sn = t * co;
    const double l1 = a - t * b, l2 = c + t * b;
    const double s1 = l1 > 0 ? sqrt(l1) : 0.0, s2 = l2 > 0 ? sqrt(l2) : 0.0;
    tt = co * co * s1 + sn * sn * s2;
    tr = -co * sn * s1 + sn * co * s2;
    rr = sn * sn * s1 + co * co * s2;
}

// Coefficients (placement of pair_block_entries) of K^{1/2}, K a colloid pair
// block with coefficients k (eigenvalues floored at 0), in closed form.  K
// commutes with the exchange of the two colloids (d -> -d) and with rotations
// about d: in the basis [U_lo + U_hi, W_lo - W_hi] / sqrt2 (block I) and
// [U_lo - U_hi, W_lo + W_hi] / sqrt2 (block II) it splits into two 6 x 6 blocks,
// each with one eigenvalue for translation along d, one for rotation along d,
// and a doubly degenerate 2 x 2 block [[a_perp, b], [b, c_perp]] that couples
// translation along e1 to rotation along e1 x d.  The square root keeps that
// structure, so it has coefficients of the same kind.
__device__ inline void colloid_pair_sqrt_coeffs(const double k[10], double g[10])
{
    auto sq = [](double v) { return v > 0 ? sqrt(v) : 0.0; };
    const double aIp = k[0] + k[1], aIIp = k[0] - k[1];        // translation along d
    const double cIp = k[6] - k[7], cIIp = k[6] + k[7];        // rotation along d
    double ttI, trI, rrI, ttII, trII, rrII;
    sqrt_sym2(k[2] + k[3], k[4] + k[5], k[8] - k[9], ttI, trI, rrI);
    sqrt_sym2(k[2] - k[3], k[4] - k[5], k[8] + k[9], ttII, trII, rrII);
    g[0] = 0.5 * (sq(aIp) + sq(aIIp)); g[1] = 0.5 * (sq(aIp) - sq(aIIp));
    g[2] = 0.5 * (ttI + ttII); g[3] = 0.5 * (ttI - ttII);
    g[4] = 0.5 * (trI + trII); g[5] = 0.5 * (trI - trII);
    g[6] = 0.5 * (sq(cIIp) + sq(cIp)); g[7] = 0.5 * (sq(cIIp) - sq(cIp));
    g[8] = 0.5 * (rrII + rrI); g[9] = 0.5 * (rrII - rrI);
}

__device__ inline void lub_pair_block(const Seg &s, const double *__restrict__ x, const double *__restrict__ tab, int nrow,
                               long lo, long hi, bool mono, double *Rm)
{
    const double a = mono ? s.beta : 1.0;
    double d[3], f[10];
    lub_pair_geom(s, x, tab, nrow, lo, hi, a, d, f);
    const int nd = mono ? 6 : 12;
    for (int k = 0; k < nd * nd; k++) Rm[k] = 0.0;
    for (int p = 0; p < 3; p++)
        for (int qq = 0; qq < 3; qq++) lub_pair_entries(d, f, a, mono, p, qq, Rm);
}

// Monomer pair block in closed form.  K = [[A11, A12], [A12, A11]] with
// A11 = a (f0 dd + f2 (I - dd)), A12 = a (f1 dd + f3 (I - dd)): the symmetric
// modes (v, v)/sqrt2 see A11 + A12, the antisymmetric (v, -v)/sqrt2 see
// A11 - A12, each with one eigenvalue along d and a double one across.
// lam = {sym along, sym across, anti along, anti across}; d = (x_hi - x_lo)/r.
__device__ inline void mono_pair_modes(const Seg &s, const double *__restrict__ x, const double *__restrict__ tab,
                                       int nrow, long lo, long hi, double d[3], double lam[4])
{
    const double a = s.beta;
    double dx = x[3 * hi] - x[3 * lo], dy = x[3 * hi + 1] - x[3 * lo + 1], dz = x[3 * hi + 2] - x[3 * lo + 2];
    mimg_l(s, dx, dy, dz);
    double rr = sqrt(dx * dx + dy * dy + dz * dz);
    d[0] = dx / rr; d[1] = dy / rr; d[2] = dz / rr;
    double f[10];
    lub_scalars(tab, nrow, rr / a, f);
    lam[0] = a * (f[0] + f[1]); lam[1] = a * (f[2] + f[3]);
    lam[2] = a * (f[0] - f[1]); lam[3] = a * (f[2] - f[3]);
}

// 6x6 matrix [[B, C], [C, B]] (row-major, leading dimension ld) from mode
// values g = {sym along, sym across, anti along, anti across}:
// B = (Gs + Ga)/2, C = (Gs - Ga)/2, G = g_along dd + g_across (I - dd)
__device__ inline void mono_pair_matrix(const double d[3], const double g[4], double *Mout, int ld)
{
    for (int p = 0; p < 3; p++)
        for (int q = 0; q < 3; q++) {
            double dd = d[p] * d[q], id = (p == q) - dd;
            double gs = g[0] * dd + g[1] * id, ga = g[2] * dd + g[3] * id;
            double B = 0.5 * (gs + ga), Cc = 0.5 * (gs - ga);
            Mout[p * ld + q] = B; Mout[(3 + p) * ld + 3 + q] = B;
            Mout[p * ld + 3 + q] = Cc; Mout[(3 + p) * ld + q] = Cc;
        }
}

}  // namespace ps
