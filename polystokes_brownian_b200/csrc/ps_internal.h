// ps_internal.h -- device-side data model and pair-tensor contractions of the
// B200 PolyStokes engine.  Internal header (not part of the C-ABI).
//
// Pair formulas restate src/mob.cpp of sgnagella/polystokes_brownian:
//   monomer-monomer (AA) translation block     mob.cpp:122-147
//   monomer-colloid (AB) rotation/stresslet     mob.cpp:362-537
//   colloid-colloid (BB) full FTS blocks        mob.cpp:96-358
//   self blocks                                 mob.cpp:65-86, 539-633
// and the block placement of the dense saddle matrix, mob.cpp:843-1144.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/polystokes_b200.h"

#define PS_MAX_NC11_SCHUR 64   // dense Schur path limit (slip_vel.cpp:97)
#define SL_KMAX 40             // Schur Lanczos noise: basis cap (slip_vel.cpp:300, kmax = 40)

// number of kernels this library has launched (host-side counter)
extern unsigned long long ps_launch_count;

// Programmatic dependent launch.  Every kernel of the library opens with
// pdl_enter(): griddepcontrol.wait returns once the grid it was launched behind
// has completed and its writes are visible (at once when it was launched without
// a programmatic dependency), and launch_dependents then lets the next kernel of
// the stream be scheduled into SM slots this grid frees.  So consecutive kernels
// keep full stream order for every load and store, and only the next grid's
// launch and block ramp overlap the tail of this one.  Every block passes the
// wait before anything else, early-exit blocks included, so a grid never
// completes before its predecessor.
#ifdef __CUDACC__
__device__ __forceinline__ void pdl_enter()
{
    asm volatile("griddepcontrol.wait;\n\tgriddepcontrol.launch_dependents;" ::: "memory");
}
#endif

#ifndef __CUDACC_RTC__
#include <cstdlib>
#include <utility>
// whether launches carry the programmatic-serialisation attribute (PS_PDL=0 turns it off)
inline bool ps_pdl_on()
{
    static const bool on = [] { const char *e = std::getenv("PS_PDL"); return !(e && e[0] == '0'); }();
    return on;
}

// launch a kernel of this library behind the previous work of the stream with
// programmatic dependent launch (the kernel must open with pdl_enter())
template <class... KArgs, class... Args>
inline void ps_launch(void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, Args &&...args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = ps_pdl_on() ? 1 : 0;
    ++::ps_launch_count;
    cudaLaunchKernelEx(&cfg, k, std::forward<Args>(args)...);
}
#endif

// Per-replica segment descriptor (device resident, one per replica).
struct Seg {
    int Nm, Nc, Np;
    int bead_off;      // first bead of this replica in the global bead arrays
    int coll_off;      // first colloid of this replica in global colloid arrays
    int vec_off;       // saddle-vector offset
    int top_off;       // offset in the concatenated mobility (nm3nc11) space
    int vel_off;       // offset in the concatenated velocity (nm3nc6) space
    int n, nm3, nc3, nc5, nc6, nc11, nm3nc3, nm3nc6, nm3nc11;
    int mm_HI, chain_HI, ab_mode, box_on, fene, mono_ev, lub_on, tether, aa_mode;
    int shell_schur;   // shell path with the dense Schur floor (nc11 <= lanczos_nc)
    int schur_off;     // offset into the per-replica nc11^2 buffers
    int sl_slot;       // shell path above the Schur limit: slot of its Schur Lanczos noise state, else -1
    int sl_off;        // offset of its Lanczos basis ((SL_KMAX + 1) nc11 doubles)
    int ba_off;        // offset (in 11-vectors) of this replica's BA partials
    int n_mtiles;      // monomer row tiles of this replica
    int bond_off, nbonds;
    int mt_first;      // index of this replica's first monomer tile (for BA partials)
    double beta, beta_inv, kT, dt, epsilon, kbond, r0, Lmax;
    double L[3];
    double hs_k;       // HS spring constant kpref/dt (or kpref/(dt beta))
    float sig[3], rverl[3], rcut[3];
    double lub_gap;
    int lub_bonded;    // lubricate bonded chain neighbours too
    int nper;          // monomers per chain
    int ss_off;        // offset of the inverse stresslet block (nc5^2 doubles), -1 if none
    int nch_aa, nch_bb; // column chunks of the far-field pair kernels (functions of Nm, Nc alone)
    // monomer-monomer scalars as x = c0/r + c1/r^3, y = c2/r + c3/r^3 (r > 2 beta)
    // and x = c4 + c5 r, y = c6 + c7 r (r <= 2 beta), for the selected aa_mode
    float aa_c[8];
};

// Column chunk widths of the far-field pair kernels.
constexpr int AA_CHUNK_COLS = 256;        // default; ps_autotune may pick another, process-wide
constexpr int BB_CHUNK_COLS = 64;        // colloid columns per chunk, for up to BB_MAX_CHUNKS chunks
constexpr int BB_MAX_CHUNKS = 64;

// Row tile of the far-field pair kernels.
struct Tile { int rep; int row0; int nrow; int mtile; };

// Search-grid cell budget per replica: CELL_CAP_PER_MONO * Nm + CELL_CAP_BASE cells
// (the longest axis is halved until the grid fits).  About one monomer per cell
// inside a compact cluster, so a 27-cell stencil visits a few tens of candidates.
constexpr long CELL_CAP_PER_MONO = 8, CELL_CAP_BASE = 64;

template <class T> struct V4;
template <> struct V4<double> { typedef double4 t; };
template <> struct V4<float> { typedef float4 t; };

template <class T> __device__ __forceinline__ T rsqrt_t(T v);
template <> __device__ __forceinline__ double rsqrt_t<double>(double v) { return rsqrt(v); }
template <> __device__ __forceinline__ float rsqrt_t<float>(float v) { return rsqrtf(v); }

// ---------------------------------------------------------------------------
// The reference's pair distance, dr = sqrt(dx*dx + dy*dy + dz*dz) in double with
// no fused multiply-add (check_dist.cpp:48-53), which decides the monomer pair
// branch dr > 2 beta (mob.cpp:123).  The reference's own monomer scalars jump
// at dr = 2 beta, and chain bonds often sit exactly there, so every kernel that
// takes that branch decides it with this distance.
__device__ __forceinline__ double ref_pair_dist(double dx, double dy, double dz)
{
    return __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
}

// ---------------------------------------------------------------------------
// AA: reference-specific monomer-monomer scalars (mob.cpp:122-131).
// mob_a = x ee + y (I - ee)   =>   mob_a u = y u + (x - y)(e.u) e
template <class T>
__device__ __forceinline__ void aa_scalars(T r, T rinv, T two_beta, T &x, T &y)
{
    if (r > two_beta) {
        T ri3 = rinv * rinv * rinv;
        x = T(0.375) * rinv - T(2.0) * ri3;
        y = T(0.75) * rinv - T(0.5) * ri3;
    } else {
        x = T(0.375) * r - T(1.0);
        y = T(1.0) - T(0.28125) * r;
    }
}

// Equal-sphere RPY of radius b = two_beta/2 in units 6 pi eta = 1, with the
// overlap form for r <= 2b (PS_AA_RPY).
template <class T>
__device__ __forceinline__ void aa_scalars_rpy(T r, T rinv, T two_beta, T &x, T &y)
{
    T b = T(0.5) * two_beta;
    if (r > two_beta) {
        T ri3 = rinv * rinv * rinv, b2 = b * b;
        x = T(1.5) * rinv - b2 * ri3;
        y = T(0.75) * rinv + T(0.5) * b2 * ri3;
    } else {
        T bi = T(1) / b;
        x = (T(1) - T(0.1875) * r * bi) * bi;
        y = (T(1) - T(0.28125) * r * bi) * bi;
    }
}

// ---------------------------------------------------------------------------
// Flattening of a symmetric-index rank-3 tensor g[k][i][j] to the 3x5 form of
// mob.cpp:221-227: [g00-g22, 2 g01, 2 g02, 2 g12, g11-g22].
// gt[k][i][j] = -xg (e_i e_j - d_ij/3) e_k + yg (e_i d_jk + e_j d_ik - 2 e_i e_j e_k)
template <class T>
__device__ __forceinline__ void gt_flat(const T e[3], T xg, T yg, T G[15])
{
#pragma unroll
    for (int k = 0; k < 3; k++) {
        T ek = e[k];
        // g[k][i][j] for the six (i,j) pairs that the flattening uses
        auto g = [&](int i, int j) -> T {
            T dij = (i == j) ? T(1) : T(0);
            T djk = (j == k) ? T(1) : T(0);
            T dik = (i == k) ? T(1) : T(0);
            return -xg * (e[i] * e[j] - dij * T(1.0 / 3.0)) * ek
                   + yg * (e[i] * djk + e[j] * dik - T(2) * e[i] * e[j] * ek);
        };
        T g22 = g(2, 2);
        G[k * 5 + 0] = g(0, 0) - g22;
        G[k * 5 + 1] = T(2) * g(0, 1);
        G[k * 5 + 2] = T(2) * g(0, 2);
        G[k * 5 + 3] = T(2) * g(1, 2);
        G[k * 5 + 4] = g(1, 1) - g22;
    }
}

// ht[k][i][j] = yh (e_i w_jk + e_j w_ik), w_ab = eps_abl e_l (mob.cpp:258-276)
template <class T>
__device__ __forceinline__ void ht_flat(const T e[3], T yh, T H[15])
{
    // w = eps . e (antisymmetric)
    T w[3][3];
    w[0][0] = 0; w[1][1] = 0; w[2][2] = 0;
    w[0][1] = e[2]; w[1][0] = -e[2];
    w[0][2] = -e[1]; w[2][0] = e[1];
    w[1][2] = e[0]; w[2][1] = -e[0];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        auto h = [&](int i, int j) -> T { return yh * (e[i] * w[j][k] + e[j] * w[i][k]); };
        T h22 = h(2, 2);
        H[k * 5 + 0] = h(0, 0) - h22;
        H[k * 5 + 1] = T(2) * h(0, 1);
        H[k * 5 + 2] = T(2) * h(0, 2);
        H[k * 5 + 3] = T(2) * h(1, 2);
        H[k * 5 + 4] = h(1, 1) - h22;
    }
}

// stress-strain rank-4 tensor entry (mob.cpp:279-298)
template <class T>
__device__ __forceinline__ T m4(const T e[3], int i, int j, int k, int l, T xm, T ym, T zm)
{
    auto d = [](int a, int b) -> T { return a == b ? T(1) : T(0); };
    T eij = e[i] * e[j], ekl = e[k] * e[l], eik = e[i] * e[k], ejk = e[j] * e[k];
    T eil = e[i] * e[l], ejl = e[j] * e[l];
    return T(1.5) * xm * (eij - T(1.0 / 3.0) * d(i, j)) * (ekl - T(1.0 / 3.0) * d(k, l))
           + T(0.5) * ym * (eik * d(j, l) + ejk * d(i, l) + eil * d(j, k) + ejl * d(i, k) - T(4) * eij * ekl)
           + T(0.5) * zm * (d(i, k) * d(j, l) + d(j, k) * d(i, l) - d(i, j) * d(k, l) + eij * d(k, l)
                            + ekl * d(i, j) - eik * d(j, l) - ejk * d(i, l) - eil * d(j, k) - ejl * d(i, k)
                            + eij * ekl);
}

// 5x5 flattening through mesid (init.cpp:340-354, mob.cpp:321-355)
template <class T>
__device__ __forceinline__ void mm_flat(const T e[3], T xm, T ym, T zm, T Mm[25])
{
    const int mes0[5] = {0, 0, 0, 1, 1}, mes1[5] = {2, 1, 2, 2, 2};
#pragma unroll
    for (int ii = 0; ii < 5; ii++) {
        int a = mes0[ii], b = mes1[ii];
        if (ii == 0 || ii == 4) {
            Mm[ii * 5 + 0] = m4(e, a, a, 0, 0, xm, ym, zm) - m4(e, a, a, 2, 2, xm, ym, zm)
                             - (m4(e, b, b, 0, 0, xm, ym, zm) - m4(e, b, b, 2, 2, xm, ym, zm));
            Mm[ii * 5 + 1] = T(2) * (m4(e, a, a, 0, 1, xm, ym, zm) - m4(e, b, b, 0, 1, xm, ym, zm));
            Mm[ii * 5 + 2] = T(2) * (m4(e, a, a, 0, 2, xm, ym, zm) - m4(e, b, b, 0, 2, xm, ym, zm));
            Mm[ii * 5 + 3] = T(2) * (m4(e, a, a, 1, 2, xm, ym, zm) - m4(e, b, b, 1, 2, xm, ym, zm));
            Mm[ii * 5 + 4] = m4(e, a, a, 1, 1, xm, ym, zm) - m4(e, a, a, 2, 2, xm, ym, zm)
                             - (m4(e, b, b, 1, 1, xm, ym, zm) - m4(e, b, b, 2, 2, xm, ym, zm));
        } else {
            Mm[ii * 5 + 0] = T(2) * (m4(e, a, b, 0, 0, xm, ym, zm) - m4(e, a, b, 2, 2, xm, ym, zm));
            Mm[ii * 5 + 1] = T(4) * m4(e, a, b, 0, 1, xm, ym, zm);
            Mm[ii * 5 + 2] = T(4) * m4(e, a, b, 0, 2, xm, ym, zm);
            Mm[ii * 5 + 3] = T(4) * m4(e, a, b, 1, 2, xm, ym, zm);
            Mm[ii * 5 + 4] = T(2) * (m4(e, a, b, 1, 1, xm, ym, zm) - m4(e, a, b, 2, 2, xm, ym, zm));
        }
    }
}

// ---------------------------------------------------------------------------
// BB: contribution to colloid `row` from colloid `col`, e = (x_lo - x_hi)/r of
// the canonically ordered pair (lo = lower colloid index); `is_lo` = row is lo.
//   lo row: U += A F - B T + G S ; W += B F + C T + H S ; E += -G^T F + H^T T + Mm S
//   hi row: U += A F - B T - G S ; W += B F + C T + H S ; E +=  G^T F + H^T T + Mm^T S
// (derived from the dense block placement, mob.cpp:1042-1143)
//
// The blocks are applied in contracted form, never built.  With the stresslet
// 5-vector S expanded to the symmetric traceless matrix S^ (S^00 = S0,
// S^11 = S4, S^22 = -S0 - S4, S^01 = S1, S^02 = S2, S^12 = S3), v = S^ e,
// s = e.v, c = T x e and flat(Z) = [Z00 - Z22, 2 Z01, 2 Z02, 2 Z12, Z11 - Z22]
// (the flattening of mob.cpp:221-227, under which isotropic parts vanish):
//   G S   = 2 yg v - (xg + 2 yg) s e          H S   = 2 yh e x v
//   G^T F = flat(yg (e F^T + F e^T) - (xg + 2 yg)(e.F) e e^T)
//   H^T T = flat(yh (e c^T + c e^T))
//   Mm S  = flat((1.5 xm - 2 ym + 0.5 zm) s e e^T + (ym - zm)(e v^T + v e^T) + zm S^)
// Mm is symmetric, so both rows use Mm S.  About 230 FLOP per directed pair
// (FMA counted as 2), against 242 for the 11 x 11 block-vector product alone
// when the block is built first.
template <class T>
__device__ __forceinline__ void bb_apply(const T e[3], T r, T rinv, bool is_lo, const T in[11], T out[11])
{
    (void)r;
    const T ri2 = rinv * rinv, ri3 = ri2 * rinv, ri4 = ri2 * ri2, ri5 = ri4 * rinv;
    const T xa = T(1.5) * rinv - ri3, ya = T(0.75) * rinv + T(0.5) * ri3;
    const T yb = T(-0.75) * ri2;
    const T xg = T(2.25) * ri2 - T(3.6) * ri4, yg = T(1.2) * ri4;
    const T xc = T(0.75) * ri3, yc = T(-0.375) * ri3;
    const T yh = T(-1.125) * ri3;
    const T xm = T(-4.5) * ri3 + T(10.8) * ri5, ym = T(2.25) * ri3 - T(7.2) * ri5, zm = T(1.8) * ri5;
    const T sg = is_lo ? T(1) : T(-1);
    const T F0 = in[0], F1 = in[1], F2 = in[2], T0 = in[3], T1 = in[4], T2 = in[5];
    const T S0 = in[6], S1 = in[7], S2 = in[8], S3 = in[9], S4 = in[10], S22 = -S0 - S4;
    const T e0 = e[0], e1 = e[1], e2 = e[2];
    const T v0 = S0 * e0 + S1 * e1 + S2 * e2;
    const T v1 = S1 * e0 + S4 * e1 + S3 * e2;
    const T v2 = S2 * e0 + S3 * e1 + S22 * e2;
    const T s = e0 * v0 + e1 * v1 + e2 * v2;
    const T eF = e0 * F0 + e1 * F1 + e2 * F2;
    const T eT = e0 * T0 + e1 * T1 + e2 * T2;
    const T c0 = T1 * e2 - T2 * e1, c1 = T2 * e0 - T0 * e2, c2 = T0 * e1 - T1 * e0;   // T x e
    const T kg = xg + T(2) * yg;
    // U row: A F - B T +- G S, with B v = yb (v x e)
    const T cu = (xa - ya) * eF - sg * kg * s, g2 = sg * T(2) * yg;
    out[0] += ya * F0 - yb * c0 + g2 * v0 + cu * e0;
    out[1] += ya * F1 - yb * c1 + g2 * v1 + cu * e1;
    out[2] += ya * F2 - yb * c2 + g2 * v2 + cu * e2;
    // W row: B F + C T + H S; C as the reference writes it: diagonal x ee + y (1 - ee),
    // off-diagonal (x + y) ee (mob.cpp:249-254)
    const T cw = (xc + yc) * eT, h2 = T(2) * yh;
    out[3] += yb * (F1 * e2 - F2 * e1) + cw * e0 + yc * T0 - T(2) * yc * e0 * e0 * T0 + h2 * (e1 * v2 - e2 * v1);
    out[4] += yb * (F2 * e0 - F0 * e2) + cw * e1 + yc * T1 - T(2) * yc * e1 * e1 * T1 + h2 * (e2 * v0 - e0 * v2);
    out[5] += yb * (F0 * e1 - F1 * e0) + cw * e2 + yc * T2 - T(2) * yc * e2 * e2 * T2 + h2 * (e0 * v1 - e1 * v0);
    // E row: flat(Z), Z = gam e e^T + e w^T + w e^T + zm S^
    const T gam = (T(1.5) * xm - T(2) * ym + T(0.5) * zm) * s + sg * kg * eF;
    const T ymz = ym - zm, sy = sg * yg;
    const T w0 = yh * c0 + ymz * v0 - sy * F0;
    const T w1 = yh * c1 + ymz * v1 - sy * F1;
    const T w2 = yh * c2 + ymz * v2 - sy * F2;
    const T z22 = gam * e2 * e2 + T(2) * e2 * w2 + zm * S22;
    out[6] += gam * e0 * e0 + T(2) * e0 * w0 + zm * S0 - z22;
    out[7] += T(2) * (gam * e0 * e1 + e0 * w1 + e1 * w0 + zm * S1);
    out[8] += T(2) * (gam * e0 * e2 + e0 * w2 + e2 * w0 + zm * S2);
    out[9] += T(2) * (gam * e1 * e2 + e1 * w2 + e2 * w1 + zm * S3);
    out[10] += gam * e1 * e1 + T(2) * e1 * w1 + zm * S4 - z22;
}

// Monomer-colloid translation scalars (x along e, y across) and, for the
// regularised mode, the rotation-translation scalar yb.  Colloid radius 1,
// monomer radius beta < 1, units 6 pi eta = 1.
//   r >= 1 + beta (far):   x = 3/(2r) - (1+b^2)/(2r^3), y = 3/(4r) + (1+b^2)/(4r^3)
//   1 - beta < r < 1 + beta (overlap, Zuk et al. eq. 3.1/3.3 middle):
//     t = (1-b)^2 + 3r^2, u = (1-b)^2 - r^2, I = (16 r^3 (1+b) - t^2)/(32 r^3)
//     y = I/b, x = (I + 3u^2/(32 r^3))/b,
//     yb = -(3/(8b)) (1-b+r)^2 (b^2 + 2b(1+r) - 3(1-r)^2)/(8 r^2)
//   r <= 1 - beta (monomer inside the colloid): x = y = 1, yb = -3r/4
template <class T>
__device__ __host__ __forceinline__ void ab_trans_scalars(T r, T rinv, T beta, bool reg, T &x, T &y, T &yb)
{
    const T b2 = beta * beta;
    if (!reg || r >= T(1) + beta) {
        T ri3 = rinv * rinv * rinv;
        x = T(1.5) * rinv - T(0.5) * (T(1) + b2) * ri3;
        y = T(0.75) * rinv + T(0.25) * (T(1) + b2) * ri3;
        return;
    }
    if (r > T(1) - beta) {
        T rd = T(1) - beta, r2 = r * r, r3 = r2 * r;
        T t = rd * rd + T(3) * r2, u = rd * rd - r2;
        T I = (T(16) * r3 * (T(1) + beta) - t * t) / (T(32) * r3);
        y = I / beta;
        x = (I + T(3) * u * u / (T(32) * r3)) / beta;
        T poly = (rd + r) * (rd + r) * (b2 + T(2) * beta * (T(1) + r) - T(3) * (T(1) - r) * (T(1) - r)) / (T(8) * r2);
        yb = -(T(3) / (T(8) * beta)) * poly;
    } else {
        x = T(1);
        y = T(1);
        yb = T(-0.75) * r;
    }
}

// AB scalars (mob.cpp:410-412, 465-466)
template <class T>
__device__ __forceinline__ void ab_scalars(T rinv, T beta2, T &yb, T &xg, T &yg)
{
    T ri2 = rinv * rinv, ri4 = ri2 * ri2;
    yb = T(-0.75) * ri2;
    xg = T(2.25) * ri2 - T(0.45) * ri4 * (T(3) + T(5) * beta2);
    yg = T(0.9) * ri4 * (T(0.5) + T(5.0 / 6.0) * beta2);
}
