// stage.cu -- per-stage kernels of the PolyStokes step on the device:
// position packing, pair geometry / Verlet and cell lists, forces (RHS),
// mob() bookkeeping, the arrowhead Schur eigenvalue floor, the Jacobi diagonal,
// Brownian noise, and the predictor-corrector update.
//
// This translation unit is compiled with --fmad=false so that distances, forces
// and position updates round exactly like the reference's plain C++ (no FMA
// contraction): pair-list membership is then bit-identical to the reference's
// `dr < rverl` tests.
//
// Reference files restated (sgnagella/polystokes_brownian):
//   check_dist.cpp:12-87, cell_list.cpp:23-172, rhs.cpp:46-346,
//   pair_interaction.{h,cpp}, mob.cpp:635-1213 (bookkeeping), slip_vel.cpp:19-349,
//   drift.cpp:9-62, traj.cpp:9-94, quat.cpp:7-54, box.cpp:40-84, run.cpp:70-162.
#include <cmath>
#include <cstdio>
#include <vector>
#include <algorithm>
#include <curand_kernel.h>
#include "ps_internal.h"
#include "ps_kernels.h"

namespace ps {

__device__ __forceinline__ void min_image(const Seg &s, double &dx, double &dy, double &dz)
{
    if (!s.box_on) return;
    dx -= s.L[0] * nearbyint(dx * (1.0 / s.L[0]));
    dy -= s.L[1] * nearbyint(dy * (1.0 / s.L[1]));
    dz -= s.L[2] * nearbyint(dz * (1.0 / s.L[2]));
}

// bead -> replica lookup (bead offsets, R+1 entries)
__device__ __forceinline__ int rep_of(const int *__restrict__ offs, int R, long k)
{
    int lo = 0, hi = R;
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (offs[mid] <= k) lo = mid; else hi = mid;
    }
    return lo;
}

// ---------------------------------------------------------------------------
// packing: x (AoS doubles) -> (x,y,z,chain) in FP64 and FP32
__global__ void k_pack(long ntot, const double *__restrict__ x, const double *__restrict__ chain,
                       double4 *__restrict__ p64, float4 *__restrict__ p32, float4 *__restrict__ p32lo)
{
    pdl_enter();
    long b = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= ntot) return;
    double cx = x[3 * b], cy = x[3 * b + 1], cz = x[3 * b + 2], ch = chain[b];
    p64[b] = make_double4(cx, cy, cz, ch);
    float hx = (float)cx, hy = (float)cy, hz = (float)cz;
    p32[b] = make_float4(hx, hy, hz, (float)ch);
    p32lo[b] = make_float4((float)(cx - (double)hx), (float)(cy - (double)hy), (float)(cz - (double)hz), 0.f);
}

// Exact radius of the FP32 monomer kernel, one block per replica: with X the
// largest monomer coordinate magnitude of the replica, hi-only separations carry
// an error of at most 2^-23 X, so beyond r = X / 16 their relative error stays
// below 2^-19; inside max(2.1 beta, X / 16) the kernel adds the low parts.  The
// radius covers the overlap form (r <= 2 beta).  Stored squared, as a float.
// A max over the replica's own beads: independent of the other replicas.
__global__ void k_aa_radius(const Seg *__restrict__ segs, const double *__restrict__ x, float *__restrict__ te2)
{
    pdl_enter();
    const Seg &s = segs[blockIdx.x];
    __shared__ double red[256];
    double m = 0.0;
    for (long i = threadIdx.x; i < 3L * s.Nm; i += blockDim.x) m = fmax(m, fabs(x[3L * s.bead_off + i]));
    red[threadIdx.x] = m;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double t = fmax(2.1 * s.beta, red[0] * (1.0 / 16.0));
        te2[blockIdx.x] = isfinite(t) ? (float)fmin(t * t, 3.0e38) : 3.0e38f;
    }
}

int stage_pack(Engine &E, cudaStream_t st)
{
    int thr = 256;
    E.ps_setup_valid = false;     // positions change: the pair-space blocks are stale
    ps_launch(k_pack, (unsigned)((E.ntot + thr - 1) / thr), thr, 0, st, E.ntot, E.d_x, E.d_chain, E.d_pos64, E.d_pos32, E.d_pos32lo);
    if (E.n_aa_tiles)
        ps_launch(k_aa_radius, E.R, 256, 0, st, E.d_segs, E.d_x, E.d_aa_te2);
    PS_CK(cudaGetLastError());
    return PS_OK;
}

// clamp in double before converting: NaN and out-of-range values map into [0, nc)
__device__ __forceinline__ int cell_coord(double v, double org, double size, int nc)
{
    double f = floor((v - org) / size);
    if (!(f >= 0.0)) return 0;
    if (f >= (double)nc) return nc - 1;
    return (int)f;
}

// ---------------------------------------------------------------------------
// monomer cell list (search structure only: its pair sets equal the
// reference's because membership is decided by the same `dr < cutoff` test).
// Geometry per replica: bounding box of the monomers (or the periodic box),
// cells of edge >= rc (rc = rverl[0] = 0.05 + 2 beta, cell_list.cpp:26), with
// the cell count capped at CELL_CAP_PER_MONO Nm + CELL_CAP_BASE by halving the longest axis.
// cellgeo per replica: org[3], size[3], nc[3], periodic  (10 doubles)
__global__ void k_cell_geo(const Seg *__restrict__ segs, const double *__restrict__ x, double *__restrict__ geo,
                           const long *__restrict__ cell_off)
{
    pdl_enter();
    // geo per replica (20 doubles): [0,10) the search grid, [10,20) the
    // reference's own grid of build_monomer_cell_list (cell_list.cpp:23-62),
    // each as org[3], size[3], nc[3], periodic.
    const Seg &s = segs[blockIdx.x];
    __shared__ double lo[3][256], hi[3][256];
    double l[3] = {1e300, 1e300, 1e300}, h[3] = {-1e300, -1e300, -1e300};
    for (int i = threadIdx.x; i < s.Nm; i += blockDim.x)
        for (int d = 0; d < 3; d++) {
            double v = x[3 * ((long)s.bead_off + i) + d];
            l[d] = fmin(l[d], v); h[d] = fmax(h[d], v);
        }
    for (int d = 0; d < 3; d++) { lo[d][threadIdx.x] = l[d]; hi[d][threadIdx.x] = h[d]; }
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o)
            for (int d = 0; d < 3; d++) {
                lo[d][threadIdx.x] = fmin(lo[d][threadIdx.x], lo[d][threadIdx.x + o]);
                hi[d][threadIdx.x] = fmax(hi[d][threadIdx.x], hi[d][threadIdx.x + o]);
            }
        __syncthreads();
    }
    if (threadIdx.x != 0) return;
    double *g = geo + 20 * blockIdx.x;
    for (int pass = 0; pass < 2; pass++) {
        // pass 0: search grid, edge >= every monomer-pair cutoff, capped cell count
        // pass 1: reference grid, edge rverl[0], uncapped
        double rc = (double)s.rverl[0];
        if (pass == 0) {
            rc = fmax(rc, (double)s.rcut[0]);
            if (s.lub_on) rc = fmax(rc, (2.0 + s.lub_gap) * s.beta);
        }
        // cell counts are computed in double and clamped to [1, 2^20] before any
        // integer conversion, so non-finite or huge coordinates cannot overflow
        double cap = pass == 0 ? (double)CELL_CAP_PER_MONO * s.Nm + (double)CELL_CAP_BASE : 1e18;
        int nc[3];
        double org[3], size[3], ext[3];
        int periodic = 0;
        auto count = [&](double len) {
            double n = floor(len / rc);
            if (!(n >= 1.0)) n = 1.0;
            if (n > 1048576.0) n = 1048576.0;
            return (int)n;
        };
        if (s.box_on) {
            for (int d = 0; d < 3; d++) { nc[d] = count(s.L[d]); ext[d] = s.L[d]; org[d] = -0.5 * s.L[d]; }
            periodic = (nc[0] >= 3 && nc[1] >= 3 && nc[2] >= 3);
        } else {
            for (int d = 0; d < 3; d++) {
                double a = s.Nm ? lo[d][0] : 0.0, b = s.Nm ? hi[d][0] : 0.0;
                if (!isfinite(a) || !isfinite(b)) { a = 0.0; b = 0.0; }
                ext[d] = b - a; org[d] = a;
                nc[d] = count(ext[d]);
            }
        }
        while ((double)nc[0] * (double)nc[1] * (double)nc[2] > cap) {
            int m = 0;
            for (int d = 1; d < 3; d++) if (nc[d] > nc[m]) m = d;
            nc[m] = (nc[m] + 1) / 2;
            if (nc[m] < 3) periodic = 0;
        }
        if (s.box_on && !periodic) for (int d = 0; d < 3; d++) nc[d] = 1;
        for (int d = 0; d < 3; d++) {
            if (s.box_on) size[d] = s.L[d] / nc[d];
            else size[d] = ext[d] > 0.0 ? ext[d] / nc[d] : rc;
            if (!(size[d] > 0.0) || !isfinite(size[d])) size[d] = rc;
        }
        if (s.box_on && !periodic)
            for (int d = 0; d < 3; d++) size[d] = s.L[d] > 0.0 ? s.L[d] : 1.0;
        double *gg = g + 10 * pass;
        for (int d = 0; d < 3; d++) { gg[d] = org[d]; gg[3 + d] = size[d]; gg[6 + d] = nc[d]; }
        gg[9] = periodic;
    }
    (void)cell_off;
}

// the reference's grid considers (i, j) only when their cells are adjacent
// (cell_list.cpp:109-113,436-453): |dc| <= 1 per axis, modulo nc when periodic
__device__ __forceinline__ bool ref_cells_adjacent(const double *__restrict__ gref, const double *__restrict__ x,
                                                   long i, long j)
{
    for (int d = 0; d < 3; d++) {
        int nc = (int)gref[6 + d];
        int ci = cell_coord(x[3 * i + d], gref[d], gref[3 + d], nc);
        int cj = cell_coord(x[3 * j + d], gref[d], gref[3 + d], nc);
        int dc = ci - cj;
        if (gref[9] != 0.0) {
            dc = ((dc % nc) + nc) % nc;
            if (dc > 1 && dc < nc - 1) return false;
        } else if (dc > 1 || dc < -1) return false;
    }
    return true;
}


__global__ void k_cell_assign(long ntot, const int *__restrict__ bead_offs, int R, const Seg *__restrict__ segs,
                              const double *__restrict__ x, const double *__restrict__ geo,
                              const long *__restrict__ cell_off, int *__restrict__ cell, int *__restrict__ count)
{
    pdl_enter();
    long b = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= ntot) return;
    int r = rep_of(bead_offs, R, b);
    const Seg &s = segs[r];
    int i = (int)(b - s.bead_off);
    if (i >= s.Nm) { cell[b] = -1; return; }
    const double *g = geo + 20 * r;
    int nc0 = (int)g[6], nc1 = (int)g[7], nc2 = (int)g[8];
    int c0 = cell_coord(x[3 * b], g[0], g[3], nc0);
    int c1 = cell_coord(x[3 * b + 1], g[1], g[4], nc1);
    int c2 = cell_coord(x[3 * b + 2], g[2], g[5], nc2);
    long c = cell_off[r] + c0 + (long)nc0 * (c1 + (long)nc1 * c2);
    cell[b] = (int)c;
    atomicAdd(&count[c], 1);
}

// exclusive scan over all cells (single block, sequential chunks; cell counts are small)
// deterministic fill: each cell's members in ascending bead order
__global__ void k_cell_fill(long ntot, const int *__restrict__ cell, const int *__restrict__ start,
                            int *__restrict__ fillc, int *__restrict__ sorted)
{
    pdl_enter();
    long b = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= ntot) return;
    int c = cell[b];
    if (c < 0) return;
    int slot = atomicAdd(&fillc[c], 1);
    sorted[start[c] + slot] = (int)b;
}
// Each cell's members in ascending bead order (the fill above places them by atomic slots).
// Cells of up to 64 members are sorted in place by one thread; larger cells (piled or
// collapsed beads) are listed for k_cell_sort_big, which ranks their members in parallel.
constexpr int CELL_SORT_SERIAL = 64;

__global__ void k_cell_sort(long ncells, const int *__restrict__ start, int *__restrict__ sorted,
                            int *__restrict__ big, int *__restrict__ nbig)
{
    pdl_enter();
    long c = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncells) return;
    int a = start[c], e = start[c + 1];
    if (e - a > CELL_SORT_SERIAL) {
        big[atomicAdd(nbig, 1)] = (int)c;
        return;
    }
    for (int i = a + 1; i < e; i++) {
        int v = sorted[i], j = i - 1;
        while (j >= a && sorted[j] > v) { sorted[j + 1] = sorted[j]; j--; }
        sorted[j + 1] = v;
    }
}

// one block per listed cell at a time: every member's rank is the number of smaller members
// (bead indices are distinct), written to tmp and copied back
__global__ void k_cell_sort_big(const int *__restrict__ start, int *__restrict__ sorted, const int *__restrict__ big,
                                const int *__restrict__ nbig, int *__restrict__ tmp)
{
    pdl_enter();
    const int n = *nbig;
    for (int q = blockIdx.x; q < n; q += gridDim.x) {
        const int c = big[q], a = start[c], k = start[c + 1] - a;
        for (int i = threadIdx.x; i < k; i += blockDim.x) {
            const int v = sorted[a + i];
            int rank = 0;
            for (int j = 0; j < k; j++) rank += sorted[a + j] < v;
            tmp[a + rank] = v;
        }
        __syncthreads();
        for (int i = threadIdx.x; i < k; i += blockDim.x) sorted[a + i] = tmp[a + i];
        __syncthreads();
    }
}

int stage_cells(Engine &E, cudaStream_t st, const long *d_cell_off, long ncells)
{
    ps_launch(k_cell_geo, E.R, 256, 0, st, E.d_segs, E.d_x, E.d_cellgeo, d_cell_off);
    PS_CK(cudaMemsetAsync(E.d_cell_count, 0, sizeof(int) * (ncells + 1), st));
    int thr = 256;
    unsigned nb = (unsigned)((E.ntot + thr - 1) / thr);
    ps_launch(k_cell_assign, nb, thr, 0, st, E.ntot, E.d_bead_offs, E.R, E.d_segs, E.d_x, E.d_cellgeo, d_cell_off, E.d_cell,
            E.d_cell_count);
    int rc = exclusive_scan(E, E.d_cell_count, E.d_cell_start, ncells, st);
    if (rc) return rc;
    PS_CK(cudaMemsetAsync(E.d_cell_count, 0, sizeof(int) * (ncells + 1), st));
    ps_launch(k_cell_fill, nb, thr, 0, st, E.ntot, E.d_cell, E.d_cell_start, E.d_cell_count, E.d_cell_sorted);
    PS_CK(cudaMemsetAsync(E.d_cell_nbig, 0, sizeof(int), st));
    ps_launch(k_cell_sort, (unsigned)((ncells + thr - 1) / thr), thr, 0, st, ncells, E.d_cell_start, E.d_cell_sorted,
            E.d_cell_big, E.d_cell_nbig);
    ps_launch(k_cell_sort_big, 148, 256, 0, st, E.d_cell_start, E.d_cell_sorted, E.d_cell_big, E.d_cell_nbig,
            E.d_cell_tmp);
    PS_CK(cudaGetLastError());
    return PS_OK;
}

// Visit monomer neighbours j of monomer bead b (global indices) within the
// 27-cell stencil; f(j) is called for every other monomer found.
template <class F>
__device__ __forceinline__ void for_cell_neighbours(const Seg &s, int r, long b, const double *__restrict__ x,
                                                    const double *__restrict__ geo, const long *__restrict__ cell_off,
                                                    const int *__restrict__ start, const int *__restrict__ sorted, F f)
{
    const double *g = geo + 20 * r;
    int nc[3] = {(int)g[6], (int)g[7], (int)g[8]};
    int periodic = (int)g[9];
    int c[3];
    for (int d = 0; d < 3; d++) c[d] = cell_coord(x[3 * b + d], g[d], g[3 + d], nc[d]);
    int lo[3], hi[3];
    for (int d = 0; d < 3; d++) {
        if (periodic) { lo[d] = -1; hi[d] = 1; }
        else { lo[d] = c[d] > 0 ? -1 : 0; hi[d] = c[d] < nc[d] - 1 ? 1 : 0; }
    }
    for (int dz = lo[2]; dz <= hi[2]; dz++)
        for (int dy = lo[1]; dy <= hi[1]; dy++)
            for (int dx = lo[0]; dx <= hi[0]; dx++) {
                int q[3] = {c[0] + dx, c[1] + dy, c[2] + dz};
                if (periodic)
                    for (int d = 0; d < 3; d++) q[d] = (q[d] % nc[d] + nc[d]) % nc[d];
                long cc = cell_off[r] + q[0] + (long)nc[0] * (q[1] + (long)nc[1] * q[2]);
                for (int k = start[cc]; k < start[cc + 1]; k++) {
                    int j = sorted[k];
                    if (j != b) f(j);
                }
            }
}

// ---------------------------------------------------------------------------
// forces (rhs.cpp:160-260): fint is the negative of the physical force.
// One thread per bead gathers every contribution acting on it.
__device__ __forceinline__ double hs_mag(double dr, double sig, double k)
{
    double se = sig * (1.0 + 0.01);
    if (dr >= se) return 0.0;
    return k * (se - dr);
}
__device__ __forceinline__ double wca_mag(double dr, double ri, double sig, double rcut, double eps)
{
    if (dr >= rcut) return 0.0;
    double s1 = sig * ri, s2 = s1 * s1, s6 = s2 * s2 * s2, s12 = s6 * s6;
    return 24.0 * eps * ri * (2.0 * s12 - s6);
}

// pair (lo, hi) geometry as check_dist.cpp:49-71; returns dr; e = d/dr
__device__ __forceinline__ double pair_geom(const Seg &s, const double *__restrict__ x, long lo, long hi, double e[3])
{
    double dx = x[3 * lo] - x[3 * hi], dy = x[3 * lo + 1] - x[3 * hi + 1], dz = x[3 * lo + 2] - x[3 * hi + 2];
    min_image(s, dx, dy, dz);
    double dr = sqrt(dx * dx + dy * dy + dz * dz);
    double ri = 1 / dr;
    e[0] = dx * ri; e[1] = dy * ri; e[2] = dz * ri;
    return dr;
}

// Colloid-monomer HS sum of one colloid, one warp per colloid: lanes test 32
// monomers at a time and lane 0 adds the hits in ascending monomer order, the
// order (and the arithmetic) of a serial sweep over the replica's monomers.
// Out: chs[3 c] = sum over monomers m of the colloid's hs_pair(m) term.
__global__ void k_colloid_hs(long ncoll, const int *__restrict__ coll_rep, const Seg *__restrict__ segs,
                             const double *__restrict__ x, double *__restrict__ chs)
{
    pdl_enter();
    const long g = blockIdx.x;
    if (g >= ncoll) return;
    const int lane = threadIdx.x;
    const Seg &s = segs[coll_rep[g]];
    const long b = (long)s.bead_off + s.Nm + (g - s.coll_off);
    const double k = s.hs_k, rv = (double)s.rverl[1], sig = (double)s.sig[1];
    double f0 = 0.0, f1 = 0.0, f2 = 0.0;
    for (int m0 = 0; m0 < s.Nm; m0 += 32) {
        const int m = m0 + lane;
        double c0 = 0.0, c1 = 0.0, c2 = 0.0;
        bool hit = false;
        if (m < s.Nm) {
            // pair (lo = monomer, hi = colloid); the colloid is the pair's second bead: sign +1
            double e[3];
            const double dr = pair_geom(s, x, (long)s.bead_off + m, b, e);
            if (dr < rv) {
                const double fm = hs_mag(dr, sig, k);
                if (fm != 0.0) { hit = true; c0 = fm * e[0]; c1 = fm * e[1]; c2 = fm * e[2]; }
            }
        }
        unsigned mask = __ballot_sync(0xffffffffu, hit);
        while (mask) {
            const int src = __ffs(mask) - 1;
            mask &= mask - 1;
            const double a0 = __shfl_sync(0xffffffffu, c0, src), a1 = __shfl_sync(0xffffffffu, c1, src),
                         a2 = __shfl_sync(0xffffffffu, c2, src);
            f0 += 1.0 * a0; f1 += 1.0 * a1; f2 += 1.0 * a2;
        }
    }
    if (lane == 0) { chs[3 * g] = f0; chs[3 * g + 1] = f1; chs[3 * g + 2] = f2; }
}

__global__ void k_forces(long ntot, const int *__restrict__ bead_offs, int R, const Seg *__restrict__ segs,
                         const double *__restrict__ x, const double *__restrict__ xpos0,
                         const double *__restrict__ geo, const long *__restrict__ cell_off,
                         const int *__restrict__ cstart, const int *__restrict__ csorted,
                         const int *__restrict__ bptr, const int *__restrict__ bnbr, const double *__restrict__ bsgn,
                         const double *__restrict__ time, double *__restrict__ ktrap, const double *__restrict__ trapinfo,
                         const double *__restrict__ chs, double *__restrict__ rhs)
{
    pdl_enter();
    long b = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= ntot) return;
    int r = rep_of(bead_offs, R, b);
    const Seg &s = segs[r];
    const int i = (int)(b - s.bead_off);
    const bool mono = i < s.Nm;
    double f[3] = {0.0, 0.0, 0.0};
    const double k = s.hs_k;
    // HS repulsion over Verlet pairs (pair_interaction_hs, pair_interaction.cpp:160-227),
    // partners in ascending index order (the order the reference's vlist sweep adds them)
    auto hs_pair = [&](long j, int type) {
        long lo = b < j ? b : j, hi = b < j ? j : b;
        double e[3];
        double dr = pair_geom(s, x, lo, hi, e);
        if (!(dr < (double)s.rverl[type])) return;
        double fm = hs_mag(dr, (double)s.sig[type], k);
        if (fm == 0.0) return;
        double sg = (b == lo) ? -1.0 : 1.0;
        f[0] += sg * (fm * e[0]); f[1] += sg * (fm * e[1]); f[2] += sg * (fm * e[2]);
    };
    if (mono) {
        if (s.mm_HI && s.mono_ev) {
            // AA Verlet partners via the cell list, applied in ascending order.  Up to 64 are
            // gathered and sorted in registers; a bead with more (overlapping, diverging
            // configurations) takes them by repeated ascending selection over its cells, so no
            // partner is ever dropped and the order stays the reference's.
            const double rv = (double)s.rverl[0];
            auto is_partner = [&](int j) {
                double dx = x[3 * b] - x[3 * (long)j], dy = x[3 * b + 1] - x[3 * (long)j + 1], dz = x[3 * b + 2] - x[3 * (long)j + 2];
                min_image(s, dx, dy, dz);
                double d2 = dx * dx + dy * dy + dz * dz;
                return d2 < rv * rv * 1.0000001;
            };
            int cnt = 0, tot = 0;
            int nb[64];
            for_cell_neighbours(s, r, b, x, geo, cell_off, cstart, csorted, [&](int j) {
                if (!is_partner(j)) return;
                if (cnt < 64) nb[cnt++] = j;
                tot++;
            });
            if (tot <= 64) {
                for (int a = 1; a < cnt; a++) { int v = nb[a], c = a - 1; while (c >= 0 && nb[c] > v) { nb[c + 1] = nb[c]; c--; } nb[c + 1] = v; }
                for (int a = 0; a < cnt; a++) hs_pair(nb[a], 0);
            } else {
                // each pass applies the smallest partner above the last one: tot passes at most
                int last = -1;
                for (int pass = 0; pass < tot; pass++) {
                    int best = 0x7fffffff;
                    for_cell_neighbours(s, r, b, x, geo, cell_off, cstart, csorted, [&](int j) {
                        if (j > last && j < best && is_partner(j)) best = j;
                    });
                    if (best == 0x7fffffff) break;
                    hs_pair(best, 0);
                    last = best;
                }
            }
        }
        for (int c = 0; c < s.Nc; c++) hs_pair((long)s.bead_off + s.Nm + c, 1);
        if (!s.mm_HI && s.mono_ev) {
            // monomer WCA through the cell list (cell_list.cpp:98-172)
            double rc = (double)s.rcut[0], sig = (double)s.sig[0];
            for_cell_neighbours(s, r, b, x, geo, cell_off, cstart, csorted, [&](int j) {
                double dx = x[3 * b] - x[3 * (long)j], dy = x[3 * b + 1] - x[3 * (long)j + 1], dz = x[3 * b + 2] - x[3 * (long)j + 2];
                min_image(s, dx, dy, dz);
                double d2 = dx * dx + dy * dy + dz * dz;
                if (d2 >= rc * rc || d2 == 0.0) return;
                if (!ref_cells_adjacent(geo + 20 * r + 10, x, b, j)) return;
                double dr = sqrt(d2), ri = 1.0 / dr;
                double fm = wca_mag(dr, ri, sig, rc, s.epsilon);
                if (fm == 0.0) return;
                // reference: f_i -= fm d/r for the lower index i of the pair (visited as (i,j))
                f[0] -= fm * dx * ri; f[1] -= fm * dy * ri; f[2] -= fm * dz * ri;
            });
        }
    } else {
        // the sweep over the replica's monomers ran in k_colloid_hs, in the same order
        const long g = (long)s.coll_off + (i - s.Nm);
        f[0] = chs[3 * g]; f[1] = chs[3 * g + 1]; f[2] = chs[3 * g + 2];
        for (int c = 0; c < s.Nc; c++)
            if (s.Nm + c != i) hs_pair((long)s.bead_off + s.Nm + c, 2);
    }
    // bonds (rhs.cpp:102-158): partner list in bond-index order
    for (int q = bptr[b]; q < bptr[b + 1]; q++) {
        long j = bnbr[q];
        double sg = bsgn[q];   // -1: b is the bond's first bead, +1: second
        long kk = sg < 0 ? b : j, jj = sg < 0 ? j : b;
        double rr[4];
        rr[0] = x[3 * kk] - x[3 * jj]; rr[1] = x[3 * kk + 1] - x[3 * jj + 1]; rr[2] = x[3 * kk + 2] - x[3 * jj + 2];
        min_image(s, rr[0], rr[1], rr[2]);
        rr[3] = sqrt(rr[0] * rr[0] + rr[1] * rr[1] + rr[2] * rr[2]);
        double fb[3];
        for (int d = 0; d < 3; d++) fb[d] = -s.kbond * (1 - (s.r0 / rr[3])) * rr[d];
        if (s.fene) {
            double ext2 = 1 / (1 - (rr[3] / s.Lmax) * (rr[3] / s.Lmax));
            for (int d = 0; d < 3; d++) fb[d] *= ext2;
        }
        for (int d = 0; d < 3; d++) f[d] += sg * fb[d];
    }
    // static trap (rhs.cpp:46-100)
    if (!mono) {
        const double *ti = trapinfo + 3 * r;   // tstop, weaken_trap, active
        double kt = ktrap[r];
        if (fabs(kt) >= 1e-12) {
            if (time[r] > ti[0] && ti[1] >= 0) kt = ti[1];
            int c = i - s.Nm;
            double dx = x[3 * b] - xpos0[3 * ((long)s.coll_off + c)];
            double dy = x[3 * b + 1] - xpos0[3 * ((long)s.coll_off + c) + 1];
            double dz = x[3 * b + 2] - xpos0[3 * ((long)s.coll_off + c) + 2];
            min_image(s, dx, dy, dz);
            f[0] += kt * dx; f[1] += kt * dy; f[2] += kt * dz;
        }
    }
    double *o = rhs + s.vec_off + s.nm3nc11 + 3 * i;
    o[0] = f[0]; o[1] = f[1]; o[2] = f[2];
}

// weaken_trap mutates ktrap permanently once t > tstop (rhs.cpp:151-153)
__global__ void k_trap_weaken(int R, const Seg *__restrict__ segs, const double *__restrict__ time,
                              double *__restrict__ ktrap, const double *__restrict__ trapinfo)
{
    pdl_enter();
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= R) return;
    const double *ti = trapinfo + 3 * r;
    if (fabs(ktrap[r]) >= 1e-12 && time[r] > ti[0] && ti[1] >= 0) ktrap[r] = ti[1];
}

// rhs: zero everything but the force block (or the drift block)
__global__ void k_rhs_zero(long nvec, const int *__restrict__ vec_offs, int R, const Seg *__restrict__ segs,
                           int drift, const double *__restrict__ fext, const int *__restrict__ vel_offs,
                           double *__restrict__ rhs)
{
    pdl_enter();
    long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nvec) return;
    int r = rep_of(vec_offs, R, k);
    const Seg &s = segs[r];
    int i = (int)(k - s.vec_off);
    if (drift) {
        int j = i - s.nm3nc11;
        rhs[k] = (j >= 0) ? fext[s.vel_off + j] : 0.0;
    } else {
        // the force block [nm3nc11, nm3nc11 + nm3nc3) is written by k_forces
        int j = i - s.nm3nc11;
        if (j < 0 || j >= s.nm3nc3) rhs[k] = 0.0;
    }
    (void)vel_offs;
}

int stage_rhs(Engine &E, int drift, const double *fext, double *rhs, cudaStream_t st)
{
    int thr = 256;
    ps_launch(k_rhs_zero, (unsigned)((E.nvec + thr - 1) / thr), thr, 0, st, E.nvec, E.d_vec_offs, E.R, E.d_segs, drift, fext,
            E.d_vel_offs, rhs);
    if (!drift) {
        if (E.ncoll)
            ps_launch(k_colloid_hs, (unsigned)E.ncoll, 32, 0, st, E.ncoll, E.d_coll_rep, E.d_segs, E.d_x,
                    E.d_chs);
        ps_launch(k_forces, (unsigned)((E.ntot + thr - 1) / thr), thr, 0, st,
                E.ntot, E.d_bead_offs, E.R, E.d_segs, E.d_x, E.d_xpos0, E.d_cellgeo, E.d_cell_offs,
                E.d_cell_start, E.d_cell_sorted, E.d_bond_ptr, E.d_bond_nbr, E.d_bond_sgn, E.d_time, E.d_ktrap,
                E.d_trapinfo, E.d_chs, rhs);
        ps_launch(k_trap_weaken, (E.R + 127) / 128, 128, 0, st, E.R, E.d_segs, E.d_time, E.d_ktrap, E.d_trapinfo);
    }
    PS_CK(cudaGetLastError());
    return PS_OK;
}

int stage_pairs(Engine &E, cudaStream_t st)
{
    int rc = stage_pack(E, st);
    if (rc) return rc;
    if (E.need_cells && (rc = stage_cells(E, st, E.d_cell_offs, E.ncells))) return rc;
    if (E.any_lub) {
        if (!E.d_lubtab) { set_error("lubrication requested but no table set (ps_set_lub_table)"); return PS_ERR_STATE; }
        if ((rc = lub_build(E, st))) return rc;
        if ((rc = lub_diag(E, st))) return rc;
    }
    return PS_OK;
}

// ---------------------------------------------------------------------------
// mob() bookkeeping (mob.cpp:845-1029): the AB translational block of the
// dense path is the global mob_a left by the last pair tensor evaluated before
// the AB loop -- the last non-skipped AA pair of this call, else the previous
// call's final mob_a (BB tensor of the last colloid pair, or I from fill_self).
__global__ void k_assemble(int R, const Seg *__restrict__ segs, const double *__restrict__ x,
                           const int *__restrict__ aa_last, double *__restrict__ tab, double *__restrict__ stale)
{
    pdl_enter();
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= R) return;
    const Seg &s = segs[r];
    double *t = tab + 9 * r, *sa = stale + 9 * r;
    if (s.ab_mode != PS_AB_REFERENCE || !s.mm_HI) {
        for (int a = 0; a < 9; a++) t[a] = 0.0;
    } else {
        int li = aa_last[2 * r], lj = aa_last[2 * r + 1];
        if (li >= 0) {
            double e[3];
            double dr = pair_geom(s, x, (long)s.bead_off + li, (long)s.bead_off + lj, e);
            double ri = 1 / dr;
            double xx, yy;
            if (s.aa_mode == PS_AA_RPY) aa_scalars_rpy<double>(dr, ri, 2.0 * s.beta, xx, yy);
            else aa_scalars<double>(dr, ri, 2.0 * s.beta, xx, yy);
            for (int a = 0; a < 3; a++)
                for (int c = 0; c < 3; c++) sa[3 * a + c] = (a == c) ? xx * e[a] * e[a] + yy * (1. - e[a] * e[a])
                                                                   : xx * (e[a] * e[c]) - yy * (e[a] * e[c]);
        }
        for (int a = 0; a < 9; a++) t[a] = sa[a];
    }
    if (s.Nc >= 2) {
        double e[3];
        double dr = pair_geom(s, x, (long)s.bead_off + s.Np - 2, (long)s.bead_off + s.Np - 1, e);
        double ri = 1 / dr, ri3 = ri * ri * ri;
        double xa = 1.5 * ri - ri3, ya = 0.75 * ri + 0.5 * ri3;
        for (int a = 0; a < 3; a++)
            for (int c = 0; c < 3; c++) sa[3 * a + c] = (a == c) ? xa * e[a] * e[a] + ya * (1. - e[a] * e[a])
                                                               : xa * (e[a] * e[c]) - ya * (e[a] * e[c]);
    }
}

// ---------------------------------------------------------------------------
// Arrowhead Schur floor (slip_vel.cpp:81-203), one block per shell replica:
// S = Mcc_base - beta Mcm Mcm^T, eig, delta_j = max(0.1 - lambda_j, 0),
// Delta = Q diag(delta) Q^T; Mcc_base holds the colloid self blocks plus the
// colloid-colloid pair blocks (those the reference's shell cannot store).
// Symmetric eigendecomposition by cyclic Jacobi in shared memory.
__device__ void block_jacobi_eig(double *A, double *Q, int n, double *lam)
{
    // A, Q: n x n row-major in shared memory; all threads of the block participate
    for (int k = threadIdx.x; k < n * n; k += blockDim.x) Q[k] = (k / n == k % n) ? 1.0 : 0.0;
    __shared__ double cs_sh[2];
    __shared__ int conv;
    __syncthreads();
    for (int sweep = 0; sweep < 60; sweep++) {
        if (threadIdx.x == 0) {
            double off = 0, tot = 0;
            for (int i = 0; i < n; i++) for (int j = 0; j < n; j++) { double v = A[i * n + j] * A[i * n + j]; tot += v; if (i != j) off += v; }
            conv = (off <= 1e-30 * tot || off == 0.0);
        }
        __syncthreads();
        if (conv) break;
        for (int p = 0; p < n - 1; p++)
            for (int q = p + 1; q < n; q++) {
                if (threadIdx.x == 0) {
                    double apq = A[p * n + q];
                    if (fabs(apq) < 1e-300) { cs_sh[0] = 1.0; cs_sh[1] = 0.0; }
                    else {
                        double theta = (A[q * n + q] - A[p * n + p]) / (2 * apq);
                        double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1));
                        double c = 1 / sqrt(t * t + 1);
                        cs_sh[0] = c; cs_sh[1] = t * c;
                    }
                }
                __syncthreads();
                double c = cs_sh[0], sn = cs_sh[1];
                if (sn != 0.0) {
                    for (int k = threadIdx.x; k < n; k += blockDim.x) {
                        double akp = A[k * n + p], akq = A[k * n + q];
                        A[k * n + p] = c * akp - sn * akq; A[k * n + q] = sn * akp + c * akq;
                    }
                    __syncthreads();
                    for (int k = threadIdx.x; k < n; k += blockDim.x) {
                        double apk = A[p * n + k], aqk = A[q * n + k];
                        A[p * n + k] = c * apk - sn * aqk; A[q * n + k] = sn * apk + c * aqk;
                        double qkp = Q[k * n + p], qkq = Q[k * n + q];
                        Q[k * n + p] = c * qkp - sn * qkq; Q[k * n + q] = sn * qkp + c * qkq;
                    }
                }
                __syncthreads();
            }
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x) lam[i] = A[i * n + i];
    __syncthreads();
}

__global__ void k_schur(const Seg *__restrict__ segs, const int *__restrict__ reps, const double *__restrict__ x,
                        double *__restrict__ delta, double *__restrict__ schurQ, double *__restrict__ schurL,
                        const double *__restrict__ tab)
{
    pdl_enter();
    extern __shared__ double sm[];
    const int r = reps[blockIdx.x];
    const Seg &s = segs[r];
    const int n = s.nc11, Nm = s.Nm, Nc = s.Nc;
    double *S = sm, *Q = sm + n * n, *lam = sm + 2 * n * n;
    // Mcc_base: self + BB pairs, built by applying the pair operator to unit vectors
    for (int k = threadIdx.x; k < n * n; k += blockDim.x) S[k] = 0.0;
    __syncthreads();
    if (threadIdx.x < Nc) {
        int c = threadIdx.x, t = 3 * c, ro = s.nc3 + 3 * c, st = s.nc6 + 5 * c;
        for (int a = 0; a < 3; a++) { S[(t + a) * n + t + a] = 1.0; S[(ro + a) * n + ro + a] = 0.75; }
        for (int a = 0; a < 5; a++) S[(st + a) * n + st + a] = 1.8;
        S[st * n + st + 4] = 0.9; S[(st + 4) * n + st] = 0.9;
    }
    __syncthreads();
    // pair blocks: thread per (colloid row, column colloid, unit input component)
    for (int w = threadIdx.x; w < Nc * Nc * 11; w += blockDim.x) {
        int ci = w / (Nc * 11), rem = w % (Nc * 11), cj = rem / 11, q = rem % 11;
        if (ci == cj) continue;
        bool lo = ci < cj;
        long bl = (long)s.bead_off + Nm + (lo ? ci : cj), bh = (long)s.bead_off + Nm + (lo ? cj : ci);
        double e[3];
        double dr = pair_geom(s, x, bl, bh, e);
        double in[11], out[11];
        for (int k = 0; k < 11; k++) { in[k] = (k == q) ? 1.0 : 0.0; out[k] = 0.0; }
        bb_apply<double>(e, dr, 1.0 / dr, lo, in, out);
        int colj = q < 3 ? 3 * cj + q : (q < 6 ? s.nc3 + 3 * cj + (q - 3) : s.nc6 + 5 * cj + (q - 6));
        for (int k = 0; k < 11; k++) {
            int rowi = k < 3 ? 3 * ci + k : (k < 6 ? s.nc3 + 3 * ci + (k - 3) : s.nc6 + 5 * ci + (k - 6));
            S[rowi * n + colj] += out[k];
        }
    }
    __syncthreads();
    // Gram of Mcm: column (m,d) entries per colloid c: trans T^T[d] (reference: 0),
    // rot B[:,d], stress G[d,:]
    for (int w = threadIdx.x; w < n * n; w += blockDim.x) {
        int a = w / n, bcol = w % n;
        if (bcol < a) continue;
        int ca, qa, cb, qb;
        auto decode = [&](int j, int &c, int &q) {
            if (j < s.nc3) { c = j / 3; q = j % 3; }
            else if (j < s.nc6) { c = (j - s.nc3) / 3; q = 3 + (j - s.nc3) % 3; }
            else { c = (j - s.nc6) / 5; q = 6 + (j - s.nc6) % 5; }
        };
        decode(a, ca, qa); decode(bcol, cb, qb);
        double acc = 0.0;
        for (int m = 0; m < Nm; m++) {
            double col_a[3], col_b[3];
            for (int side = 0; side < 2; side++) {
                int c = side ? cb : ca, q = side ? qb : qa;
                double *col = side ? col_b : col_a;
                double e[3];
                double dr = pair_geom(s, x, (long)s.bead_off + m, (long)s.bead_off + Nm + c, e);
                double ri = 1.0 / dr;
                double yb, xg, yg;
                ab_scalars<double>(ri, s.beta * s.beta, yb, xg, yg);
                double xa = 0.0, ya = 0.0;
                if (s.ab_mode == PS_AB_RPY || s.ab_mode == PS_AB_RPY_REG)
                    ab_trans_scalars<double>(dr, ri, s.beta, s.ab_mode == PS_AB_RPY_REG, xa, ya, yb);
                for (int d = 0; d < 3; d++) {
                    double v;
                    if (q < 3) {
                        if (s.ab_mode == PS_AB_RPY || s.ab_mode == PS_AB_RPY_REG) {
                            v = xa * e[d] * e[q] + ya * ((d == q) - e[d] * e[q]);
                        } else v = 0.0;
                    } else if (q < 6) {
                        int aa = q - 3;   // B[aa][d] = yb eps_{aa d k} e_k
                        int kk = 3 - aa - d;
                        double eps = 0.0;
                        if (aa != d && kk >= 0 && kk < 3) eps = ((aa - d + 3) % 3 == 2) ? 1.0 : -1.0;
                        v = (aa != d) ? yb * eps * e[kk] : 0.0;
                    } else {
                        double G[15];
                        gt_flat<double>(e, xg, yg, G);
                        v = G[d * 5 + (q - 6)];
                    }
                    col[d] = v;
                }
            }
            acc += col_a[0] * col_b[0] + col_a[1] * col_b[1] + col_a[2] * col_b[2];
        }
        S[a * n + bcol] -= s.beta * acc;
        if (bcol != a) S[bcol * n + a] -= s.beta * acc;
    }
    __syncthreads();
    block_jacobi_eig(S, Q, n, lam);
    double *D = delta + s.schur_off, *QQ = schurQ + s.schur_off, *LL = schurL + s.schur_off;
    for (int w = threadIdx.x; w < n * n; w += blockDim.x) {
        int a = w / n, bcol = w % n;
        double corr = 0.0;
        for (int j = 0; j < n; j++) {
            double d = lam[j] < 0.1 ? 0.1 - lam[j] : 0.0;
            if (d == 0.0) continue;
            corr += Q[a * n + j] * d * Q[bcol * n + j];
        }
        D[w] = corr;
        QQ[w] = Q[w];
    }
    for (int j = threadIdx.x; j < n; j += blockDim.x) LL[j] = lam[j] < 0.1 ? 0.1 : lam[j];
    (void)tab;
}

int stage_assemble(Engine &E, cudaStream_t st)
{
    ps_launch(k_assemble, (E.R + 127) / 128, 128, 0, st, E.R, E.d_segs, E.d_x, E.d_aa_last, E.d_tab, E.d_stale);
    PS_CK(cudaGetLastError());
    return PS_OK;
}

int stage_schur(Engine &E, cudaStream_t st)
{
    if (!E.n_schur_reps) return PS_OK;
    size_t smem = sizeof(double) * (2 * 64 * 64 + 64);
    PS_CK(cudaFuncSetAttribute(k_schur, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    ps_launch(k_schur, E.n_schur_reps, 256, smem, st, E.d_segs, E.d_schur_reps, E.d_x, E.d_delta, E.d_schurQ, E.d_schurL,
            E.d_tab);
    PS_CK(cudaGetLastError());
    return PS_OK;
}

// ---------------------------------------------------------------------------
// Jacobi diagonal (matfree_A.cpp:84-102 with PCJacobiSetFixDiagonal)
__global__ void k_diag(long nvec, const int *__restrict__ vec_offs, int R, const Seg *__restrict__ segs,
                       const double *__restrict__ delta, const double *__restrict__ luby_diag, double *__restrict__ d)
{
    pdl_enter();
    long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nvec) return;
    int r = rep_of(vec_offs, R, k);
    const Seg &s = segs[r];
    int i = (int)(k - s.vec_off);
    double v;
    if (i < s.nm3) v = s.beta_inv;
    else if (i < s.nm3nc11) {
        int j = i - s.nm3;
        if (j < s.nc3) v = 1.0;
        else if (j < s.nc6) v = 0.75;
        else v = 1.8;
        if (s.shell_schur) v += delta[s.schur_off + (long)j * s.nc11 + j];
    } else {
        v = 0.0;
        if (s.lub_on && luby_diag) v = fabs(luby_diag[s.vel_off + (i - s.nm3nc11)]);
    }
    d[k] = (v == 0.0) ? 1.0 : v;
}

int diag_saddle(Engine &E, double *d, cudaStream_t st)
{
    int thr = 256;
    ps_launch(k_diag, (unsigned)((E.nvec + thr - 1) / thr), thr, 0, st, E.nvec, E.d_vec_offs, E.R, E.d_segs, E.d_delta,
            E.any_lub ? E.d_lub_diag : nullptr, d);
    PS_CK(cudaGetLastError());
    return PS_OK;
}


int pair_list(Engine &E, int which, int32_t *pi, int32_t *pj, int64_t maxp, int64_t *count, cudaStream_t st);

}  // namespace ps
