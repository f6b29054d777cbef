// pairs.cu -- explicit pair lists (CSR over beads, i < j, ascending j):
//   which 0: Verlet pairs of check_dist.cpp:37-62 (stored pairs with dr < rverl[type];
//            AA pairs only when mm_HI), found through the monomer cell list;
//   which 1: monomer WCA pairs of cell_list.cpp:98-172 (dr^2 < rcut[0]^2, dr != 0);
//   which 2: lubricated pairs (equal-radius pairs with gap < lub_gap * a).
// Compiled with --fmad=false: distances round exactly as in the reference.
#include <cmath>
#include <vector>
#include "ps_internal.h"
#include "ps_kernels.h"

namespace ps {

__device__ __forceinline__ int rep_find(const int *__restrict__ offs, int R, long k)
{
    int lo = 0, hi = R;
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (offs[mid] <= k) lo = mid; else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ void mimg(const Seg &s, double &dx, double &dy, double &dz)
{
    if (!s.box_on) return;
    dx -= s.L[0] * nearbyint(dx * (1.0 / s.L[0]));
    dy -= s.L[1] * nearbyint(dy * (1.0 / s.L[1]));
    dz -= s.L[2] * nearbyint(dz * (1.0 / s.L[2]));
}

// clamp in double before converting: NaN and out-of-range values map into [0, nc)
__device__ __forceinline__ int ccoord(double v, double org, double size, int nc)
{
    double f = floor((v - org) / size);
    if (!(f >= 0.0)) return 0;
    if (f >= (double)nc) return nc - 1;
    return (int)f;
}

// does pair (b, j), b < j (global indices, same replica) belong to list `which`?
__device__ __forceinline__ bool ref_adjacent(const double *__restrict__ gref, const double *__restrict__ x, long i, long j)
{
    for (int d = 0; d < 3; d++) {
        int nc = (int)gref[6 + d];
        int ci = ccoord(x[3 * i + d], gref[d], gref[3 + d], nc);
        int cj = ccoord(x[3 * j + d], gref[d], gref[3 + d], nc);
        int dc = ci - cj;
        if (gref[9] != 0.0) {
            dc = ((dc % nc) + nc) % nc;
            if (dc > 1 && dc < nc - 1) return false;
        } else if (dc > 1 || dc < -1) return false;
    }
    return true;
}

__device__ __forceinline__ bool in_list(const Seg &s, const double *__restrict__ x, long b, long j, int which,
                                        const double *__restrict__ gref)
{
    int i = (int)(b - s.bead_off), k = (int)(j - s.bead_off);
    bool mi = i < s.Nm, mk = k < s.Nm;
    double dx = x[3 * b] - x[3 * j], dy = x[3 * b + 1] - x[3 * j + 1], dz = x[3 * b + 2] - x[3 * j + 2];
    mimg(s, dx, dy, dz);
    double d2 = dx * dx + dy * dy + dz * dz;
    if (which == 0) {
        int type = (mi && mk) ? 0 : ((mi || mk) ? 1 : 2);
        if (type == 0 && !s.mm_HI) return false;
        double dr = sqrt(d2);
        return dr < (double)s.rverl[type];
    }
    if (which == 1) {
        if (!(mi && mk)) return false;
        double rc = (double)s.rcut[0];
        return d2 < rc * rc && d2 != 0.0 && ref_adjacent(gref, x, b, j);
    }
    // which == 2 or 3 (lubrication)
    if (mi != mk) return false;
    if (mi && !s.lub_bonded && i / s.nper == k / s.nper && (k - i == 1 || i - k == 1)) return false;
    double a = mi ? s.beta : 1.0;
    double dr = sqrt(d2);
    return dr - 2 * a < s.lub_gap * a;
}

template <class F>
__device__ __forceinline__ void partners(const Seg &s, int r, long b, const double *__restrict__ x,
                                         const double *__restrict__ geo, const long *__restrict__ cell_off,
                                         const int *__restrict__ cstart, const int *__restrict__ csorted, int which, F f)
{
    int i = (int)(b - s.bead_off);
    if (i < s.Nm && (which != 0 || s.mm_HI)) {
        const double *g = geo + 20 * r;
        int nc[3] = {(int)g[6], (int)g[7], (int)g[8]};
        int periodic = (int)g[9];
        int c[3];
        for (int d = 0; d < 3; d++) c[d] = ccoord(x[3 * b + d], g[d], g[3 + d], nc[d]);
        for (int dz = -1; dz <= 1; dz++)
            for (int dy = -1; dy <= 1; dy++)
                for (int dxx = -1; dxx <= 1; dxx++) {
                    int q[3] = {c[0] + dxx, c[1] + dy, c[2] + dz};
                    bool ok = true;
                    for (int d = 0; d < 3; d++) {
                        if (periodic) q[d] = (q[d] % nc[d] + nc[d]) % nc[d];
                        else if (q[d] < 0 || q[d] >= nc[d]) ok = false;
                    }
                    if (!ok) continue;
                    // a periodic axis with fewer than 3 cells would visit a cell twice
                    long cc = cell_off[r] + q[0] + (long)nc[0] * (q[1] + (long)nc[1] * q[2]);
                    for (int k = cstart[cc]; k < cstart[cc + 1]; k++) {
                        long j = csorted[k];
                        bool take = (which == 3) ? (j != b) : (j > b);
                        if (take && in_list(s, x, b, j, which, geo + 20 * r + 10)) f(j);
                    }
                }
    }
    if (which == 0 && i < s.Nm) {
        // a monomer's colloid partners (all colloids follow all monomers);
        // lubrication pairs are equal-radius, so monomers have none there
        for (int c = 0; c < s.Nc; c++) {
            long j = (long)s.bead_off + s.Nm + c;
            bool take = (which == 3) ? (j != b) : (j > b);
            if (take && in_list(s, x, b, j, which, geo + 20 * r + 10)) f(j);
        }
    }
}

// A colloid's partners are colloids only (monomer-colloid pairs belong to the
// monomer): one warp per colloid scans the replica's colloids 32 at a time and a
// ballot hands each partner its rank, so the list comes out in ascending order.
template <class F>
__device__ __forceinline__ int colloid_partners_warp(const Seg &s, int r, long b, const double *__restrict__ x,
                                                     const double *__restrict__ geo, int which, int lane, F f)
{
    int n = 0;
    if (which == 1) return 0;
    const int i = (int)(b - s.bead_off);
    const int c0 = (which == 3) ? 0 : i - s.Nm + 1;
    for (int cb = c0; cb < s.Nc; cb += 32) {
        const int c = cb + lane;
        const long j = (long)s.bead_off + s.Nm + c;
        const bool hit = c < s.Nc && ((which == 3) ? (j != b) : (j > b)) && in_list(s, x, b, j, which, geo + 20 * r + 10);
        const unsigned m = __ballot_sync(0xffffffffu, hit);
        if (hit) f(j, n + __popc(m & ((1u << lane) - 1u)));
        n += __popc(m);
    }
    return n;
}

// Monomers: one thread each (cell-list stencil, then the colloids); colloids:
// one warp each in the blocks past the bead blocks.
__global__ void k_pairs_count(long ntot, const int *__restrict__ bead_offs, int R, const Seg *__restrict__ segs,
                              const double *__restrict__ x, const double *__restrict__ geo,
                              const long *__restrict__ cell_off, const int *__restrict__ cstart,
                              const int *__restrict__ csorted, long ncoll, const int *__restrict__ coll_rep,
                              int which, int *__restrict__ cnt)
{
    pdl_enter();
    const long nbb = (ntot + blockDim.x - 1) / blockDim.x;
    if (blockIdx.x >= nbb) {
        const long c = (long)(blockIdx.x - nbb) * (blockDim.x >> 5) + (threadIdx.x >> 5);
        if (c >= ncoll) return;
        const int lane = threadIdx.x & 31, r = coll_rep[c];
        const Seg &s = segs[r];
        const long b = s.bead_off + s.Nm + (c - s.coll_off);
        const int n = colloid_partners_warp(s, r, b, x, geo, which, lane, [&](long, int) {});
        if (lane == 0) cnt[b] = n;
        return;
    }
    long b = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= ntot) return;
    int r = rep_find(bead_offs, R, b);
    if (b - segs[r].bead_off >= segs[r].Nm) return;
    int n = 0;
    partners(segs[r], r, b, x, geo, cell_off, cstart, csorted, which, [&](long) { n++; });
    cnt[b] = n;
}

__global__ void k_pairs_fill(long ntot, const int *__restrict__ bead_offs, int R, const Seg *__restrict__ segs,
                             const double *__restrict__ x, const double *__restrict__ geo,
                             const long *__restrict__ cell_off, const int *__restrict__ cstart,
                             const int *__restrict__ csorted, long ncoll, const int *__restrict__ coll_rep, int which,
                             const int *__restrict__ ptr, int *__restrict__ nbr)
{
    pdl_enter();
    const long nbb = (ntot + blockDim.x - 1) / blockDim.x;
    if (blockIdx.x >= nbb) {
        const long c = (long)(blockIdx.x - nbb) * (blockDim.x >> 5) + (threadIdx.x >> 5);
        if (c >= ncoll) return;
        const int lane = threadIdx.x & 31, r = coll_rep[c];
        const Seg &s = segs[r];
        const long b = s.bead_off + s.Nm + (c - s.coll_off);
        const int a = ptr[b];
        colloid_partners_warp(s, r, b, x, geo, which, lane, [&](long j, int k) { nbr[a + k] = (int)j; });
        return;
    }
    long b = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= ntot) return;
    int r = rep_find(bead_offs, R, b);
    if (b - segs[r].bead_off >= segs[r].Nm) return;
    int a = ptr[b], n = 0;
    partners(segs[r], r, b, x, geo, cell_off, cstart, csorted, which, [&](long j) { nbr[a + n++] = (int)j; });
    // ascending partner order
    for (int u = a + 1; u < a + n; u++) {
        int v = nbr[u], w = u - 1;
        while (w >= a && nbr[w] > v) { nbr[w + 1] = nbr[w]; w--; }
        nbr[w + 1] = v;
    }
}

// Exclusive scan out[0..n] of in[0..n-1] (out[n] = total), three phases: each
// block scans SCAN_SPAN elements (16 per thread, warp-shuffle scan of the thread
// totals), one block scans the block totals, then every block adds its offset.
constexpr int SCAN_T = 256, SCAN_E = 16, SCAN_SPAN = SCAN_T * SCAN_E;

__global__ void __launch_bounds__(SCAN_T) k_scan_local(long n, const int *__restrict__ in, int *__restrict__ out,
                                                       int *__restrict__ sums)
{
    pdl_enter();
    __shared__ int ws[SCAN_T / 32];
    const long base = (long)blockIdx.x * SCAN_SPAN + (long)threadIdx.x * SCAN_E;
    int v[SCAN_E], tot = 0;
#pragma unroll
    for (int e = 0; e < SCAN_E; e++) {
        long k = base + e;
        v[e] = k < n ? in[k] : 0;
        tot += v[e];
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int inc = tot;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane == 31) ws[w] = inc;
    __syncthreads();
    if (w == 0) {
        int x = lane < SCAN_T / 32 ? ws[lane] : 0, xi = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int t = __shfl_up_sync(0xffffffffu, xi, o);
            if (lane >= o) xi += t;
        }
        if (lane < SCAN_T / 32) ws[lane] = xi - x;
    }
    __syncthreads();
    int ex = ws[w] + inc - tot;
#pragma unroll
    for (int e = 0; e < SCAN_E; e++) {
        long k = base + e;
        if (k < n) out[k] = ex;
        ex += v[e];
    }
    if (threadIdx.x == SCAN_T - 1) sums[blockIdx.x] = ws[w] + inc;
}

// in-place exclusive scan of the m block totals, total into sums[m]
__global__ void k_scan_sums(int m, int *__restrict__ sums)
{
    pdl_enter();
    __shared__ int carry;
    __shared__ int tmp[1024];
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < m; base += 1024) {
        int k = base + threadIdx.x;
        int v = k < m ? sums[k] : 0;
        tmp[threadIdx.x] = v;
        __syncthreads();
        for (int o = 1; o < 1024; o <<= 1) {
            int t = threadIdx.x >= o ? tmp[threadIdx.x - o] : 0;
            __syncthreads();
            tmp[threadIdx.x] += t;
            __syncthreads();
        }
        if (k < m) sums[k] = carry + tmp[threadIdx.x] - v;
        __syncthreads();
        if (threadIdx.x == 1023) carry += tmp[1023];
        __syncthreads();
    }
    if (threadIdx.x == 0) sums[m] = carry;
}

__global__ void __launch_bounds__(SCAN_T) k_scan_add(long n, int m, const int *__restrict__ sums, int *__restrict__ out)
{
    pdl_enter();
    const int off = sums[blockIdx.x];
    const long base = (long)blockIdx.x * SCAN_SPAN;
    for (int e = threadIdx.x; e < SCAN_SPAN; e += SCAN_T) {
        long k = base + e;
        if (k < n) out[k] += off;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = sums[m];
}

int exclusive_scan(Engine &E, const int *in, int *out, long n, cudaStream_t st)
{
    long m = (n + SCAN_SPAN - 1) / SCAN_SPAN;
    if (m < 1) m = 1;
    if (m + 1 > E.scan_cap) { set_error("scan scratch too small"); return PS_ERR_STATE; }
    ps_launch(k_scan_local, (unsigned)m, SCAN_T, 0, st, n, in, out, E.d_scan_sums);
    ps_launch(k_scan_sums, 1, 1024, 0, st, (int)m, E.d_scan_sums);
    ps_launch(k_scan_add, (unsigned)m, SCAN_T, 0, st, n, (int)m, E.d_scan_sums, out);
    PS_CK(cudaGetLastError());
    return PS_OK;
}

__global__ void k_pairs_expand(long ntot, const int *__restrict__ ptr, const int *__restrict__ nbr,
                               int32_t *__restrict__ pi, int32_t *__restrict__ pj, long maxp)
{
    pdl_enter();
    long b = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= ntot) return;
    for (int k = ptr[b]; k < ptr[b + 1]; k++)
        if (k < maxp) { pi[k] = (int32_t)b; pj[k] = nbr[k]; }
}

// Builds the CSR list into E.d_nbr_ptr / E.d_nbr (grown on demand).
int build_list(Engine &E, int which, long *npairs, cudaStream_t st)
{
    int thr = 128;
    unsigned nbk = (unsigned)((E.ntot + thr - 1) / thr + (E.ncoll + thr / 32 - 1) / (thr / 32));
    ps_launch(k_pairs_count, nbk, thr, 0, st, E.ntot, E.d_bead_offs, E.R, E.d_segs, E.d_x, E.d_cellgeo, E.d_cell_offs,
            E.d_cell_start, E.d_cell_sorted, E.ncoll, E.d_coll_rep, which, E.d_nbr_count);
    int rc = exclusive_scan(E, E.d_nbr_count, E.d_nbr_ptr, E.ntot, st);
    if (rc) return rc;
    int tot = 0;
    PS_CK(cudaMemcpyAsync(&tot, E.d_nbr_ptr + E.ntot, sizeof(int), cudaMemcpyDeviceToHost, st));
    PS_CK(cudaStreamSynchronize(st));
    if (tot > E.nbr_cap) {
        cudaFree(E.d_nbr);
        E.nbr_cap = (long)tot * 3 / 2 + 1024;
        PS_CK(cudaMalloc(&E.d_nbr, sizeof(int) * E.nbr_cap));
    }
    ps_launch(k_pairs_fill, nbk, thr, 0, st, E.ntot, E.d_bead_offs, E.R, E.d_segs, E.d_x, E.d_cellgeo, E.d_cell_offs,
            E.d_cell_start, E.d_cell_sorted, E.ncoll, E.d_coll_rep, which, E.d_nbr_ptr, E.d_nbr);
    PS_CK(cudaGetLastError());
    *npairs = tot;
    return PS_OK;
}

int pair_list(Engine &E, int which, int32_t *pi, int32_t *pj, int64_t maxp, int64_t *count, cudaStream_t st)
{
    long np = 0;
    int rc = build_list(E, which, &np, st);
    if (rc) return rc;
    if (pi && pj && maxp > 0) {
        int thr = 128;
        ps_launch(k_pairs_expand, (unsigned)((E.ntot + thr - 1) / thr), thr, 0, st, E.ntot, E.d_nbr_ptr, E.d_nbr, pi, pj, maxp);
        PS_CK(cudaGetLastError());
    }
    if (count) *count = np;
    return PS_OK;
}

}  // namespace ps
