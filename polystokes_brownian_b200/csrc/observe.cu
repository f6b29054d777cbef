// observe.cu -- trajectory observables accumulated on the device (the analysis
// the reference runs on its output files: bond and trap statistics of
// test_sim_dumbbells_thermal.py:178-330, the MSD tensor of get_msd.py:5-28).
//
// One launch per observation updates per-bead accumulators (no atomics on
// floating-point sums, so results are deterministic), integer histograms per
// replica (exact atomic counts) and, for every colloid, a ring buffer of past
// positions from which the windowed MSD tensor sums are accumulated for lags
// 0..L-1.  ps_obs_read reduces the per-bead sums per replica on the host.
// Positions are taken as stored: under periodic boxes bond and trap vectors use
// the minimum image, the MSD uses the wrapped positions as they are.
#include <cmath>
#include <vector>
#include "ps_internal.h"
#include "ps_kernels.h"

namespace ps {

__device__ __forceinline__ int obs_rep(const int *__restrict__ offs, int R, long k)
{
    int lo = 0, hi = R;
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (offs[mid] <= k) lo = mid; else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ void obs_mimg(const Seg &s, double &dx, double &dy, double &dz)
{
    if (!s.box_on) return;
    dx -= s.L[0] * nearbyint(dx * (1.0 / s.L[0]));
    dy -= s.L[1] * nearbyint(dy * (1.0 / s.L[1]));
    dz -= s.L[2] * nearbyint(dz * (1.0 / s.L[2]));
}

// per bead: its bonds to higher-index partners (each bond once) and, for a
// colloid, its displacement from the trap centre.  acc: OBS_K doubles per bead.
__global__ void k_observe(long ntot, const int *__restrict__ bead_offs, int R, const Seg *__restrict__ segs,
                          const double *__restrict__ x, const double *__restrict__ xpos0,
                          const int *__restrict__ bptr, const int *__restrict__ bnbr, double *__restrict__ acc,
                          double *__restrict__ prev, int *__restrict__ has_prev, unsigned long long *__restrict__ hb,
                          unsigned long long *__restrict__ ht, int nbins, double bmax, double tmax)
{
    pdl_enter();
    long b = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= ntot) return;
    const int r = obs_rep(bead_offs, R, b);
    const Seg &s = segs[r];
    double *a = acc + (long)OBS_K * b;
    for (int t = bptr[b]; t < bptr[b + 1]; t++) {
        long j = bnbr[t];
        if (j <= b) continue;
        double vx = x[3 * j] - x[3 * b], vy = x[3 * j + 1] - x[3 * b + 1], vz = x[3 * j + 2] - x[3 * b + 2];
        obs_mimg(s, vx, vy, vz);
        double l = sqrt(vx * vx + vy * vy + vz * vz);
        a[0] += 1.0; a[1] += vx; a[2] += vy; a[3] += vz; a[4] += l; a[5] += l * l;
        if (has_prev[t]) {
            a[6] += 1.0;
            a[7] += vx - prev[3 * t]; a[8] += vy - prev[3 * t + 1]; a[9] += vz - prev[3 * t + 2];
        }
        prev[3 * t] = vx; prev[3 * t + 1] = vy; prev[3 * t + 2] = vz;
        has_prev[t] = 1;
        int bin = (int)(l / bmax * nbins);
        if (bin >= 0 && bin < nbins) atomicAdd(&hb[(long)r * nbins + bin], 1ull);
    }
    const int i = (int)(b - s.bead_off);
    if (i >= s.Nm) {
        const long c = s.coll_off + (i - s.Nm);
        double dx = x[3 * b] - xpos0[3 * c], dy = x[3 * b + 1] - xpos0[3 * c + 1], dz = x[3 * b + 2] - xpos0[3 * c + 2];
        obs_mimg(s, dx, dy, dz);
        double d2 = dx * dx + dy * dy + dz * dz, d = sqrt(d2);
        a[10] += 1.0; a[11] += dx; a[12] += dy; a[13] += dz; a[14] += d; a[15] += d2;
        a[16] += dx * dx; a[17] += dy * dy; a[18] += dz * dz;
        int bin = (int)(d / tmax * nbins);
        if (bin >= 0 && bin < nbins) atomicAdd(&ht[(long)r * nbins + bin], 1ull);
    }
}

// per colloid: MSD tensor sums against the positions of the last L samples
__global__ void k_observe_msd(long ncoll, const int *__restrict__ coll_rep, const Seg *__restrict__ segs,
                              const double *__restrict__ x, double *__restrict__ ring, double *__restrict__ msd,
                              unsigned long long *__restrict__ cnt, int L, long n)
{
    pdl_enter();
    long c = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncoll) return;
    const Seg &s = segs[coll_rep[c]];
    const long b = (long)s.bead_off + s.Nm + (c - s.coll_off);
    const double px = x[3 * b], py = x[3 * b + 1], pz = x[3 * b + 2];
    double *rg = ring + 3L * L * c;
    const long nl = n < L ? n : L - 1;
    for (long l = 0; l <= nl; l++) {
        double dx = 0.0, dy = 0.0, dz = 0.0;
        if (l > 0) {
            const long o = (n - l) % L;
            dx = px - rg[3 * o]; dy = py - rg[3 * o + 1]; dz = pz - rg[3 * o + 2];
        }
        double *m = msd + 6L * (L * c + l);
        m[0] += dx * dx; m[1] += dy * dy; m[2] += dz * dz; m[3] += dx * dy; m[4] += dx * dz; m[5] += dy * dz;
        cnt[L * c + l] += 1ull;
    }
    const long o = n % L;
    rg[3 * o] = px; rg[3 * o + 1] = py; rg[3 * o + 2] = pz;
}

int obs_reset(Engine &E, int nbins, double bond_max, double trap_max, int lags)
{
    if (nbins < 1 || nbins > 4096 || lags < 1 || lags > 4096 || !(bond_max > 0) || !(trap_max > 0)) {
        set_error("ps_obs_reset: nbins and lags in [1, 4096], positive ranges");
        return PS_ERR_ARG;
    }
    void *ptrs[] = {E.d_obs_acc, E.d_obs_prev, E.d_obs_hasprev, E.d_obs_hb, E.d_obs_ht, E.d_obs_ring, E.d_obs_msd,
                    E.d_obs_msdn};
    for (void *p : ptrs) if (p) cudaFree(p);
    int nbond_slots = 0;
    PS_CK(cudaMemcpy(&nbond_slots, E.d_bond_ptr + E.ntot, sizeof(int), cudaMemcpyDeviceToHost));
    const long nc = std::max<long>(E.ncoll, 1), ns = std::max(nbond_slots, 1);
    PS_CK(cudaMalloc(&E.d_obs_acc, sizeof(double) * OBS_K * E.ntot));
    PS_CK(cudaMalloc(&E.d_obs_prev, sizeof(double) * 3 * ns));
    PS_CK(cudaMalloc(&E.d_obs_hasprev, sizeof(int) * ns));
    PS_CK(cudaMalloc(&E.d_obs_hb, sizeof(unsigned long long) * nbins * E.R));
    PS_CK(cudaMalloc(&E.d_obs_ht, sizeof(unsigned long long) * nbins * E.R));
    PS_CK(cudaMalloc(&E.d_obs_ring, sizeof(double) * 3 * lags * nc));
    PS_CK(cudaMalloc(&E.d_obs_msd, sizeof(double) * 6 * lags * nc));
    PS_CK(cudaMalloc(&E.d_obs_msdn, sizeof(unsigned long long) * lags * nc));
    PS_CK(cudaMemset(E.d_obs_acc, 0, sizeof(double) * OBS_K * E.ntot));
    PS_CK(cudaMemset(E.d_obs_hasprev, 0, sizeof(int) * ns));
    PS_CK(cudaMemset(E.d_obs_hb, 0, sizeof(unsigned long long) * nbins * E.R));
    PS_CK(cudaMemset(E.d_obs_ht, 0, sizeof(unsigned long long) * nbins * E.R));
    PS_CK(cudaMemset(E.d_obs_msd, 0, sizeof(double) * 6 * lags * nc));
    PS_CK(cudaMemset(E.d_obs_msdn, 0, sizeof(unsigned long long) * lags * nc));
    E.obs_nbins = nbins; E.obs_bmax = bond_max; E.obs_tmax = trap_max; E.obs_lags = lags; E.obs_n = 0;
    return PS_OK;
}

int obs_sample(Engine &E, cudaStream_t st)
{
    if (!E.d_obs_acc) { set_error("ps_observe: call ps_obs_reset first"); return PS_ERR_STATE; }
    int thr = 128;
    ps_launch(k_observe, (unsigned)((E.ntot + thr - 1) / thr), thr, 0, st,
            E.ntot, E.d_bead_offs, E.R, E.d_segs, E.d_x, E.d_xpos0, E.d_bond_ptr, E.d_bond_nbr, E.d_obs_acc, E.d_obs_prev,
            E.d_obs_hasprev, E.d_obs_hb, E.d_obs_ht, E.obs_nbins, E.obs_bmax, E.obs_tmax);
    if (E.ncoll)
        ps_launch(k_observe_msd, (unsigned)((E.ncoll + thr - 1) / thr), thr, 0, st,
                E.ncoll, E.d_coll_rep, E.d_segs, E.d_x, E.d_obs_ring, E.d_obs_msd, E.d_obs_msdn, E.obs_lags, E.obs_n);
    PS_CK(cudaGetLastError());
    E.obs_n++;
    return PS_OK;
}

int obs_read(Engine &E, ps_obs_out *out, cudaStream_t st)
{
    if (!E.d_obs_acc) { set_error("ps_obs_read: call ps_obs_reset first"); return PS_ERR_STATE; }
    PS_CK(cudaStreamSynchronize(st));
    const int R = E.R, nb = E.obs_nbins, L = E.obs_lags;
    std::vector<double> acc((size_t)OBS_K * E.ntot);
    PS_CK(cudaMemcpy(acc.data(), E.d_obs_acc, sizeof(double) * acc.size(), cudaMemcpyDeviceToHost));
    for (int r = 0; r < R; r++) {
        const Seg &s = E.segs[r];
        double bsum[10] = {0}, tsum[9] = {0};
        for (int i = 0; i < s.Np; i++) {
            const double *a = acc.data() + (size_t)OBS_K * (s.bead_off + i);
            for (int k = 0; k < 10; k++) bsum[k] += a[k];
            for (int k = 0; k < 9; k++) tsum[k] += a[10 + k];
        }
        if (out->bond) for (int k = 0; k < 10; k++) out->bond[10L * r + k] = bsum[k];
        if (out->trap) for (int k = 0; k < 9; k++) out->trap[9L * r + k] = tsum[k];
    }
    if (out->bond_hist)
        PS_CK(cudaMemcpy(out->bond_hist, E.d_obs_hb, sizeof(unsigned long long) * nb * R, cudaMemcpyDeviceToHost));
    if (out->trap_hist)
        PS_CK(cudaMemcpy(out->trap_hist, E.d_obs_ht, sizeof(unsigned long long) * nb * R, cudaMemcpyDeviceToHost));
    if ((out->msd || out->msd_count) && E.ncoll) {
        std::vector<double> m((size_t)6 * L * E.ncoll);
        std::vector<unsigned long long> n((size_t)L * E.ncoll);
        PS_CK(cudaMemcpy(m.data(), E.d_obs_msd, sizeof(double) * m.size(), cudaMemcpyDeviceToHost));
        PS_CK(cudaMemcpy(n.data(), E.d_obs_msdn, sizeof(unsigned long long) * n.size(), cudaMemcpyDeviceToHost));
        for (int r = 0; r < R; r++) {
            const Seg &s = E.segs[r];
            for (int l = 0; l < L; l++) {
                double t[6] = {0};
                unsigned long long cnt = 0;
                for (int c = 0; c < s.Nc; c++) {
                    const long cc = s.coll_off + c;
                    for (int k = 0; k < 6; k++) t[k] += m[6 * ((size_t)L * cc + l) + k];
                    cnt += n[(size_t)L * cc + l];
                }
                if (out->msd) for (int k = 0; k < 6; k++) out->msd[6 * ((long)L * r + l) + k] = t[k];
                if (out->msd_count) out->msd_count[(long)L * r + l] = cnt;
            }
        }
    } else {
        if (out->msd) for (long k = 0; k < 6L * L * R; k++) out->msd[k] = 0.0;
        if (out->msd_count) for (long k = 0; k < (long)L * R; k++) out->msd_count[k] = 0;
    }
    return PS_OK;
}

}  // namespace ps
