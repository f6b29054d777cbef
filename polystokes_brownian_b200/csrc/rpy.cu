// rpy.cu -- matrix-free grand-mobility and saddle-operator apply.
//
// y = M u over every replica of the batch, with M the grand mobility that the
// reference assembles densely into A's top-left block (mm_HI, mob.cpp:843-1160)
// or applies as the arrowhead shell (matfree_A.cpp:38-80).  Pair tensors are
// recomputed on the fly from the positions (O(N) memory); the O(N^2) loops are
// thread-per-row with column tiles staged in shared memory, so every lane of a
// warp reads the same column entry (a shared-memory broadcast).  Columns are
// split into chunks across blockIdx.y (AA_CHUNK_COLS monomer or BB_CHUNK_COLS
// colloid columns per chunk, so the chunking of a replica depends on its own
// size only); chunk partials are summed in fixed order by k_combine, so results
// are deterministic and bit-identical whatever else shares the batch.
#include <algorithm>
#include "ps_internal.h"
#include "ps_kernels.h"
#include "ps_reduce.cuh"

namespace ps {

constexpr int RPY_THREADS = 128;

// Compensated accumulator: plain for FP64, Kahan across column tiles for FP32.
template <class T> struct Acc {
    T s, c;
    __device__ __forceinline__ void zero() { s = T(0); c = T(0); }
    __device__ __forceinline__ void add(T v) { s += v; }
    __device__ __forceinline__ T get() const { return s; }
};
template <> struct Acc<float> {
    float s, c;
    __device__ __forceinline__ void zero() { s = 0.f; c = 0.f; }
    __device__ __forceinline__ void add(float v) {
        float y = v - c, t = s + y;
        c = (t - s) - y;
        s = t;
    }
    __device__ __forceinline__ float get() const { return s; }
};

// ---------------------------------------------------------------------------
// AA in FP32 with packed FP32x2 arithmetic (sm_100 FFMA2/FADD2/FMUL2), column
// pairs in the two lanes: a thread owns rows i and i + 64 of a 128-row tile,
// each held as a broadcast pair (loop-invariant), and advances both against
// columns (j, j + 1) per step, four pairs per step.  Shared columns are stored
// pairwise, so the loads deliver every operand pair as it is consumed, with no
// per-column broadcast: sXY (-x_j, -x_j+1, -y_j, -y_j+1), sZU (-z_j, -z_j+1,
// u0_j, u0_j+1), sUU (u1_j, u1_j+1, u2_j, u2_j+1); sLA (lo x_j, x_j+1, lo y_j,
// y_j+1) and sLB (lo z_j, z_j+1, chain_j, chain_j+1) are read inside the exact
// radius or by CHECK tiles.  An odd tile is padded with a column at 1e18
// carrying u = 0.  Each row's two lane sums are added once per column tile,
// then Kahan-summed across tiles.
//
// Positions are hi + lo floats.  Separations start as d = hi_i - hi_j, whose
// error is at most 2^-23 X for a replica whose coordinates stay below X in
// magnitude; within the replica's exact radius (r <= max(2.1 beta, X / 16), so
// the hi-only relative error stays below 2^-19 where it is used) the warp adds
// the low parts, d = (hi_i - hi_j) + (lo_i - lo_j), the same rounding as a full
// hi + lo difference.  Self pairs and skipped same-chain pairs get rinv = 0,
// which zeroes their contribution without a branch; the near-overlap form
// (r <= 2 beta) lies inside the exact radius.  Far form in factored scalars:
// y = ri (c + d ri^2), (x - y)/r^2 = ri^3 (a + b ri^2), a = c0 - c2, b = c1 - c3,
// c = c2, d = c3; the near form (r^2 <= (2 beta)^2) overwrites both.
constexpr int AAF_THREADS = 64;
constexpr float AAC_PAD = 1e18f;

__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }

__device__ __forceinline__ void aa_near_lane(bool n, float r2, float ri, float ri2, float nx0, float nx1, float ny0,
                                             float ny1, float &yv, float &g)
{
    if (n) {
        const float r = r2 * ri, x = nx0 + nx1 * r;
        yv = ny0 + ny1 * r;
        g = (x - yv) * ri2;
    }
}

template <bool CHECK, bool REF>
__device__ __forceinline__ void aa_f2_cols(const float4 *__restrict__ sXY, const float4 *__restrict__ sZU,
                                           const float4 *__restrict__ sUU, const float4 *__restrict__ sLA,
                                           const float4 *__restrict__ sLB, int jt, int np, int iA, int iB,
                                           bool chain_hi, float wA, float wB, float2 ax, float2 ay, float2 az,
                                           float2 bx, float2 by, float2 bz, const float4 *__restrict__ plo, int bA,
                                           int bB, float2 fa, float2 fb, float2 fc, float2 fd, const Seg &sg,
                                           float te2, const double4 *__restrict__ p64, float2 (&t)[6])
{
#pragma unroll 1
    for (int k = 0; k < np; k++) {
        const float4 XY = sXY[k], ZU = sZU[k], UU = sUU[k];
        float2 dA[3], dB[3];
        dA[0] = __fadd2_rn(ax, make_float2(XY.x, XY.y)); dA[1] = __fadd2_rn(ay, make_float2(XY.z, XY.w));
        dA[2] = __fadd2_rn(az, make_float2(ZU.x, ZU.y));
        dB[0] = __fadd2_rn(bx, make_float2(XY.x, XY.y)); dB[1] = __fadd2_rn(by, make_float2(XY.z, XY.w));
        dB[2] = __fadd2_rn(bz, make_float2(ZU.x, ZU.y));
        float2 r2A = __ffma2_rn(dA[2], dA[2], __ffma2_rn(dA[1], dA[1], __fmul2_rn(dA[0], dA[0])));
        float2 r2B = __ffma2_rn(dB[2], dB[2], __ffma2_rn(dB[1], dB[1], __fmul2_rn(dB[0], dB[0])));
        bool eA0 = false, eA1 = false, eB0 = false, eB1 = false;
        if constexpr (CHECK) {
            const int j = jt + 2 * k;
            const float4 LB = sLB[k];
            eA0 = (j == iA) || (chain_hi && wA == LB.z);
            eA1 = (j + 1 == iA) || (chain_hi && wA == LB.w);
            eB0 = (j == iB) || (chain_hi && wB == LB.z);
            eB1 = (j + 1 == iB) || (chain_hi && wB == LB.w);
        }
        const bool inner = __any_sync(0xffffffffu, fminf(fminf(r2A.x, r2A.y), fminf(r2B.x, r2B.y)) <= te2);
        if (inner) {
            const float4 LA = sLA[k], LB = sLB[k], RA = __ldg(plo + bA), RB = __ldg(plo + bB);
            const float2 cx = make_float2(-LA.x, -LA.y), cy = make_float2(-LA.z, -LA.w), cz = make_float2(-LB.x, -LB.y);
            dA[0] = __fadd2_rn(dA[0], __fadd2_rn(f2(RA.x), cx)); dA[1] = __fadd2_rn(dA[1], __fadd2_rn(f2(RA.y), cy));
            dA[2] = __fadd2_rn(dA[2], __fadd2_rn(f2(RA.z), cz));
            dB[0] = __fadd2_rn(dB[0], __fadd2_rn(f2(RB.x), cx)); dB[1] = __fadd2_rn(dB[1], __fadd2_rn(f2(RB.y), cy));
            dB[2] = __fadd2_rn(dB[2], __fadd2_rn(f2(RB.z), cz));
            r2A = __ffma2_rn(dA[2], dA[2], __ffma2_rn(dA[1], dA[1], __fmul2_rn(dA[0], dA[0])));
            r2B = __ffma2_rn(dB[2], dB[2], __ffma2_rn(dB[1], dB[1], __fmul2_rn(dB[0], dB[0])));
        }
        const float2 riA = make_float2(eA0 ? 0.f : rsqrtf(r2A.x), eA1 ? 0.f : rsqrtf(r2A.y));
        const float2 riB = make_float2(eB0 ? 0.f : rsqrtf(r2B.x), eB1 ? 0.f : rsqrtf(r2B.y));
        const float2 ri2A = __fmul2_rn(riA, riA), ri2B = __fmul2_rn(riB, riB);
        float2 yA = __fmul2_rn(__ffma2_rn(fd, ri2A, fc), riA), yB = __fmul2_rn(__ffma2_rn(fd, ri2B, fc), riB);
        float2 gA = __fmul2_rn(__ffma2_rn(fb, ri2A, fa), __fmul2_rn(ri2A, riA));
        float2 gB = __fmul2_rn(__ffma2_rn(fb, ri2B, fa), __fmul2_rn(ri2B, riB));
        if (inner) {
            const float tb2 = (float)(4.0 * sg.beta * sg.beta);
            const float nx0 = sg.aa_c[4], nx1 = sg.aa_c[5], ny0 = sg.aa_c[6], ny1 = sg.aa_c[7];
            bool nA0 = !eA0 && r2A.x <= tb2, nA1 = !eA1 && r2A.y <= tb2, nB0 = !eB0 && r2B.x <= tb2,
                 nB1 = !eB1 && r2B.y <= tb2;
            if constexpr (REF) {
                // the reference's scalars jump at 2 beta (chain bonds often sit there): within a
                // band of the FP32 test its own FP64 distance decides (RPY is continuous there)
                const double tb = 2.0 * sg.beta;
                const int j = jt + 2 * k;
                auto decide = [&](bool e, float r2, int bi, int jj, bool &n) {
                    if (e || fabsf(r2 - tb2) > 1e-5f * tb2) return;
                    const double4 P = p64[bi], Q = p64[sg.bead_off + jj];
                    n = !(ref_pair_dist(P.x - Q.x, P.y - Q.y, P.z - Q.z) > tb);
                };
                decide(eA0, r2A.x, bA, j, nA0); decide(eA1, r2A.y, bA, j + 1, nA1);
                decide(eB0, r2B.x, bB, j, nB0); decide(eB1, r2B.y, bB, j + 1, nB1);
            }
            aa_near_lane(nA0, r2A.x, riA.x, ri2A.x, nx0, nx1, ny0, ny1, yA.x, gA.x);
            aa_near_lane(nA1, r2A.y, riA.y, ri2A.y, nx0, nx1, ny0, ny1, yA.y, gA.y);
            aa_near_lane(nB0, r2B.x, riB.x, ri2B.x, nx0, nx1, ny0, ny1, yB.x, gB.x);
            aa_near_lane(nB1, r2B.y, riB.y, ri2B.y, nx0, nx1, ny0, ny1, yB.y, gB.y);
        }
        // mob_a u = y u + (x - y)(d.u) d / r^2
        const float2 u0 = make_float2(ZU.z, ZU.w), u1 = make_float2(UU.x, UU.y), u2 = make_float2(UU.z, UU.w);
        const float2 hA = __fmul2_rn(gA, __ffma2_rn(dA[2], u2, __ffma2_rn(dA[1], u1, __fmul2_rn(dA[0], u0))));
        const float2 hB = __fmul2_rn(gB, __ffma2_rn(dB[2], u2, __ffma2_rn(dB[1], u1, __fmul2_rn(dB[0], u0))));
        t[0] = __ffma2_rn(hA, dA[0], __ffma2_rn(yA, u0, t[0]));
        t[1] = __ffma2_rn(hA, dA[1], __ffma2_rn(yA, u1, t[1]));
        t[2] = __ffma2_rn(hA, dA[2], __ffma2_rn(yA, u2, t[2]));
        t[3] = __ffma2_rn(hB, dB[0], __ffma2_rn(yB, u0, t[3]));
        t[4] = __ffma2_rn(hB, dB[1], __ffma2_rn(yB, u1, t[4]));
        t[5] = __ffma2_rn(hB, dB[2], __ffma2_rn(yB, u2, t[5]));
    }
}

template <bool REF>
__global__ void __launch_bounds__(AAF_THREADS, 12)
k_rpy_aa_f2(const Seg *__restrict__ segs, const Tile *__restrict__ tiles, const float4 *__restrict__ pos,
            const float4 *__restrict__ plo, const float *__restrict__ aa_te2, const double4 *__restrict__ p64,
            const double *__restrict__ u, int in_top, double *__restrict__ part, long part_stride, int nchunk,
            const char *__restrict__ done, int done_stride)
{
    pdl_enter();
    if (done && *(const int *)(done + (long)tiles[blockIdx.x].rep * done_stride)) return;
    __shared__ float4 sXY[64], sZU[64], sUU[64], sLA[64], sLB[64];
    __shared__ float sK[12][AAF_THREADS];     // Kahan sums [0, 6) and compensations [6, 12), thread-private
    const Tile tl = tiles[blockIdx.x];
    const Seg &sg = segs[tl.rep];
    const int c = blockIdx.y;
    nchunk = sg.nch_aa;               // per-replica chunk count: a function of Nm alone
    if (c >= nchunk) return;
    // one instance per pair-scalar family: the reference's scalars take the FP64 branch decision
    if ((sg.aa_mode == PS_AA_REFERENCE) != REF) return;
    const int Nm = sg.Nm, tid = threadIdx.x;
    const int j0 = (int)((long)Nm * c / nchunk), j1 = (int)((long)Nm * (c + 1) / nchunk);
    const int iA = tl.row0 + tid, iB = iA + AAF_THREADS;
    const bool actA = tid < tl.nrow, actB = tid + AAF_THREADS < tl.nrow;
    const int uoff = in_top ? sg.top_off : sg.vec_off;
    const int bA = sg.bead_off + (actA ? iA : tl.row0), bB = sg.bead_off + (actB ? iB : tl.row0);
    const float4 PA = pos[bA], PB = pos[bB];
    const float2 ax = f2(PA.x), ay = f2(PA.y), az = f2(PA.z), bx = f2(PB.x), by = f2(PB.y), bz = f2(PB.z);
    const bool chain_hi = sg.chain_HI != 0;
    const float2 fa = f2(sg.aa_c[0] - sg.aa_c[2]), fb = f2(sg.aa_c[1] - sg.aa_c[3]);
    const float2 fc = f2(sg.aa_c[2]), fd = f2(sg.aa_c[3]);
    const float te2 = aa_te2[tl.rep];
#pragma unroll
    for (int q = 0; q < 12; q++) sK[q][tid] = 0.f;
    for (int jt = j0; jt < j1; jt += 128) {
        const int nj = min(128, j1 - jt), np = (nj + 1) >> 1;
        __syncthreads();
        // one column pair per thread (64 pairs = 128 columns)
        if (tid < np) {
            float4 A[2], B[2];
            float v[2][3];
            for (int h = 0; h < 2; h++) {
                const int jl = 2 * tid + h, j = jt + jl;
                if (jl < nj) {
                    A[h] = pos[sg.bead_off + j]; B[h] = plo[sg.bead_off + j];
                    for (int a = 0; a < 3; a++) v[h][a] = (float)u[uoff + 3 * j + a];
                } else {
                    A[h] = make_float4(AAC_PAD, AAC_PAD, AAC_PAD, __int_as_float(0x7fc00000));
                    B[h] = make_float4(0.f, 0.f, 0.f, 0.f);
                    v[h][0] = v[h][1] = v[h][2] = 0.f;
                }
            }
            sXY[tid] = make_float4(-A[0].x, -A[1].x, -A[0].y, -A[1].y);
            sZU[tid] = make_float4(-A[0].z, -A[1].z, v[0][0], v[1][0]);
            sUU[tid] = make_float4(v[0][1], v[1][1], v[0][2], v[1][2]);
            sLA[tid] = make_float4(B[0].x, B[1].x, B[0].y, B[1].y);
            sLB[tid] = make_float4(B[0].z, B[1].z, A[0].w, A[1].w);
        }
        __syncthreads();
        float2 t[6] = {f2(0.f), f2(0.f), f2(0.f), f2(0.f), f2(0.f), f2(0.f)};
        // rows of this tile are [row0, row0 + 128): only overlapping column tiles hold self pairs
        const bool check = chain_hi || (jt < tl.row0 + 2 * AAF_THREADS && jt + nj > tl.row0);
        if (check)
            aa_f2_cols<true, REF>(sXY, sZU, sUU, sLA, sLB, jt, np, iA, iB, chain_hi, PA.w, PB.w, ax, ay, az, bx, by,
                                  bz, plo, bA, bB, fa, fb, fc, fd, sg, te2, p64, t);
        else
            aa_f2_cols<false, REF>(sXY, sZU, sUU, sLA, sLB, jt, np, iA, iB, chain_hi, PA.w, PB.w, ax, ay, az, bx, by,
                                   bz, plo, bA, bB, fa, fb, fc, fd, sg, te2, p64, t);
        // fold the two column lanes, then Kahan across column tiles
#pragma unroll
        for (int q = 0; q < 6; q++) {
            const float x = t[q].x + t[q].y;
            const float sq = sK[q][tid], kq = sK[6 + q][tid];
            const float yy = x - kq, tt = sq + yy;
            sK[6 + q][tid] = (tt - sq) - yy;
            sK[q][tid] = tt;
        }
    }
    double *o = part + (long)c * part_stride + sg.top_off;
    if (actA) { o[3 * iA] = sK[0][tid]; o[3 * iA + 1] = sK[1][tid]; o[3 * iA + 2] = sK[2][tid]; }
    if (actB) { o[3 * iB] = sK[3][tid]; o[3 * iB + 1] = sK[4][tid]; o[3 * iB + 2] = sK[5][tid]; }
}

// ---------------------------------------------------------------------------
// AA in FP64, two rows per thread.  A thread owns rows i and i + 64 of a 128-row
// tile and sweeps 128-column tiles staged in shared memory as (x, y, z, chain)
// and (u0, u1, u2, 0) double4 pairs, so each column's loads serve both rows.
// Reciprocal square root: a single-precision seed (the float image taken with integer
// operations) refined by the second-order
// term of the binomial series (1 - e)^(-1/2) = 1 + e/2 + 3 e^2 / 8 + O(e^3),
// e = 1 - a y0^2 (Householder's iteration of order 2 for f(y) = y^-2 - a): from
// a seed accurate to 2^-22 the truncation is below 2^-64, so the result is
// within a couple of ulp of the correctly rounded value (checked against CUDA's
// rsqrt by ps_rsqrt_check).  Self pairs and skipped same-chain pairs get
// ri = 0, which zeroes their contribution; the near form (r <= 2 beta) is taken
// under a warp vote.  Far form in factored scalars: y = ri (c + d ri^2),
// (x - y) / r^2 = ri^3 (a + b ri^2), a = c0 - c2, b = c1 - c3, c = c2, d = c3.
constexpr int AAD_THREADS = 64;

// Single-precision image of a positive double in [2^-126, 2^128) by exponent re-bias and
// mantissa truncation (relative error below 2^-23), with integer operations only, so the
// FP64 pipe is left to the arithmetic; seed_as_double widens a positive normal float exactly.
__device__ __forceinline__ float trunc_to_float(double a)
{
    const int hi = __double2hiint(a), lo = __double2loint(a);
    return __int_as_float(((hi - (896 << 20)) << 3) | (int)((unsigned)lo >> 29));
}
__device__ __forceinline__ double seed_as_double(float f)
{
    const int b = __float_as_int(f);
    return __hiloint2double((b >> 3) + (896 << 20), b << 29);
}

__device__ __forceinline__ double rsqrt_seeded(double a, float af)
{
    const double y = seed_as_double(rsqrtf(af));
    const double e = fma(-(a * y), y, 1.0);
    return fma(y * e, fma(0.375, e, 0.5), y);
}
__device__ __forceinline__ double rsqrt_seeded(double a) { return rsqrt_seeded(a, trunc_to_float(a)); }

template <bool CHECK>
__device__ __forceinline__ void aa_d2_cols(const double4 *__restrict__ sP, const double4 *__restrict__ sU, int jt,
                                           int nj, int iA, int iB, bool chain_hi, double4 PA, double4 PB, double ca,
                                           double cb, double cc, double cd, double tb, float tb2f, double n0,
                                           double n1, double n2, double n3, double (&t)[6])
{
#pragma unroll 1
    for (int k = 0; k < nj; k++) {
        const double4 P = sP[k], U = sU[k];
        const double ax = PA.x - P.x, ay = PA.y - P.y, az = PA.z - P.z;
        const double bx = PB.x - P.x, by = PB.y - P.y, bz = PB.z - P.z;
        const double r2A = fma(az, az, fma(ay, ay, ax * ax));
        const double r2B = fma(bz, bz, fma(by, by, bx * bx));
        bool sA = false, sB = false;
        if constexpr (CHECK) {
            const int j = jt + k;
            sA = (j == iA) || (chain_hi && PA.w == P.w);
            sB = (j == iB) || (chain_hi && PB.w == P.w);
        }
        const float fA = trunc_to_float(r2A), fB = trunc_to_float(r2B);
        const double riA = sA ? 0.0 : rsqrt_seeded(r2A, fA), riB = sB ? 0.0 : rsqrt_seeded(r2B, fB);
        const double qA = riA * riA, qB = riB * riB;
        double yA = riA * fma(cd, qA, cc), yB = riB * fma(cd, qB, cc);
        double gA = (qA * riA) * fma(cb, qA, ca), gB = (qB * riB) * fma(cb, qB, ca);
        // candidates for the near form (a single-precision test with a 1e-6 margin, off the FP64
        // pipe); the reference's own distance decides within the band
        const bool nA = !sA && fA <= tb2f, nB = !sB && fB <= tb2f;
        if (__any_sync(0xffffffffu, nA || nB)) {
            if (nA) {
                const double r = ref_pair_dist(ax, ay, az);
                if (!(r > tb)) { const double ri = 1.0 / r, x = fma(n1, r, n0); yA = fma(n3, r, n2); gA = (x - yA) * ri * ri; }
            }
            if (nB) {
                const double r = ref_pair_dist(bx, by, bz);
                if (!(r > tb)) { const double ri = 1.0 / r, x = fma(n1, r, n0); yB = fma(n3, r, n2); gB = (x - yB) * ri * ri; }
            }
        }
        const double hA = gA * fma(az, U.z, fma(ay, U.y, ax * U.x));
        const double hB = gB * fma(bz, U.z, fma(by, U.y, bx * U.x));
        t[0] = fma(hA, ax, fma(yA, U.x, t[0]));
        t[1] = fma(hA, ay, fma(yA, U.y, t[1]));
        t[2] = fma(hA, az, fma(yA, U.z, t[2]));
        t[3] = fma(hB, bx, fma(yB, U.x, t[3]));
        t[4] = fma(hB, by, fma(yB, U.y, t[4]));
        t[5] = fma(hB, bz, fma(yB, U.z, t[5]));
    }
}

__global__ void __launch_bounds__(AAD_THREADS, 8)
k_rpy_aa_d2(const Seg *__restrict__ segs, const Tile *__restrict__ tiles, const double4 *__restrict__ pos,
            const double *__restrict__ u, int in_top, double *__restrict__ part, long part_stride, int nchunk,
            const char *__restrict__ done, int done_stride)
{
    pdl_enter();
    if (done && *(const int *)(done + (long)tiles[blockIdx.x].rep * done_stride)) return;
    __shared__ double4 sP[128], sU[128];
    const Tile tl = tiles[blockIdx.x];
    const Seg &sg = segs[tl.rep];
    const int c = blockIdx.y;
    nchunk = sg.nch_aa;               // per-replica chunk count: a function of Nm alone
    if (c >= nchunk) return;
    const int Nm = sg.Nm, tid = threadIdx.x;
    const int j0 = (int)((long)Nm * c / nchunk), j1 = (int)((long)Nm * (c + 1) / nchunk);
    const int iA = tl.row0 + tid, iB = iA + AAD_THREADS;
    const bool actA = tid < tl.nrow, actB = tid + AAD_THREADS < tl.nrow;
    const int uoff = in_top ? sg.top_off : sg.vec_off;
    const double4 PA = pos[sg.bead_off + (actA ? iA : tl.row0)], PB = pos[sg.bead_off + (actB ? iB : tl.row0)];
    const bool chain_hi = sg.chain_HI != 0;
    double c0, c1, c2, c3, n0, n1, n2, n3;
    if (sg.aa_mode == PS_AA_RPY) {
        const double b = sg.beta, b2 = b * b;
        c0 = 1.5; c1 = -b2; c2 = 0.75; c3 = 0.5 * b2;
        n0 = 1.0 / b; n1 = -0.1875 / b2; n2 = 1.0 / b; n3 = -0.28125 / b2;
    } else {
        c0 = 0.375; c1 = -2.0; c2 = 0.75; c3 = -0.5;
        n0 = -1.0; n1 = 0.375; n2 = 1.0; n3 = -0.28125;
    }
    const double tb = 2.0 * sg.beta, ca = c0 - c2, cb = c1 - c3;
    const float tb2f = (float)(tb * tb * (1.0 + 1e-6));
    double a[6] = {0, 0, 0, 0, 0, 0};
    for (int jt = j0; jt < j1; jt += 128) {
        const int nj = min(128, j1 - jt);
        __syncthreads();
        for (int h = 0; h < 2; h++) {
            const int jl = tid + h * AAD_THREADS;
            if (jl < nj) {
                const int j = jt + jl;
                sP[jl] = pos[sg.bead_off + j];
                sU[jl] = make_double4(u[uoff + 3 * j], u[uoff + 3 * j + 1], u[uoff + 3 * j + 2], 0.0);
            }
        }
        __syncthreads();
        double t[6] = {0, 0, 0, 0, 0, 0};
        // rows of this tile are [row0, row0 + 128): only overlapping column tiles hold self pairs
        const bool check = chain_hi || (jt < tl.row0 + 2 * AAD_THREADS && jt + nj > tl.row0);
        if (check)
            aa_d2_cols<true>(sP, sU, jt, nj, iA, iB, chain_hi, PA, PB, ca, cb, c2, c3, tb, tb2f, n0, n1, n2, n3, t);
        else
            aa_d2_cols<false>(sP, sU, jt, nj, iA, iB, chain_hi, PA, PB, ca, cb, c2, c3, tb, tb2f, n0, n1, n2, n3, t);
#pragma unroll
        for (int q = 0; q < 6; q++) a[q] += t[q];
    }
    double *o = part + (long)c * part_stride + sg.top_off;
    if (actA) { o[3 * iA] = a[0]; o[3 * iA + 1] = a[1]; o[3 * iA + 2] = a[2]; }
    if (actB) { o[3 * iB] = a[3]; o[3 * iB + 1] = a[4]; o[3 * iB + 2] = a[5]; }
}

// max |own - CUDA| / ulp(CUDA) of the reciprocal square root over a[0..n)
__global__ void k_rsqrt_check(long n, const double *__restrict__ a, unsigned long long *__restrict__ worst)
{
    pdl_enter();
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double ref = rsqrt(a[i]), own = rsqrt_seeded(a[i]);
    long long d = __double_as_longlong(own) - __double_as_longlong(ref);
    atomicMax(worst, (unsigned long long)(d < 0 ? -d : d));
}

// ---------------------------------------------------------------------------
// AB/BA: monomer rows x colloids of the same replica.  Monomer outputs go to
// part_m (no chunking: Nc is small whenever Nm > 0); each colloid's output from
// this tile's monomers is block-reduced into part_ba (one 11-vector per
// (monomer tile, colloid)).  tab: per-replica 3x3 translational block
// (reference mode, row-major mob_a[a][b]); ignored in RPY mode.
template <class T>
__global__ void __launch_bounds__(RPY_THREADS)
k_rpy_ab(const Seg *__restrict__ segs, const Tile *__restrict__ tiles, const typename V4<T>::t *__restrict__ pos,
         const float4 *__restrict__ plo, const double *__restrict__ u, int in_top, const double *__restrict__ tab,
         double *__restrict__ part_m, double *__restrict__ part_ba, const char *__restrict__ done, int done_stride)
{
    pdl_enter();
    if (done && *(const int *)(done + (long)tiles[blockIdx.x].rep * done_stride)) return;
    typedef typename V4<T>::t P4;
    constexpr bool F32 = sizeof(T) == 4;
    __shared__ T red[RPY_THREADS / 32][12];
    const Tile tl = tiles[blockIdx.x];
    const Seg &sg = segs[tl.rep];
    const int i = tl.row0 + threadIdx.x;
    const bool active = threadIdx.x < tl.nrow;
    const int uoff = in_top ? sg.top_off : sg.vec_off;
    const int Nm = sg.Nm, Nc = sg.Nc;
    P4 pm = pos[sg.bead_off + (active ? i : tl.row0)];
    T fm[3];
    for (int a = 0; a < 3; a++) fm[a] = active ? (T)u[uoff + 3 * i + a] : T(0);
    T Tm[9];
    const int mode = sg.ab_mode;
    const bool shell = !sg.mm_HI;
    for (int a = 0; a < 9; a++) Tm[a] = (T)tab[9 * tl.rep + a];
    const T beta2 = T(sg.beta * sg.beta);
    T om0 = 0, om1 = 0, om2 = 0;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int cc = 0; cc < Nc; cc++) {
        P4 pc = pos[sg.bead_off + Nm + cc];
        T Fc[3], Tc[3], Sc[5];
        for (int a = 0; a < 3; a++) {
            Fc[a] = (T)u[uoff + sg.nm3 + 3 * cc + a];
            Tc[a] = (T)u[uoff + sg.nm3 + sg.nc3 + 3 * cc + a];
        }
        for (int q = 0; q < 5; q++) Sc[q] = (T)u[uoff + sg.nm3nc6 + 5 * cc + q];
        T dx = pm.x - pc.x, dy = pm.y - pc.y, dz = pm.z - pc.z;
        if constexpr (F32) {
            float4 lm = plo[sg.bead_off + (active ? i : tl.row0)], lc = plo[sg.bead_off + Nm + cc];
            dx += lm.x - lc.x; dy += lm.y - lc.y; dz += lm.z - lc.z;
        }
        T r2 = dx * dx + dy * dy + dz * dz;
        T rinv = rsqrt_t<T>(r2);
        T e[3] = {dx * rinv, dy * rinv, dz * rinv};
        T yb, xg, yg;
        ab_scalars<T>(rinv, beta2, yb, xg, yg);
        T G[15];
        gt_flat<T>(e, xg, yg, G);
        T TT[9];
        if (mode == PS_AB_RPY || mode == PS_AB_RPY_REG) {
            T xa, ya;
            ab_trans_scalars<T>(r2 * rinv, rinv, T(sg.beta), mode == PS_AB_RPY_REG, xa, ya, yb);
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++) TT[a * 3 + b] = xa * e[a] * e[b] + ya * ((a == b ? T(1) : T(0)) - e[a] * e[b]);
        } else if (shell) {
            for (int a = 0; a < 9; a++) TT[a] = T(0);
        } else {
            for (int a = 0; a < 9; a++) TT[a] = Tm[a];
        }
        // monomer row: T F_c + B^T T_c + G S_c, B^T v = yb (e x v)
        T btx = yb * (e[1] * Tc[2] - e[2] * Tc[1]);
        T bty = yb * (e[2] * Tc[0] - e[0] * Tc[2]);
        T btz = yb * (e[0] * Tc[1] - e[1] * Tc[0]);
        T gs[3];
        for (int a = 0; a < 3; a++) {
            T acc = 0;
            for (int q = 0; q < 5; q++) acc += G[a * 5 + q] * Sc[q];
            gs[a] = acc;
        }
        om0 += TT[0] * Fc[0] + TT[1] * Fc[1] + TT[2] * Fc[2] + btx + gs[0];
        om1 += TT[3] * Fc[0] + TT[4] * Fc[1] + TT[5] * Fc[2] + bty + gs[1];
        om2 += TT[6] * Fc[0] + TT[7] * Fc[1] + TT[8] * Fc[2] + btz + gs[2];
        // colloid row from this monomer: [T^T F_m ; B F_m ; G^T F_m], B v = yb (v x e)
        T cv[11];
        for (int a = 0; a < 3; a++) cv[a] = TT[0 * 3 + a] * fm[0] + TT[1 * 3 + a] * fm[1] + TT[2 * 3 + a] * fm[2];
        cv[3] = yb * (fm[1] * e[2] - fm[2] * e[1]);
        cv[4] = yb * (fm[2] * e[0] - fm[0] * e[2]);
        cv[5] = yb * (fm[0] * e[1] - fm[1] * e[0]);
        for (int q = 0; q < 5; q++) cv[6 + q] = G[0 * 5 + q] * fm[0] + G[1 * 5 + q] * fm[1] + G[2 * 5 + q] * fm[2];
        if (!active)
            for (int q = 0; q < 11; q++) cv[q] = T(0);
        // deterministic block reduction
        for (int q = 0; q < 11; q++) {
            T v = cv[q];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            if (lane == 0) red[wid][q] = v;
        }
        __syncthreads();
        if (threadIdx.x < 11) {
            T v = 0;
            for (int w = 0; w < RPY_THREADS / 32; w++) v += red[w][threadIdx.x];
            part_ba[((long)sg.ba_off + (long)tl.mtile * Nc + cc) * 11 + threadIdx.x] = (double)v;
        }
        __syncthreads();
    }
    if (active) {
        double *o = part_m + sg.top_off + 3 * i;
        o[0] = (double)om0; o[1] = (double)om1; o[2] = (double)om2;
    }
}

// ---------------------------------------------------------------------------
// BB: colloid rows x colloid columns (FTS, 11 -> 11).  BB_SPLIT threads per row
// (a block is BB_SPLIT x RPY_THREADS threads): thread group h takes the tile
// columns h, h + BB_SPLIT, ...; the groups' sums are joined in group order in
// shared memory, so a replica of a thousand colloids fills the SMs without
// more chunk partials.
constexpr int BB_SPLIT = 4;
template <class T>
__global__ void __launch_bounds__(RPY_THREADS * BB_SPLIT)
k_rpy_bb(const Seg *__restrict__ segs, const Tile *__restrict__ tiles, const typename V4<T>::t *__restrict__ pos,
         const float4 *__restrict__ plo, const double *__restrict__ u, int in_top, double *__restrict__ part,
         long part_stride, int nchunk, const char *__restrict__ done, int done_stride)
{
    pdl_enter();
    if (done && *(const int *)(done + (long)tiles[blockIdx.x].rep * done_stride)) return;
    typedef typename V4<T>::t P4;
    constexpr bool F32 = sizeof(T) == 4;
    constexpr int CT = 64;
    __shared__ P4 sp[CT];
    __shared__ float4 sl[F32 ? CT : 1];
    __shared__ T su[CT * 11];
    __shared__ T sred[BB_SPLIT - 1][11][RPY_THREADS];
    const Tile tl = tiles[blockIdx.x];
    const Seg &sg = segs[tl.rep];
    const int c = blockIdx.y;
    nchunk = sg.nch_bb;
    if (c >= nchunk) return;
    const int row = threadIdx.x % RPY_THREADS, grp = threadIdx.x / RPY_THREADS;
    const int Nc = sg.Nc, Nm = sg.Nm;
    const int j0 = (int)((long)Nc * c / nchunk), j1 = (int)((long)Nc * (c + 1) / nchunk);
    const int i = tl.row0 + row;
    const bool active = row < tl.nrow;
    const int uoff = in_top ? sg.top_off : sg.vec_off;
    P4 pi = pos[sg.bead_off + Nm + (active ? i : tl.row0)];
    float4 li = make_float4(0.f, 0.f, 0.f, 0.f);
    if constexpr (F32) li = plo[sg.bead_off + Nm + (active ? i : tl.row0)];
    T out[11];   // accumulated over the chunk's column tiles in column order
    for (int q = 0; q < 11; q++) out[q] = T(0);
    for (int jt = j0; jt < j1; jt += CT) {
        int nj = min(CT, j1 - jt);
        __syncthreads();
        for (int t = threadIdx.x; t < nj * 11; t += blockDim.x) {
            int k = t / 11, q = t - 11 * k, j = jt + k;
            int idx = q < 3 ? sg.nm3 + 3 * j + q : (q < 6 ? sg.nm3 + sg.nc3 + 3 * j + (q - 3) : sg.nm3nc6 + 5 * j + (q - 6));
            su[t] = (T)u[uoff + idx];
        }
        if (threadIdx.x < nj) {
            sp[threadIdx.x] = pos[sg.bead_off + Nm + jt + threadIdx.x];
            if constexpr (F32) sl[threadIdx.x] = plo[sg.bead_off + Nm + jt + threadIdx.x];
        }
        __syncthreads();
        for (int k = grp; k < nj; k += BB_SPLIT) {
            int j = jt + k;
            if (j == i) continue;
            P4 pj = sp[k];
            bool lo = i < j;
            T dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
            if constexpr (F32) {
                float4 lj = sl[k];
                dx += li.x - lj.x; dy += li.y - lj.y; dz += li.z - lj.z;
            }
            if (!lo) { dx = -dx; dy = -dy; dz = -dz; }
            T r2 = dx * dx + dy * dy + dz * dz;
            T rinv = rsqrt_t<T>(r2);
            T e[3] = {dx * rinv, dy * rinv, dz * rinv};
            bb_apply<T>(e, r2 * rinv, rinv, lo, su + 11 * k, out);
        }
    }
    if (grp > 0)
        for (int q = 0; q < 11; q++) sred[grp - 1][q][row] = out[q];
    __syncthreads();
    if (grp == 0 && active) {
        for (int g = 0; g < BB_SPLIT - 1; g++)
            for (int q = 0; q < 11; q++) out[q] += sred[g][q][row];
        double *o = part + (long)c * part_stride + sg.top_off;
        for (int a = 0; a < 3; a++) {
            o[sg.nm3 + 3 * i + a] = (double)out[a];
            o[sg.nm3 + sg.nc3 + 3 * i + a] = (double)out[3 + a];
        }
        for (int q = 0; q < 5; q++) o[sg.nm3nc6 + 5 * i + q] = (double)out[6 + q];
    }
}

// ---------------------------------------------------------------------------
// Combine: self terms + pair partials (fixed order) + constraint blocks.
// mode 0: saddle   y = [[M, B], [B^T, -R_lub]] x   (vectors in saddle layout)
// mode 1: mobility y_top = M u                      (vectors in top layout)
__device__ __forceinline__ int find_rep(const int *__restrict__ offs, int R, long k)
{
    int lo = 0, hi = R;   // offs[R] = total
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (offs[mid] <= k) lo = mid; else hi = mid;
    }
    return lo;
}

// One block column per entry of the replica-aligned block table of the output
// layout (saddle vectors for mode 0, mobility vectors for mode 1), so the
// replica is known without a search and a converged replica's blocks leave at
// once; blockIdx.y splits an entry's span so that each thread sums one output
// (a single large replica otherwise leaves most SMs idle while every thread
// walks its chunk partials four times over).
__global__ void k_combine(const Seg *__restrict__ segs, RedTable T, int mode, const double *__restrict__ x,
                          const double *__restrict__ scale, const double *__restrict__ partAA, int nchAA,
                          const double *__restrict__ partAB, const double *__restrict__ partBB, int nchBB,
                          const double *__restrict__ partBA, const double *__restrict__ delta,
                          const double *__restrict__ lub_y, long part_stride, double *__restrict__ y,
                          const char *__restrict__ done, int done_stride)
{
    pdl_enter();
    const RBlk B = T.d_blk[blockIdx.x];
    const int r = B.rep;
    if (done && *(const int *)(done + (long)r * done_stride)) return;   // converged replica: skip
    const Seg &sg = segs[r];
    const int xo = mode == 0 ? sg.vec_off : sg.top_off;
    const double s = scale ? scale[r] : 1.0;
    for (int e = blockIdx.y * blockDim.x + threadIdx.x; e < B.len; e += blockDim.x * gridDim.y) {
        const long k = (long)B.start + e;
        const int i = (int)(k - xo);
        double v = 0.0;
        if (i < sg.nm3nc11) {
            if (i < sg.nm3) {
                v = sg.beta_inv * x[xo + i];
                if (sg.mm_HI) {
                    const int nc = nchAA ? sg.nch_aa : 0;
#pragma unroll 8
                    for (int c = 0; c < nc; c++) v += partAA[(long)c * part_stride + sg.top_off + i];
                }
                if (sg.Nc > 0) v += partAB[sg.top_off + i];
            } else {
                int j = i - sg.nm3;          // colloid-local DOF in [0, nc11)
                int cidx, q;                 // colloid index, component
                double self;
                if (j < sg.nc3) { cidx = j / 3; q = j % 3; self = x[xo + i]; }
                else if (j < sg.nc6) { cidx = (j - sg.nc3) / 3; q = 3 + (j - sg.nc3) % 3; self = 0.75 * x[xo + i]; }
                else {
                    cidx = (j - sg.nc6) / 5; q = 6 + (j - sg.nc6) % 5;
                    int sb = xo + sg.nm3nc6 + 5 * cidx, p = q - 6;
                    self = 1.8 * x[sb + p];
                    if (p == 0) self += 0.9 * x[sb + 4];
                    if (p == 4) self += 0.9 * x[sb + 0];
                }
                v = self;
                if (sg.Nc >= 2) {
#pragma unroll 8
                    for (int c = 0; c < sg.nch_bb; c++) v += partBB[(long)c * part_stride + sg.top_off + i];
                }
                if (sg.Nm > 0)
                    for (int t = 0; t < sg.n_mtiles; t++) v += partBA[((long)sg.ba_off + (long)t * sg.Nc + cidx) * 11 + q];
                if (sg.shell_schur) {
                    const double *D = delta + sg.schur_off + (long)j * sg.nc11;
                    double acc = 0.0;
                    for (int b = 0; b < sg.nc11; b++) acc += D[b] * x[xo + sg.nm3 + b];
                    v += acc;
                }
            }
            if (mode == 0 && i < sg.nm3nc6) v -= x[xo + sg.nm3nc11 + i];
        } else {
            int j = i - sg.nm3nc11;
            v = -x[xo + j];
            if (sg.lub_on && lub_y) v -= lub_y[sg.vel_off + j];
        }
        y[k] = s * v;
    }
}

// ---------------------------------------------------------------------------
// host launchers
template <class T>
void launch_pairs(Engine &E, const double *u, int in_top, cudaStream_t st, const char *done, int dstride, bool skip_aa)
{
    const typename V4<T>::t *pos = (const typename V4<T>::t *)(sizeof(T) == 8 ? (const void *)E.d_pos64 : (const void *)E.d_pos32);
    // the monomer-colloid and colloid-colloid kernels (a few microseconds each, few blocks)
    // run on the side stream beside the monomer kernel; they write their own partials,
    // and the join orders them before the combine
    const bool fork = E.side && E.n_aa_tiles && !skip_aa && (E.n_ab_tiles || E.n_bb_tiles);
    cudaStream_t ss = st;
    if (fork) {
        cudaEventRecord(E.ev_fork, st);
        cudaStreamWaitEvent(E.side, E.ev_fork, 0);
        ss = E.side;
    }
    if (E.n_aa_tiles && !skip_aa) {
        if constexpr (sizeof(T) == 4)
        {
            if (E.any_aa_rpy)
                ps_launch(k_rpy_aa_f2<false>, dim3(E.n_aa_tiles, E.nch_aa), AAF_THREADS, 0, st,
                        E.d_segs, E.d_aa_tiles, E.d_pos32, E.d_pos32lo, E.d_aa_te2, E.d_pos64, u, in_top, E.d_partAA,
                        E.part_stride, E.nch_aa, done, dstride);
            if (E.any_aa_ref)
                ps_launch(k_rpy_aa_f2<true>, dim3(E.n_aa_tiles, E.nch_aa), AAF_THREADS, 0, st,
                        E.d_segs, E.d_aa_tiles, E.d_pos32, E.d_pos32lo, E.d_aa_te2, E.d_pos64, u, in_top, E.d_partAA,
                        E.part_stride, E.nch_aa, done, dstride);
        }
        else
            ps_launch(k_rpy_aa_d2, dim3(E.n_aa_tiles, E.nch_aa), AAD_THREADS, 0, st,
                    E.d_segs, E.d_aa_tiles, E.d_pos64, u, in_top, E.d_partAA, E.part_stride, E.nch_aa, done, dstride);
    }
    if (E.n_ab_tiles)
        ps_launch(k_rpy_ab<T>, E.n_ab_tiles, RPY_THREADS, 0, ss, E.d_segs, E.d_ab_tiles, pos, E.d_pos32lo, u, in_top, E.d_tab, E.d_partAB,
                E.d_partBA, done, dstride);
    // colloid-colloid FTS blocks stay FP64 in the mixed form: near contact the
    // far-field FTS mobility is ill-conditioned and FP32 blocks leave a 1.2e-6
    // velocity error on a suspension at gap 0.01 (FP64: tracks rtol); they are
    // cheap wherever monomers carry the O(N^2) work
    if (E.n_bb_tiles)
        ps_launch(k_rpy_bb<double>, dim3(E.n_bb_tiles, E.nch_bb), RPY_THREADS * BB_SPLIT, 0, ss,
                E.d_segs, E.d_bb_tiles, E.d_pos64, E.d_pos32lo, u, in_top, E.d_partBB, E.part_stride, E.nch_bb, done, dstride);
    if (fork) {
        cudaEventRecord(E.ev_join, E.side);
        cudaStreamWaitEvent(st, E.ev_join, 0);
    }
}

void apply_operator(Engine &E, int mode, const double *x, double *y, const double *scale, bool fp32, cudaStream_t st,
                    const void *done, int done_stride, bool skip_aa)
{
    int in_top = mode == 1;
    const char *dn = (const char *)done;
    if (fp32) launch_pairs<float>(E, x, in_top, st, dn, done_stride, skip_aa);
    else launch_pairs<double>(E, x, in_top, st, dn, done_stride, skip_aa);
    const double *lub_y = nullptr;
    if (mode == 0 && E.any_lub) {
        lub_apply(E, x, E.d_luby, st);
        lub_y = E.d_luby;
    }
    const RedTable &T = mode == 0 ? E.red : E.red_top;
    ps_launch(k_combine, dim3((unsigned)T.nblk, RB_EPT), RB_THREADS, 0, st,
            E.d_segs, T, mode, x, scale, E.d_partAA, skip_aa ? 0 : E.nch_aa, E.d_partAB, E.d_partBB, E.nch_bb,
            E.d_partBA, E.d_delta, lub_y, E.part_stride, y, dn, done_stride);
}


int g_aa_chunk_cols = AA_CHUNK_COLS;

// re-chunk the monomer far field of a context: per-replica chunk counts, the
// grid extent and the partial buffer
int set_aa_chunking(Engine &E, int cols)
{
    E.nch_aa = 1;
    for (auto &s : E.segs) {
        s.nch_aa = std::max(1, (s.Nm + cols - 1) / cols);
        E.nch_aa = std::max(E.nch_aa, s.nch_aa);
    }
    PS_CK(cudaDeviceSynchronize());
    cudaFree(E.d_partAA);
    E.d_partAA = nullptr;
    PS_CK(cudaMalloc(&E.d_partAA, sizeof(double) * std::max<long>(E.ntop, 1) * E.nch_aa));
    PS_CK(cudaMemcpy(E.d_segs, E.segs.data(), sizeof(Seg) * E.segs.size(), cudaMemcpyHostToDevice));
    return PS_OK;
}

// ---------------------------------------------------------------------------
// diagnostics: average duration (CUDA events on `st`) of one far-field kernel
// which: 0 AA pair kernel, 1 AB/BA kernel, 2 BB kernel, 3 whole mobility apply
int time_pairs(Engine &E, int which, int reps, const double *u, double *ms, cudaStream_t st)
{
    bool fp32 = E.precision == PS_PREC_MIXED;
    const void *pos = fp32 ? (const void *)E.d_pos32 : (const void *)E.d_pos64;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    auto launch = [&]() {
        if (which == 0 && E.n_aa_tiles) {
            if (fp32) {
                if (E.any_aa_rpy) ps_launch(k_rpy_aa_f2<false>, dim3(E.n_aa_tiles, E.nch_aa), AAF_THREADS, 0, st, E.d_segs, E.d_aa_tiles, (const float4 *)pos, E.d_pos32lo, E.d_aa_te2, E.d_pos64, u, 1, E.d_partAA, E.part_stride, E.nch_aa, nullptr, 0);
                if (E.any_aa_ref) ps_launch(k_rpy_aa_f2<true>, dim3(E.n_aa_tiles, E.nch_aa), AAF_THREADS, 0, st, E.d_segs, E.d_aa_tiles, (const float4 *)pos, E.d_pos32lo, E.d_aa_te2, E.d_pos64, u, 1, E.d_partAA, E.part_stride, E.nch_aa, nullptr, 0);
            }
            else ps_launch(k_rpy_aa_d2, dim3(E.n_aa_tiles, E.nch_aa), AAD_THREADS, 0, st, E.d_segs, E.d_aa_tiles, E.d_pos64, u, 1, E.d_partAA, E.part_stride, E.nch_aa, nullptr, 0);
        } else if (which == 1 && E.n_ab_tiles) {
            if (fp32) ps_launch(k_rpy_ab<float>, E.n_ab_tiles, RPY_THREADS, 0, st, E.d_segs, E.d_ab_tiles, (const float4 *)pos, E.d_pos32lo, u, 1, E.d_tab, E.d_partAB, E.d_partBA, nullptr, 0);
            else ps_launch(k_rpy_ab<double>, E.n_ab_tiles, RPY_THREADS, 0, st, E.d_segs, E.d_ab_tiles, (const double4 *)pos, E.d_pos32lo, u, 1, E.d_tab, E.d_partAB, E.d_partBA, nullptr, 0);
        } else if (which == 2 && E.n_bb_tiles) {
            ps_launch(k_rpy_bb<double>, dim3(E.n_bb_tiles, E.nch_bb), RPY_THREADS * BB_SPLIT, 0, st, E.d_segs, E.d_bb_tiles, E.d_pos64, E.d_pos32lo, u, 1, E.d_partBB, E.part_stride, E.nch_bb, nullptr, 0);
        } else if (which == 3) {
            apply_operator(E, 1, u, E.d_tmp_top2, nullptr, fp32, st);
        }
    };
    launch();   // warm
    cudaEventRecord(a, st);
    for (int k = 0; k < reps; k++) launch();
    cudaEventRecord(b, st);
    cudaEventSynchronize(b);
    float t = 0;
    cudaEventElapsedTime(&t, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    *ms = reps > 0 ? (double)t / reps : 0.0;
    PS_CK(cudaGetLastError());
    return PS_OK;
}

// largest distance in ulp between rsqrt_seeded and CUDA's rsqrt over a device array
int rsqrt_check(const double *a, long n, unsigned long long *max_ulp, cudaStream_t st)
{
    unsigned long long *d = nullptr;
    PS_CK(cudaMallocAsync(&d, sizeof(unsigned long long), st));
    PS_CK(cudaMemsetAsync(d, 0, sizeof(unsigned long long), st));
    if (n > 0) ps_launch(k_rsqrt_check, (unsigned)((n + 255) / 256), 256, 0, st, n, a, d);
    PS_CK(cudaMemcpyAsync(max_ulp, d, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    PS_CK(cudaFreeAsync(d, st));
    PS_CK(cudaStreamSynchronize(st));
    return PS_OK;
}

// measured FMA throughput: 8 independent FMA chains per thread, all SMs busy
template <class T>
__global__ void k_fma(T *out, int iters, T seed)
{
    pdl_enter();
    T a[8];
#pragma unroll
    for (int k = 0; k < 8; k++) a[k] = seed + T(k) * T(1e-3) + T(threadIdx.x) * T(1e-7);
    const T m = T(0.999999), c = T(1e-7);
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 8; k++) a[k] = a[k] * m + c;
    }
    T s = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) s += a[k];
    if (s == T(-12345)) out[0] = s;
}

// the same with packed FP32x2 FMAs (FFMA2): 8 independent float2 chains per thread
__global__ void k_fma2(float *out, int iters, float seed)
{
    pdl_enter();
    float2 a[8];
#pragma unroll
    for (int k = 0; k < 8; k++) a[k] = make_float2(seed + k * 1e-3f + threadIdx.x * 1e-7f, seed - k * 1e-3f);
    const float2 m = make_float2(0.999999f, 0.999999f), c = make_float2(1e-7f, 1e-7f);
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 8; k++) a[k] = __ffma2_rn(a[k], m, c);
    }
    float s = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) s += a[k].x + a[k].y;
    if (s == -12345.f) out[0] = s;
}

int fma_peak(int fp64, double *tflops, cudaStream_t st)
{
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    void *buf = nullptr;
    PS_CK(cudaMalloc(&buf, 64));
    const int thr = 256, blocks = nsm * 8, iters = 1 << 14;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    // FP32: the larger of the scalar and the packed (FFMA2) throughput
    double best_tf = 0;
    for (int form = 0; form < (fp64 ? 1 : 2); form++) {
        float best = 1e30f;
        for (int rep = 0; rep < 4; rep++) {
            cudaEventRecord(a, st);
            if (fp64) ::ps_launch_count++, k_fma<double><<<blocks, thr, 0, st>>>((double *)buf, iters, 1.0);
            else if (form == 0) ::ps_launch_count++, k_fma<float><<<blocks, thr, 0, st>>>((float *)buf, iters, 1.0f);
            else ::ps_launch_count++, k_fma2<<<blocks, thr, 0, st>>>((float *)buf, iters / 2, 1.0f);
            cudaEventRecord(b, st);
            cudaEventSynchronize(b);
            float t = 0;
            cudaEventElapsedTime(&t, a, b);
            if (rep > 0) best = std::min(best, t);
        }
        // both forms: 8 chains x iters FMA per thread (packed: iters / 2 steps of 2 lanes)
        double flops = 2.0 * 8.0 * (double)iters * thr * blocks;
        best_tf = std::max(best_tf, flops / (best * 1e-3) / 1e12);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(buf);
    *tflops = best_tf;
    PS_CK(cudaGetLastError());
    return PS_OK;
}
}  // namespace ps
