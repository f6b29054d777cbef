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
// AA: monomer rows x monomer columns (mm_HI only), 3 -> 3.
// pos: (x,y,z,chain) per bead.  u: input vector, monomer F at off + 3 m.
template <class T>
__global__ void __launch_bounds__(RPY_THREADS, 4)
k_rpy_aa(const Seg *__restrict__ segs, const Tile *__restrict__ tiles, const typename V4<T>::t *__restrict__ pos,
         const float4 *__restrict__ plo, const double *__restrict__ u, int in_top, double *__restrict__ part,
         long part_stride, int nchunk, const char *__restrict__ done, int done_stride)
{
    if (done && *(const int *)(done + (long)tiles[blockIdx.x].rep * done_stride)) return;
    // FP32: positions are split hi + lo (both float) so that pair separations
    // keep FP64-level accuracy: d = (hi_i - hi_j) + (lo_i - lo_j).
    typedef typename V4<T>::t P4;
    constexpr bool F32 = sizeof(T) == 4;
    __shared__ P4 sp[RPY_THREADS];
    __shared__ float4 sl[F32 ? RPY_THREADS : 1];
    __shared__ T su[RPY_THREADS * 3];
    const Tile tl = tiles[blockIdx.x];
    const Seg &sg = segs[tl.rep];
    const int c = blockIdx.y;
    nchunk = sg.nch_aa;               // per-replica chunk count: a function of Nm alone
    if (c >= nchunk) return;
    const int Nm = sg.Nm;
    const int j0 = (int)((long)Nm * c / nchunk), j1 = (int)((long)Nm * (c + 1) / nchunk);
    const int i = tl.row0 + threadIdx.x;
    const bool active = threadIdx.x < tl.nrow;
    const int uoff = in_top ? sg.top_off : sg.vec_off;
    P4 pi = active ? pos[sg.bead_off + i] : pos[sg.bead_off + tl.row0];
    float4 li = make_float4(0.f, 0.f, 0.f, 0.f);
    if constexpr (F32) li = plo[sg.bead_off + (active ? i : tl.row0)];
    const T two_beta = T(2.0 * sg.beta);
    const bool chain_hi = sg.chain_HI != 0;
    // scalars in FP64 from the mode (x = c0/r + c1/r^3, ... as in Seg::aa_c)
    T c0, c1, c2, c3, c4, c5, c6, c7;
    if (sg.aa_mode == PS_AA_RPY) {
        T b = T(sg.beta), b2 = b * b;
        c0 = T(1.5); c1 = -b2; c2 = T(0.75); c3 = T(0.5) * b2;
        c4 = T(1) / b; c5 = T(-0.1875) / b2; c6 = T(1) / b; c7 = T(-0.28125) / b2;
    } else {
        c0 = T(0.375); c1 = T(-2.0); c2 = T(0.75); c3 = T(-0.5);
        c4 = T(-1.0); c5 = T(0.375); c6 = T(1.0); c7 = T(-0.28125);
    }
    Acc<T> a0, a1, a2;
    a0.zero(); a1.zero(); a2.zero();
    for (int jt = j0; jt < j1; jt += RPY_THREADS) {
        int nj = min(RPY_THREADS, j1 - jt);
        __syncthreads();
        if (threadIdx.x < nj) {
            int j = jt + threadIdx.x;
            sp[threadIdx.x] = pos[sg.bead_off + j];
            if constexpr (F32) sl[threadIdx.x] = plo[sg.bead_off + j];
            su[3 * threadIdx.x + 0] = (T)u[uoff + 3 * j + 0];
            su[3 * threadIdx.x + 1] = (T)u[uoff + 3 * j + 1];
            su[3 * threadIdx.x + 2] = (T)u[uoff + 3 * j + 2];
        }
        __syncthreads();
        T t0 = 0, t1 = 0, t2 = 0;
        for (int k = 0; k < nj; k++) {
            P4 pj = sp[k];
            T dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
            if constexpr (F32) {
                float4 lj = sl[k];
                dx += li.x - lj.x; dy += li.y - lj.y; dz += li.z - lj.z;
            }
            T r2 = dx * dx + dy * dy + dz * dz;
            bool skip = (jt + k == i) || (chain_hi && pi.w == pj.w);
            if (skip) continue;
            T rinv = rsqrt_t<T>(r2);
            T r = r2 * rinv;
            T x, y;
            if (r > two_beta) {
                T ri3 = rinv * rinv * rinv;
                x = c0 * rinv + c1 * ri3;
                y = c2 * rinv + c3 * ri3;
            } else {
                x = c4 + c5 * r;
                y = c6 + c7 * r;
            }
            T u0 = su[3 * k], u1 = su[3 * k + 1], u2 = su[3 * k + 2];
            // mob_a u = y u + (x - y)(e.u) e,  e = d / r
            T f = (x - y) * (dx * u0 + dy * u1 + dz * u2) * rinv * rinv;
            t0 += y * u0 + f * dx;
            t1 += y * u1 + f * dy;
            t2 += y * u2 + f * dz;
        }
        a0.add(t0); a1.add(t1); a2.add(t2);
    }
    if (active) {
        double *o = part + (long)c * part_stride + sg.top_off + 3 * i;
        o[0] = (double)a0.get(); o[1] = (double)a1.get(); o[2] = (double)a2.get();
    }
}

// ---------------------------------------------------------------------------
// AA in FP32 with packed FP32x2 arithmetic (sm_100 FFMA2/FADD2/FMUL2): each
// thread owns two rows (i and i + 64 of a 128-row tile) held in the two lanes of
// float2 registers, so one packed instruction advances two pairs against the
// same shared-memory column.  Positions are hi + lo floats.  Separations start
// as d = hi_i - hi_j, whose error is at most 2^-23 X for a replica whose
// coordinates stay below X in magnitude; within the replica's exact radius
// (r <= max(2.1 beta, X / 16), so the hi-only relative error stays below 2^-19
// where it is used) the warp adds the low parts, d = (hi_i - hi_j) + (lo_i - lo_j),
// the same rounding as a full hi + lo difference.  Self pairs and skipped
// same-chain pairs get rinv = 0, which zeroes their contribution without a
// branch; the near-overlap form (r <= 2 beta) lies inside the exact radius and is
// applied only when some lane of the warp needs it.
constexpr int AAF_THREADS = 64;

__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }

// one staged column tile against the thread's two rows; CHECK: the tile may
// hold the rows themselves or (chain_HI) same-chain partners, which get rinv = 0.
// Far form in factored scalars: y = ri (c + d ri^2), (x - y)/r^2 = ri^3 (a + b ri^2),
// a = c0 - c2, b = c1 - c3, c = c2, d = c3; the near form (r^2 <= (2 beta)^2)
// overwrites both.  Shared columns: sA (hi x, y, z, u0), sB (lo x, y, z, chain),
// sC (u1, u2); sB is read only inside the exact radius or by CHECK tiles.
template <bool CHECK>
__device__ __forceinline__ void aa_f2_cols(const float4 *__restrict__ sA, const float4 *__restrict__ sB,
                                           const float2 *__restrict__ sC, int jt, int nj, int i0, int i1,
                                           bool chain_hi, float w0, float w1, float2 px, float2 py, float2 pz,
                                           const float4 *__restrict__ plo, int b0, int b1, float2 fa, float2 fb,
                                           float2 fc, float2 fd, const Seg &sg, float te2, float2 &tx, float2 &ty,
                                           float2 &tz)
{
#pragma unroll 4
    for (int k = 0; k < nj; k++) {
        const float4 A = sA[k];
        const float2 C = sC[k];
        float2 dx = __fadd2_rn(px, f2(-A.x));
        float2 dy = __fadd2_rn(py, f2(-A.y));
        float2 dz = __fadd2_rn(pz, f2(-A.z));
        float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
        bool e0 = false, e1 = false;
        if constexpr (CHECK) {
            const int j = jt + k;
            const float cw = sB[k].w;
            e0 = (j == i0) || (chain_hi && w0 == cw);
            e1 = (j == i1) || (chain_hi && w1 == cw);
        }
        const bool inner = __any_sync(0xffffffffu, r2.x <= te2 || r2.y <= te2);
        if (inner) {
            // row low parts re-read from L1 here rather than held in registers
            const float4 B = sB[k], L0 = __ldg(plo + b0), L1 = __ldg(plo + b1);
            const float2 lx = make_float2(L0.x, L1.x), ly = make_float2(L0.y, L1.y), lz = make_float2(L0.z, L1.z);
            dx = __fadd2_rn(dx, __fadd2_rn(lx, f2(-B.x)));
            dy = __fadd2_rn(dy, __fadd2_rn(ly, f2(-B.y)));
            dz = __fadd2_rn(dz, __fadd2_rn(lz, f2(-B.z)));
            r2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
        }
        float2 ri = make_float2(e0 ? 0.f : rsqrtf(r2.x), e1 ? 0.f : rsqrtf(r2.y));
        float2 ri2 = __fmul2_rn(ri, ri);
        float2 yv = __fmul2_rn(__ffma2_rn(fd, ri2, fc), ri);                     // y
        float2 g = __fmul2_rn(__ffma2_rn(fb, ri2, fa), __fmul2_rn(ri2, ri));    // (x - y) / r^2
        if (inner) {
            // overlap constants re-read here: they are needed only inside the exact radius
            const float tb2 = (float)(4.0 * sg.beta * sg.beta);
            const float nx0 = sg.aa_c[4], nx1 = sg.aa_c[5], ny0 = sg.aa_c[6], ny1 = sg.aa_c[7];
            const bool n0 = !e0 && r2.x <= tb2, n1 = !e1 && r2.y <= tb2;
            if (n0) {
                float r = r2.x * ri.x, x = nx0 + nx1 * r;
                yv.x = ny0 + ny1 * r;
                g.x = (x - yv.x) * ri2.x;
            }
            if (n1) {
                float r = r2.y * ri.y, x = nx0 + nx1 * r;
                yv.y = ny0 + ny1 * r;
                g.y = (x - yv.y) * ri2.y;
            }
        }
        // mob_a u = y u + (x - y)(d.u) d / r^2
        float2 du = __ffma2_rn(dz, f2(C.y), __ffma2_rn(dy, f2(C.x), __fmul2_rn(dx, f2(A.w))));
        float2 f = __fmul2_rn(g, du);
        tx = __ffma2_rn(f, dx, __ffma2_rn(yv, f2(A.w), tx));
        ty = __ffma2_rn(f, dy, __ffma2_rn(yv, f2(C.x), ty));
        tz = __ffma2_rn(f, dz, __ffma2_rn(yv, f2(C.y), tz));
    }
}

__global__ void __launch_bounds__(AAF_THREADS, 16)
k_rpy_aa_f2(const Seg *__restrict__ segs, const Tile *__restrict__ tiles, const float4 *__restrict__ pos,
            const float4 *__restrict__ plo, const float *__restrict__ aa_te2, const double *__restrict__ u, int in_top,
            double *__restrict__ part, long part_stride, int nchunk, const char *__restrict__ done, int done_stride)
{
    if (done && *(const int *)(done + (long)tiles[blockIdx.x].rep * done_stride)) return;
    __shared__ float4 sA[128];   // hi x, y, z, u0
    __shared__ float4 sB[128];   // lo x, y, z, chain
    __shared__ float2 sC[128];   // u1, u2
    const Tile tl = tiles[blockIdx.x];
    const Seg &sg = segs[tl.rep];
    const int c = blockIdx.y;
    nchunk = sg.nch_aa;               // per-replica chunk count: a function of Nm alone
    if (c >= nchunk) return;
    const int Nm = sg.Nm;
    const int j0 = (int)((long)Nm * c / nchunk), j1 = (int)((long)Nm * (c + 1) / nchunk);
    const int i0 = tl.row0 + threadIdx.x, i1 = i0 + AAF_THREADS;
    const bool a0 = threadIdx.x < tl.nrow, a1 = threadIdx.x + AAF_THREADS < tl.nrow;
    const int uoff = in_top ? sg.top_off : sg.vec_off;
    const float4 P0 = pos[sg.bead_off + (a0 ? i0 : tl.row0)], P1 = pos[sg.bead_off + (a1 ? i1 : tl.row0)];
    const int b0 = sg.bead_off + (a0 ? i0 : tl.row0), b1 = sg.bead_off + (a1 ? i1 : tl.row0);
    const float2 px = make_float2(P0.x, P1.x), py = make_float2(P0.y, P1.y), pz = make_float2(P0.z, P1.z);
    const bool chain_hi = sg.chain_HI != 0;
    const float2 fa = f2(sg.aa_c[0] - sg.aa_c[2]), fb = f2(sg.aa_c[1] - sg.aa_c[3]);
    const float2 fc = f2(sg.aa_c[2]), fd = f2(sg.aa_c[3]);
    const float te2 = aa_te2[tl.rep];
    // Kahan sums across column tiles (sum, compensation per row and axis) live in
    // shared memory, thread-private, so the pair loop keeps their registers
    __shared__ float2 sKs[6][AAF_THREADS];
    for (int q = 0; q < 6; q++) sKs[q][threadIdx.x] = f2(0.f);
    for (int jt = j0; jt < j1; jt += 128) {
        const int nj = min(128, j1 - jt);
        __syncthreads();
        for (int t = threadIdx.x; t < nj; t += AAF_THREADS) {
            const int j = jt + t;
            const float4 A = pos[sg.bead_off + j], B = plo[sg.bead_off + j];
            sA[t] = make_float4(A.x, A.y, A.z, (float)u[uoff + 3 * j]);
            sB[t] = make_float4(B.x, B.y, B.z, A.w);
            sC[t] = make_float2((float)u[uoff + 3 * j + 1], (float)u[uoff + 3 * j + 2]);
        }
        __syncthreads();
        float2 tx = f2(0.f), ty = f2(0.f), tz = f2(0.f);
        // rows of this tile are [row0, row0 + 128): only overlapping column tiles hold self pairs
        const bool check = chain_hi || (jt < tl.row0 + 2 * AAF_THREADS && jt + nj > tl.row0);
        if (check)
            aa_f2_cols<true>(sA, sB, sC, jt, nj, i0, i1, chain_hi, P0.w, P1.w, px, py, pz, plo, b0, b1, fa,
                             fb, fc, fd, sg, te2, tx, ty, tz);
        else
            aa_f2_cols<false>(sA, sB, sC, jt, nj, i0, i1, chain_hi, P0.w, P1.w, px, py, pz, plo, b0, b1, fa,
                              fb, fc, fd, sg, te2, tx, ty, tz);
        // Kahan across column tiles
        const float2 t3[3] = {tx, ty, tz};
#pragma unroll
        for (int q = 0; q < 3; q++) {
            const float2 sq = sKs[q][threadIdx.x], kq = sKs[3 + q][threadIdx.x];
            const float2 yy = __fadd2_rn(t3[q], make_float2(-kq.x, -kq.y)), tt = __fadd2_rn(sq, yy);
            sKs[3 + q][threadIdx.x] = __fadd2_rn(__fadd2_rn(tt, make_float2(-sq.x, -sq.y)), make_float2(-yy.x, -yy.y));
            sKs[q][threadIdx.x] = tt;
        }
    }
    const float2 sx = sKs[0][threadIdx.x], sy = sKs[1][threadIdx.x], sz = sKs[2][threadIdx.x];
    double *o = part + (long)c * part_stride + sg.top_off;
    if (a0) { o[3 * i0] = sx.x; o[3 * i0 + 1] = sy.x; o[3 * i0 + 2] = sz.x; }
    if (a1) { o[3 * i1] = sx.y; o[3 * i1 + 1] = sy.y; o[3 * i1 + 2] = sz.y; }
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
// BB: colloid rows x colloid columns (FTS, 11 -> 11).
template <class T>
__global__ void __launch_bounds__(RPY_THREADS)
k_rpy_bb(const Seg *__restrict__ segs, const Tile *__restrict__ tiles, const typename V4<T>::t *__restrict__ pos,
         const float4 *__restrict__ plo, const double *__restrict__ u, int in_top, double *__restrict__ part,
         long part_stride, int nchunk, const char *__restrict__ done, int done_stride)
{
    if (done && *(const int *)(done + (long)tiles[blockIdx.x].rep * done_stride)) return;
    typedef typename V4<T>::t P4;
    constexpr bool F32 = sizeof(T) == 4;
    constexpr int CT = 64;
    __shared__ P4 sp[CT];
    __shared__ float4 sl[F32 ? CT : 1];
    __shared__ T su[CT * 11];
    const Tile tl = tiles[blockIdx.x];
    const Seg &sg = segs[tl.rep];
    const int c = blockIdx.y;
    nchunk = sg.nch_bb;
    if (c >= nchunk) return;
    const int Nc = sg.Nc, Nm = sg.Nm;
    const int j0 = (int)((long)Nc * c / nchunk), j1 = (int)((long)Nc * (c + 1) / nchunk);
    const int i = tl.row0 + threadIdx.x;
    const bool active = threadIdx.x < tl.nrow;
    const int uoff = in_top ? sg.top_off : sg.vec_off;
    P4 pi = pos[sg.bead_off + Nm + (active ? i : tl.row0)];
    float4 li = make_float4(0.f, 0.f, 0.f, 0.f);
    if constexpr (F32) li = plo[sg.bead_off + Nm + (active ? i : tl.row0)];
    Acc<T> acc[11];
    for (int q = 0; q < 11; q++) acc[q].zero();
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
        T out[11];
        for (int q = 0; q < 11; q++) out[q] = T(0);
        for (int k = 0; k < nj; k++) {
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
        for (int q = 0; q < 11; q++) acc[q].add(out[q]);
    }
    if (active) {
        double *o = part + (long)c * part_stride + sg.top_off;
        for (int a = 0; a < 3; a++) {
            o[sg.nm3 + 3 * i + a] = (double)acc[a].get();
            o[sg.nm3 + sg.nc3 + 3 * i + a] = (double)acc[3 + a].get();
        }
        for (int q = 0; q < 5; q++) o[sg.nm3nc6 + 5 * i + q] = (double)acc[6 + q].get();
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

__global__ void k_combine(const Seg *__restrict__ segs, const int *__restrict__ offs, int R, long total, int mode,
                          const double *__restrict__ x, const double *__restrict__ scale,
                          const double *__restrict__ partAA, int nchAA, const double *__restrict__ partAB,
                          const double *__restrict__ partBB, int nchBB, const double *__restrict__ partBA,
                          const double *__restrict__ delta, const double *__restrict__ lub_y,
                          long part_stride, double *__restrict__ y, const char *__restrict__ done, int done_stride)
{
    long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= total) return;
    int r = find_rep(offs, R, k);
    if (done && *(const int *)(done + (long)r * done_stride)) return;   // converged replica: skip
    const Seg &sg = segs[r];
    int i = (int)(k - offs[r]);
    const int xo = mode == 0 ? sg.vec_off : sg.top_off;
    const double s = scale ? scale[r] : 1.0;
    double v = 0.0;
    if (i < sg.nm3nc11) {
        if (i < sg.nm3) {
            v = sg.beta_inv * x[xo + i];
            if (sg.mm_HI)
                for (int c = 0; c < (nchAA ? sg.nch_aa : 0); c++) v += partAA[(long)c * part_stride + sg.top_off + i];
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
            if (sg.Nc >= 2)
                for (int c = 0; c < sg.nch_bb; c++) v += partBB[(long)c * part_stride + sg.top_off + i];
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

// ---------------------------------------------------------------------------
// host launchers
template <class T>
void launch_pairs(Engine &E, const double *u, int in_top, cudaStream_t st, const char *done, int dstride, bool skip_aa)
{
    const typename V4<T>::t *pos = (const typename V4<T>::t *)(sizeof(T) == 8 ? (const void *)E.d_pos64 : (const void *)E.d_pos32);
    if (E.n_aa_tiles && !skip_aa) {
        if constexpr (sizeof(T) == 4)
            ::ps_launch_count++, k_rpy_aa_f2<<<dim3(E.n_aa_tiles, E.nch_aa), AAF_THREADS, 0, st>>>(
                E.d_segs, E.d_aa_tiles, E.d_pos32, E.d_pos32lo, E.d_aa_te2, u, in_top, E.d_partAA, E.part_stride, E.nch_aa, done, dstride);
        else
            ::ps_launch_count++, k_rpy_aa<T><<<dim3(E.n_aa_tiles, E.nch_aa), RPY_THREADS, 0, st>>>(
                E.d_segs, E.d_aa_tiles, pos, E.d_pos32lo, u, in_top, E.d_partAA, E.part_stride, E.nch_aa, done, dstride);
    }
    if (E.n_ab_tiles)
        ::ps_launch_count++, k_rpy_ab<T><<<E.n_ab_tiles, RPY_THREADS, 0, st>>>(E.d_segs, E.d_ab_tiles, pos, E.d_pos32lo, u, in_top, E.d_tab, E.d_partAB,
                                                         E.d_partBA, done, dstride);
    // colloid-colloid FTS blocks stay FP64 in the mixed form: near contact the
    // far-field FTS mobility is ill-conditioned and FP32 blocks leave a 1.2e-6
    // velocity error on a suspension at gap 0.01 (FP64: tracks rtol); they are
    // cheap wherever monomers carry the O(N^2) work
    if (E.n_bb_tiles)
        ::ps_launch_count++, k_rpy_bb<double><<<dim3(E.n_bb_tiles, E.nch_bb), RPY_THREADS, 0, st>>>(
            E.d_segs, E.d_bb_tiles, E.d_pos64, E.d_pos32lo, u, in_top, E.d_partBB, E.part_stride, E.nch_bb, done, dstride);
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
    long total = mode == 0 ? E.nvec : E.ntop;
    const int *offs = mode == 0 ? E.d_vec_offs : E.d_top_offs;
    int thr = 256;
    ::ps_launch_count++, k_combine<<<(unsigned)((total + thr - 1) / thr), thr, 0, st>>>(
        E.d_segs, offs, E.R, total, mode, x, scale, E.d_partAA, skip_aa ? 0 : E.nch_aa, E.d_partAB, E.d_partBB, E.nch_bb,
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
            if (fp32) ::ps_launch_count++, k_rpy_aa_f2<<<dim3(E.n_aa_tiles, E.nch_aa), AAF_THREADS, 0, st>>>(E.d_segs, E.d_aa_tiles, (const float4 *)pos, E.d_pos32lo, E.d_aa_te2, u, 1, E.d_partAA, E.part_stride, E.nch_aa, nullptr, 0);
            else ::ps_launch_count++, k_rpy_aa<double><<<dim3(E.n_aa_tiles, E.nch_aa), RPY_THREADS, 0, st>>>(E.d_segs, E.d_aa_tiles, (const double4 *)pos, E.d_pos32lo, u, 1, E.d_partAA, E.part_stride, E.nch_aa, nullptr, 0);
        } else if (which == 1 && E.n_ab_tiles) {
            if (fp32) ::ps_launch_count++, k_rpy_ab<float><<<E.n_ab_tiles, RPY_THREADS, 0, st>>>(E.d_segs, E.d_ab_tiles, (const float4 *)pos, E.d_pos32lo, u, 1, E.d_tab, E.d_partAB, E.d_partBA, nullptr, 0);
            else ::ps_launch_count++, k_rpy_ab<double><<<E.n_ab_tiles, RPY_THREADS, 0, st>>>(E.d_segs, E.d_ab_tiles, (const double4 *)pos, E.d_pos32lo, u, 1, E.d_tab, E.d_partAB, E.d_partBA, nullptr, 0);
        } else if (which == 2 && E.n_bb_tiles) {
            ::ps_launch_count++, k_rpy_bb<double><<<dim3(E.n_bb_tiles, E.nch_bb), RPY_THREADS, 0, st>>>(E.d_segs, E.d_bb_tiles, E.d_pos64, E.d_pos32lo, u, 1, E.d_partBB, E.part_stride, E.nch_bb, nullptr, 0);
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

// measured FMA throughput: 8 independent FMA chains per thread, all SMs busy
template <class T>
__global__ void k_fma(T *out, int iters, T seed)
{
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
