// ps_reduce.cuh -- segmented per-replica reductions shared by the Krylov
// solvers: a block covers a contiguous range of one replica's vector; the last
// block of a replica to arrive (atomic counter) sums the partials in fixed
// order, so results never depend on block scheduling or on other replicas.
#pragma once
#include "ps_kernels.h"

namespace ps {

constexpr int RB_THREADS = 256;
constexpr int RB_EPT = 4;                       // elements per thread
constexpr int RB_SPAN = RB_THREADS * RB_EPT;    // elements per block

// Block-level sum of NV values; result valid in thread 0.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double (*sh)[NV])
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < NV; q++) {
        double t = v[q];
        for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
        if (lane == 0) sh[wid][q] = t;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NV; q++) {
            double t = 0;
            for (int w = 0; w < RB_THREADS / 32; w++) t += sh[w][q];
            v[q] = t;
        }
    }
}

// Writes this block's partials and returns true in thread 0 of the last block
// of its replica; that thread then holds the replica totals in tot[].
template <int NV>
__device__ __forceinline__ bool finish_block(const RedTable &T, const RBlk &b, int bid, double (&v)[NV], double (&tot)[NV])
{
    __shared__ bool last;
    if (threadIdx.x == 0) {
        for (int q = 0; q < NV; q++) T.d_part[4 * bid + q] = v[q];
        __threadfence();
        int t = atomicAdd(&T.d_counter[b.rep], 1);
        last = (t == T.d_count[b.rep] - 1);
    }
    __syncthreads();
    if (!last) return false;
    if (threadIdx.x == 0) {
        __threadfence();
        int f = T.d_first[b.rep], c = T.d_count[b.rep];
        for (int q = 0; q < NV; q++) tot[q] = 0.0;
        for (int k = 0; k < c; k++)
            for (int q = 0; q < NV; q++) tot[q] += ((volatile double *)T.d_part)[4 * (f + k) + q];
        T.d_counter[b.rep] = 0;
        return true;
    }
    return false;
}

}  // namespace ps
