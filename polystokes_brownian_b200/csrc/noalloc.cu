// noalloc.cu -- ps_mobility_apply_noalloc: the monomer-monomer far-field
// mobility apply y = M u for ONE system of N monomers, with no device memory
// allocation of any kind.
//
// Some callers cannot allocate device memory: for example a matrix-free
// operator callback that a host solver framework calls inside its iteration
// loop while that framework owns the device memory pool, or a latency-critical
// loop where cudaMalloc's implicit device synchronisation, or its failure under
// memory pressure, is not acceptable.  For them this entry point keeps its
// scratch memory (packed positions and the per-column-chunk partial sums) in a
// file-scope __device__ array of fixed size, resident on every GPU that loads
// this library until the process exits.  The caller passes only the inputs and
// the output.
//
// Scratch layout (doubles): [ 4 * PS_NOALLOC_MAX_BEADS packed (x,y,z,chain) |
// PS_NOALLOC_CHUNKS * 3 * PS_NOALLOC_MAX_BEADS chunk partials ].  Every partial
// that the combine kernel reads is written by the pair kernel of the same call,
// so nothing needs clearing between calls; the array keeps the last call's
// contents.  All calls share the one array: calls whose kernels overlap on the
// GPU (different streams, or different host threads) race on it and must be
// serialised by the caller.
#include <algorithm>
#include <mutex>
#include <string>
#include "ps_internal.h"
#include "ps_kernels.h"

#define PS_NOALLOC_MAX_BEADS 8192
#define PS_NOALLOC_CHUNKS 16
#define PS_NOALLOC_DOUBLES (4 * PS_NOALLOC_MAX_BEADS + PS_NOALLOC_CHUNKS * 3 * PS_NOALLOC_MAX_BEADS)

static __device__ __align__(256) double g_noalloc_scratch[PS_NOALLOC_DOUBLES];

namespace {

constexpr int NA_THREADS = 128;

__global__ void k_na_pack(const double *__restrict__ x, int N, int nper, double *__restrict__ scratch)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    double4 *p = reinterpret_cast<double4 *>(scratch);
    p[i] = make_double4(x[3 * i], x[3 * i + 1], x[3 * i + 2], (double)(i / nper));
}

// monomer rows x monomer columns of one chunk (reference AA scalars, mob.cpp:122-131)
__global__ void __launch_bounds__(NA_THREADS)
k_na_pairs(const double *__restrict__ u, int N, double beta, int chain_hi, int nchunk, double *__restrict__ scratch)
{
    __shared__ double4 sp[NA_THREADS];
    __shared__ double su[3 * NA_THREADS];
    const double4 *pos = reinterpret_cast<const double4 *>(scratch);
    double *part = scratch + 4 * PS_NOALLOC_MAX_BEADS;
    const int c = blockIdx.y;
    const int j0 = (int)((long)N * c / nchunk), j1 = (int)((long)N * (c + 1) / nchunk);
    const int i = blockIdx.x * NA_THREADS + threadIdx.x;
    const bool active = i < N;
    const double4 pi = pos[active ? i : 0];
    double a0 = 0, a1 = 0, a2 = 0;
    for (int jt = j0; jt < j1; jt += NA_THREADS) {
        int nj = min(NA_THREADS, j1 - jt);
        __syncthreads();
        if (threadIdx.x < nj) {
            int j = jt + threadIdx.x;
            sp[threadIdx.x] = pos[j];
            su[3 * threadIdx.x] = u[3 * j];
            su[3 * threadIdx.x + 1] = u[3 * j + 1];
            su[3 * threadIdx.x + 2] = u[3 * j + 2];
        }
        __syncthreads();
        for (int k = 0; k < nj; k++) {
            double4 pj = sp[k];
            if (jt + k == i || (chain_hi && pi.w == pj.w)) continue;
            double dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
            double r2 = dx * dx + dy * dy + dz * dz;
            double rinv = rsqrt(r2), r = r2 * rinv, xx, yy;
            // near the jump of the reference's scalars at 2 beta, its own distance decides the branch
            if (fabs(r2 - 4.0 * beta * beta) <= 1e-10 * r2) { r = ref_pair_dist(dx, dy, dz); rinv = 1.0 / r; }
            aa_scalars<double>(r, rinv, 2.0 * beta, xx, yy);
            double u0 = su[3 * k], u1 = su[3 * k + 1], u2 = su[3 * k + 2];
            double f = (xx - yy) * (dx * u0 + dy * u1 + dz * u2) * rinv * rinv;
            a0 += yy * u0 + f * dx;
            a1 += yy * u1 + f * dy;
            a2 += yy * u2 + f * dz;
        }
    }
    if (active) {
        double *o = part + (long)c * 3 * PS_NOALLOC_MAX_BEADS + 3 * i;
        o[0] = a0; o[1] = a1; o[2] = a2;
    }
}

// y = beta^{-1} u + sum of chunk partials in fixed chunk order
__global__ void k_na_combine(const double *__restrict__ u, int N, double beta_inv, int nchunk,
                             const double *__restrict__ scratch, double *__restrict__ y)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= 3 * N) return;
    const double *part = scratch + 4 * PS_NOALLOC_MAX_BEADS;
    double v = beta_inv * u[k];
    for (int c = 0; c < nchunk; c++) v += part[(long)c * 3 * PS_NOALLOC_MAX_BEADS + k];
    y[k] = v;
}

std::mutex g_na_mutex;
double *g_na_ptr[256] = {nullptr};

}  // namespace

extern "C" int ps_mobility_apply_noalloc(const double *x, const double *u, double *y, int32_t N, double beta,
                                         int32_t chain_HI, int32_t Nmono_per_chain, void *stream)
{
    if (!x || !u || !y || N < 1 || !(beta > 0) || Nmono_per_chain < 1) {
        ps::set_error("ps_mobility_apply_noalloc: bad arguments");
        return PS_ERR_ARG;
    }
    if (N > PS_NOALLOC_MAX_BEADS) {
        ps::set_error("ps_mobility_apply_noalloc: N = " + std::to_string(N) + " exceeds the fixed scratch limit of " +
                      std::to_string(PS_NOALLOC_MAX_BEADS) + " monomers");
        return PS_ERR_TOO_LARGE;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256) {
        ps::set_error("ps_mobility_apply_noalloc: no current CUDA device");
        return PS_ERR_CUDA;
    }
    double *scratch;
    {
        // one-time set-up per device: the device address of the scratch array
        // (its name in host code is only a host-side stand-in)
        std::lock_guard<std::mutex> lk(g_na_mutex);
        if (!g_na_ptr[dev]) {
            void *p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p) {
                ps::set_error(std::string("ps_mobility_apply_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
                return PS_ERR_CUDA;
            }
            g_na_ptr[dev] = static_cast<double *>(p);
        }
        scratch = g_na_ptr[dev];
    }
    cudaStream_t st = (cudaStream_t)stream;
    const int ntiles = (N + NA_THREADS - 1) / NA_THREADS;
    int nchunk = (148 * 4 + ntiles - 1) / ntiles;
    nchunk = std::max(1, std::min(nchunk, std::min(PS_NOALLOC_CHUNKS, std::max(1, N / NA_THREADS))));
    ::ps_launch_count++, k_na_pack<<<(N + 255) / 256, 256, 0, st>>>(x, N, Nmono_per_chain, scratch);
    ::ps_launch_count++, k_na_pairs<<<dim3(ntiles, nchunk), NA_THREADS, 0, st>>>(u, N, beta, chain_HI, nchunk, scratch);
    ::ps_launch_count++, k_na_combine<<<(3 * N + 255) / 256, 256, 0, st>>>(u, N, 1.0 / beta, nchunk, scratch, y);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        ps::set_error(std::string("ps_mobility_apply_noalloc: launch: ") + cudaGetErrorString(e));
        return PS_ERR_CUDA;
    }
    return PS_OK;
}
