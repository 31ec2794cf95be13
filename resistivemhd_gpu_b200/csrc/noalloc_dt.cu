// noalloc_dt.cu -- CFL dt of a caller-owned device state with no device
// allocation (rmhd2d_calculate_dt_noalloc).  Compiled with -fmad=false: the
// per-cell rate and the dt round exactly as rate_kernel and the solver's
// rmhd2d_calculate_dt do.
//
// All scratch lives in one file-scope device array (g_dt_scratch, 33,024
// bytes), laid out in 8-byte words:
//
//   [0, NA_MAX_BLOCKS)      per-block maxima of the rate bits (every block
//                           of a call writes its own word before any read)
//   W_FIRST_NAN             1 if cell 0's dt candidate is NaN (written by
//                           block 0 on every call)
//   W_COUNTER               blocks finished; MUST START AT ZERO -- cleared
//                           by a memset before every launch
//   W_RESULT                the dt of the call (bits of a double)
//
// One launch of ceil(ncell / NA_CELLS_PER_BLOCK) blocks: each block reduces
// its cells to one word, and the block that finishes last (completion
// counter) reduces those words, applies the diffusive limit and writes dt.
// Every call on a device uses the same array, so calls that overlap in time
// race.
#include <cuda_runtime.h>

#include "../../include/rmhd2d.h"
#include "noalloc_dt.h"
#include "physics.cuh"
#include "rmhd2d_internal.h"

namespace rmhd2d {

namespace {

constexpr int NA_THREADS = 256;
constexpr long long NA_CELLS_PER_BLOCK = 4096;
constexpr int NA_MAX_BLOCKS = (int)(RMHD2D_NOALLOC_MAX_CELLS / NA_CELLS_PER_BLOCK);
constexpr int W_FIRST_NAN = NA_MAX_BLOCKS;
constexpr int W_COUNTER = NA_MAX_BLOCKS + 1;
constexpr int W_RESULT = NA_MAX_BLOCKS + 2;
constexpr int NA_WORDS = NA_MAX_BLOCKS + 32;   // 256-byte multiple
static_assert(RMHD2D_NOALLOC_MAX_CELLS % NA_CELLS_PER_BLOCK == 0, "limit must be whole blocks");
static_assert((NA_WORDS * 8) % 256 == 0, "scratch is a 256-byte multiple");

}  // namespace

static __device__ __align__(256) unsigned long long g_dt_scratch[NA_WORDS];

namespace {

__device__ __forceinline__ unsigned long long block_max(unsigned long long v, unsigned long long *wmax)
{
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const unsigned long long o = __shfl_xor_sync(0xffffffffu, v, off);
        v = o > v ? o : v;
    }
    if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < NA_THREADS / 32; ++w) v = wmax[w] > v ? wmax[w] : v;
    }
    return v;   // valid in thread 0
}

// The rate of rate_kernel (resistiveMHD_2D.cu:247-274 calculateDtFunctor)
// over the reference's array-of-structures state, then the dt of
// resistiveMHD_2D.cu:286-288 (thrust::min_element semantics via rate_bits
// and the cell-0 NaN flag, as step_dt documents).
__global__ void __launch_bounds__(NA_THREADS) dt_noalloc_kernel(const double *__restrict__ aos, long long ncell,
                                                                double gm, double dx, double dy, double eps,
                                                                double eta, double cfl,
                                                                unsigned long long *scratch)
{
    __shared__ unsigned long long wmax[NA_THREADS / 32];
    __shared__ int is_last;
    const long long c0 = (long long)blockIdx.x * NA_CELLS_PER_BLOCK;
    const long long c1 = c0 + NA_CELLS_PER_BLOCK < ncell ? c0 + NA_CELLS_PER_BLOCK : ncell;
    unsigned long long bits = 0ull;
    for (long long c = c0 + threadIdx.x; c < c1; c += NA_THREADS) {
        const double *q = aos + c * NFIELD;
        const double r = cfl_rate(q[RHO], q[MX], q[MY], q[MZ], q[BXF], q[BYF], q[BZF], q[EN], gm, dx, dy);
        const unsigned long long b = rate_bits(r);
        bits = b > bits ? b : bits;
        if (c == 0) scratch[W_FIRST_NAN] = (r != r) ? 1ull : 0ull;
    }
    bits = block_max(bits, wmax);
    if (threadIdx.x == 0) {
        scratch[blockIdx.x] = bits;
        __threadfence();
        const unsigned long long ticket = atomicAdd(&scratch[W_COUNTER], 1ull);
        is_last = ticket == (unsigned long long)gridDim.x - 1ull;
    }
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    unsigned long long m = 0ull;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += NA_THREADS) {
        const unsigned long long v = __ldcg(&scratch[b]);
        m = v > m ? v : m;
    }
    __syncthreads();   // wmax is reused
    m = block_max(m, wmax);
    if (threadIdx.x == 0) {
        const int first_nan = __ldcg(&scratch[W_FIRST_NAN]) != 0ull;
        const double dt = step_dt(m, first_nan, dx, dy, eps, eta, cfl);
        scratch[W_RESULT] = (unsigned long long)__double_as_longlong(dt);
        scratch[W_COUNTER] = 0ull;
    }
}

}  // namespace

cudaError_t noalloc_scratch(unsigned long long **ptr)
{
    // Looked up on every call, not cached: the address belongs to the
    // module loaded into the current context, and a context reset
    // (cudaDeviceReset) loads the module again at another address.  The
    // lookup allocates nothing.
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_dt_scratch);
    if (e != cudaSuccess) return e;
    *ptr = static_cast<unsigned long long *>(p);
    return cudaSuccess;
}

cudaError_t enqueue_dt_noalloc(const double *aos, long long ncell, double gm, double dx, double dy, double eps,
                               double eta, double cfl, unsigned long long *scratch, double *dt_host,
                               cudaStream_t st)
{
    if (ncell < 1 || ncell > RMHD2D_NOALLOC_MAX_CELLS) return cudaErrorInvalidValue;
    const int blocks = (int)((ncell + NA_CELLS_PER_BLOCK - 1) / NA_CELLS_PER_BLOCK);
    cudaError_t e = cudaMemsetAsync(scratch + W_COUNTER, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess) return e;
    dt_noalloc_kernel<<<blocks, NA_THREADS, 0, st>>>(aos, ncell, gm, dx, dy, eps, eta, cfl, scratch);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return cudaMemcpyAsync(dt_host, scratch + W_RESULT, sizeof(double), cudaMemcpyDeviceToHost, st);
}

}  // namespace rmhd2d
