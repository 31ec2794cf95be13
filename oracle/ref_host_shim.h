// ref_host_shim.h -- lets the reference's CUDA C++ sources compile as plain
// host C++ against Thrust's OpenMP backend.  TEST INFRASTRUCTURE ONLY: used by
// oracle/build_ref.py to build the reference's own step as the CPU oracle /
// CPU baseline.  No arithmetic of the reference is touched: the recipe only
// rewrites the launch syntax `k<<<g, b>>>(args)` into
// `host_launch(g, b, [&]() { k(args); })`; this header supplies
//   * empty CUDA qualifiers,
//   * dim3 and per-thread blockIdx / threadIdx / blockDim,
//   * host_launch: CUDA blocks spread over OpenMP threads, the threads of a
//     block run in order (the reference kernels use neither shared memory
//     nor __syncthreads, and no thread reads what another thread of the same
//     kernel writes),
//   * cudaMemcpyToSymbol as memcpy and cudaDeviceSynchronize as a no-op,
//   * cudaMalloc / cudaMemcpy on host memory,
//   * the CUDA host overloads min(double,double) / max(double,double).
#ifndef REF_HOST_SHIM_H
#define REF_HOST_SHIM_H

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <math.h>

#define __global__
#define __device__
#define __host__
#define __constant__
#define __forceinline__ inline

struct dim3 {
    unsigned x, y, z;
    dim3(unsigned a = 1, unsigned b = 1, unsigned c = 1) : x(a), y(b), z(c) {}
};
struct ref_uint3 {
    unsigned x, y, z;
};

extern thread_local ref_uint3 blockIdx;
extern thread_local ref_uint3 threadIdx;
extern thread_local dim3 blockDim;
extern thread_local dim3 gridDim;

template <class F>
static void host_launch(dim3 g, dim3 b, F body)
{
    const long nblk = (long)g.x * g.y * g.z;
#pragma omp parallel for schedule(static)
    for (long n = 0; n < nblk; ++n) {
        blockIdx.x = (unsigned)(n % g.x);
        blockIdx.y = (unsigned)((n / g.x) % g.y);
        blockIdx.z = (unsigned)(n / ((long)g.x * g.y));
        blockDim = b;
        gridDim = g;
        for (unsigned tz = 0; tz < b.z; ++tz)
            for (unsigned ty = 0; ty < b.y; ++ty)
                for (unsigned tx = 0; tx < b.x; ++tx) {
                    threadIdx.x = tx;
                    threadIdx.y = ty;
                    threadIdx.z = tz;
                    body();
                }
    }
}
template <class F>
static void host_launch(int g, int b, F body)
{
    host_launch(dim3((unsigned)g), dim3((unsigned)b), body);
}

#define cudaMemcpyToSymbol(sym, src, n) std::memcpy(&(sym), (src), (n))
static inline int cudaDeviceSynchronize() { return 0; }

// device memory is host memory (the multi-GPU library's Boundary copies its
// MPIInfo to the device, ResistiveMHD2D_GPU/boundary.cu:4-11)
enum ref_memcpy_kind { cudaMemcpyHostToHost, cudaMemcpyHostToDevice, cudaMemcpyDeviceToHost, cudaMemcpyDeviceToDevice };
template <class T> static inline int cudaMalloc(T **p, size_t n)
{
    *p = static_cast<T *>(std::malloc(n));
    return *p ? 0 : 2;
}
static inline int cudaMemcpy(void *dst, const void *src, size_t n, ref_memcpy_kind)
{
    std::memcpy(dst, src, n);
    return 0;
}

static inline double min(double a, double b) { return fmin(a, b); }
static inline double max(double a, double b) { return fmax(a, b); }

using std::isnan;

#endif
