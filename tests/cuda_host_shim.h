// cuda_host_shim.h -- TEST INFRASTRUCTURE.  Lets the discrete adjoint's
// kernel sources (resistivemhd_gpu_b200/csrc/adjoint.cu, adjoint_prep.cu)
// compile with g++ and run on the CPU, so the CPU tests can check the
// adjoint's arithmetic against the oracle's tangent without a GPU.
//
// Those kernels are one thread per cell, interface or ghost, with no shared
// memory, barriers or atomics, so a kernel launch becomes a loop over the
// launch's blocks and threads (host_launch; the test rewrites each
// `k<<<grid, block, smem, stream>>>(args)` into a host_launch call).  The
// correctly rounded device operations map to the host's IEEE binary64
// operations; the reverse sweep's reciprocals are host divisions
// (adjoint_core.cuh: adj_rcp), so results agree with the GPU's to
// rounding.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>

#define __global__
#define __device__
#define __host__
#define __forceinline__ inline
#define __launch_bounds__(...)

struct dim3 {
    unsigned x, y, z;
    constexpr dim3(unsigned a = 1, unsigned b = 1, unsigned c = 1) : x(a), y(b), z(c) {}
};

inline dim3 blockIdx, threadIdx, blockDim, gridDim;

typedef struct CUstream_st *cudaStream_t;

template <class F> void host_launch(dim3 grid, dim3 block, F &&kernel_call)
{
    gridDim = grid;
    blockDim = block;
    for (unsigned bz = 0; bz < grid.z; ++bz)
        for (unsigned by = 0; by < grid.y; ++by)
            for (unsigned bx = 0; bx < grid.x; ++bx)
                for (unsigned tz = 0; tz < block.z; ++tz)
                    for (unsigned ty = 0; ty < block.y; ++ty)
                        for (unsigned tx = 0; tx < block.x; ++tx) {
                            blockIdx = dim3(bx, by, bz);
                            threadIdx = dim3(tx, ty, tz);
                            kernel_call();
                        }
}

// The device's __dadd_rn and the others are single correctly rounded
// operations that are never fused with a neighbouring one.  The empty asm
// statements make their operands and results opaque to the host compiler,
// so that holds here too when the rest of a file is built with contraction
// (-ffp-contract=fast), the way nvcc builds the adjoint kernels.
#if defined(__x86_64__)
#define RN_OPAQUE(v) asm("" : "+x"(v))
#else
#define RN_OPAQUE(v) ((void)0)
#endif
inline double __dadd_rn(double a, double b) { RN_OPAQUE(a); RN_OPAQUE(b); double r = a + b; RN_OPAQUE(r); return r; }
inline double __dsub_rn(double a, double b) { RN_OPAQUE(a); RN_OPAQUE(b); double r = a - b; RN_OPAQUE(r); return r; }
inline double __dmul_rn(double a, double b) { RN_OPAQUE(a); RN_OPAQUE(b); double r = a * b; RN_OPAQUE(r); return r; }
inline double __ddiv_rn(double a, double b) { RN_OPAQUE(a); RN_OPAQUE(b); double r = a / b; RN_OPAQUE(r); return r; }
inline double __dsqrt_rn(double a) { RN_OPAQUE(a); double r = std::sqrt(a); RN_OPAQUE(r); return r; }

inline long long __double_as_longlong(double x)
{
    long long r;
    std::memcpy(&r, &x, sizeof r);
    return r;
}
inline double __longlong_as_double(long long x)
{
    double r;
    std::memcpy(&r, &x, sizeof r);
    return r;
}
