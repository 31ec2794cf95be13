// cuda_host_shim.h -- TEST INFRASTRUCTURE.  Lets the discrete adjoint's
// kernel sources (resistivemhd_gpu_b200/csrc/adjoint.cu, adjoint_prep.cu)
// compile with g++ and run on the CPU, so the CPU tests can check the
// adjoint's arithmetic against the oracle's tangent without a GPU.
//
// Most kernels are one thread per cell, interface or ghost, with no shared
// memory, barriers or atomics, so a kernel launch becomes a loop over the
// launch's blocks and threads (host_launch; tests/host_build.py rewrites each
// `k<<<grid, block, smem, stream>>>(args)` into such a call).  A kernel that
// stages a tile in shared memory and synchronises its block runs with one
// host thread per CUDA thread and a block barrier (host_launch_threaded;
// __shared__ arrays become statics, one block runs at a time).  The
// correctly rounded device operations map to the host's IEEE binary64
// operations; the reverse sweep's reciprocals are host divisions
// (adjoint_core.cuh: adj_rcp), so results agree with the GPU's to
// rounding.
#pragma once

#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#define __global__
#define __device__
#define __host__
#define __forceinline__ inline
#define __launch_bounds__(...)
#define __shared__ static

struct dim3 {
    unsigned x, y, z;
    constexpr dim3(unsigned a = 1, unsigned b = 1, unsigned c = 1) : x(a), y(b), z(c) {}
};

inline thread_local dim3 blockIdx, threadIdx;
inline dim3 blockDim, gridDim;

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

// The barrier of the block that host_launch_threaded runs.  A thread that
// returns leaves it, as an exited thread does on the device.
struct ShimBarrier {
    std::mutex m;
    std::condition_variable cv;
    unsigned expected = 0, arrived = 0;
    unsigned long generation = 0;
    void release()
    {
        arrived = 0;
        ++generation;
        cv.notify_all();
    }
    void arrive_and_wait()
    {
        std::unique_lock<std::mutex> lk(m);
        const unsigned long gen = generation;
        if (++arrived == expected) {
            release();
            return;
        }
        cv.wait(lk, [&] { return generation != gen; });
    }
    void drop()
    {
        std::unique_lock<std::mutex> lk(m);
        --expected;
        if (expected > 0 && arrived == expected) release();
    }
};
inline ShimBarrier g_block_barrier;

inline void __syncthreads() { g_block_barrier.arrive_and_wait(); }

template <class F> void host_launch_threaded(dim3 grid, dim3 block, F &&kernel_call)
{
    gridDim = grid;
    blockDim = block;
    const unsigned n = block.x * block.y * block.z;
    for (unsigned bz = 0; bz < grid.z; ++bz)
        for (unsigned by = 0; by < grid.y; ++by)
            for (unsigned bx = 0; bx < grid.x; ++bx) {
                g_block_barrier.expected = n;
                g_block_barrier.arrived = 0;
                std::vector<std::thread> threads;
                threads.reserve(n);
                for (unsigned t = 0; t < n; ++t)
                    threads.emplace_back([&, t, bx, by, bz] {
                        blockIdx = dim3(bx, by, bz);
                        threadIdx = dim3(t % block.x, (t / block.x) % block.y, t / (block.x * block.y));
                        kernel_call();
                        g_block_barrier.drop();
                    });
                for (auto &th : threads) th.join();
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

inline double rsqrt(double x) { return 1.0 / std::sqrt(x); }

inline float __int_as_float(int x)
{
    float r;
    std::memcpy(&r, &x, sizeof r);
    return r;
}

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
