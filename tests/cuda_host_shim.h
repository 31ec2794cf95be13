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

#include <atomic>
#include <chrono>
#include <cmath>
#include <functional>
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
#define __grid_constant__
#define __shared__ static
#define __align__(n) __attribute__((aligned(n)))

struct dim3 {
    unsigned x, y, z;
    constexpr dim3(unsigned a = 1, unsigned b = 1, unsigned c = 1) : x(a), y(b), z(c) {}
};

inline thread_local dim3 blockIdx, threadIdx;
inline dim3 blockDim, gridDim;

typedef struct CUstream_st *cudaStream_t;

// The driver's opaque 128-byte tensor-map type; host builds fill it with
// tests/host_tma.h's HostMap.
typedef struct CUtensorMap_st {
    alignas(64) unsigned long long opaque[16];
} CUtensorMap;

// What the host build's tensor maps hold (written by cuTensorMapEncodeTiled
// below or by the tests' drivers, read by tests/host_tma.cpp).
struct HostMap {
    const double *base;
    unsigned long long dims[3];      // innermost first: j (ny), i (nx), field (8)
    unsigned long long strides[2];   // bytes between consecutive i, between fields
    unsigned box[3];                 // box extent per dimension
    int rank;                        // 2 or 3
};
static_assert(sizeof(HostMap) <= sizeof(CUtensorMap), "a host map fits a tensor map's bytes");

// Stream capture (cudaStreamBeginCapture .. EndCapture): launches and async
// copies are recorded instead of run, and a graph launch runs the record.
inline bool g_capturing = false;
inline std::vector<std::function<void()>> *g_capture_ops = nullptr;
inline bool shim_record(std::function<void()> op)
{
    if (!g_capturing) return false;
    g_capture_ops->push_back(std::move(op));
    return true;
}

template <class F> void host_launch_now(dim3 grid, dim3 block, F &kernel_call);
template <class F> void host_launch(dim3 grid, dim3 block, F &&kernel_call)
{
    std::decay_t<F> call = kernel_call;
    if (shim_record([=]() mutable { host_launch_now(grid, block, call); })) return;
    host_launch_now(grid, block, call);
}

template <class F> void host_launch_now(dim3 grid, dim3 block, F &kernel_call)
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

// A barrier of the threads that host_launch_threaded runs (a block, or one
// warp of it).  A thread that returns leaves it, as an exited thread does on
// the device.
struct ShimBarrier {
    std::mutex m;
    unsigned expected = 0, arrived = 0;
    std::atomic<unsigned long> generation{0};
    void reset(unsigned n)
    {
        std::lock_guard<std::mutex> lk(m);
        expected = n;
        arrived = 0;
    }
    void release()   // with m held
    {
        arrived = 0;
        generation.fetch_add(1);
    }
    // State changes under the mutex; the waiters spin on the generation.
    void arrive_and_wait()
    {
        unsigned long gen;
        {
            std::lock_guard<std::mutex> lk(m);
            gen = generation.load();
            if (++arrived == expected) {
                release();
                return;
            }
        }
        while (generation.load() == gen) std::this_thread::yield();
    }
    void drop()
    {
        std::lock_guard<std::mutex> lk(m);
        --expected;
        if (expected > 0 && arrived == expected) release();
    }
};
inline ShimBarrier g_block_barrier;
inline ShimBarrier g_warp_barrier[32];        // one per warp of the running block (at most 1024 threads)
inline unsigned long long g_warp_lanes[32][32];

inline void __syncthreads() { g_block_barrier.arrive_and_wait(); }

inline std::atomic<int> g_block_or{0};
inline int shim_flat_thread_id();
// Block-wide OR of pred, returned to every thread (three meetings: gather,
// read, clear).
inline int __syncthreads_or(int pred)
{
    if (pred) g_block_or.fetch_or(1);
    __syncthreads();
    const int r = g_block_or.load();
    __syncthreads();
    if (shim_flat_thread_id() == 0) g_block_or.store(0);
    __syncthreads();
    return r;
}

// Dynamic shared memory of the running block (host_launch_threaded's
// `smem_bytes`), filled with NaN bytes at each block's start so that a read
// of a word the block did not write shows up in the results.
// It is allocated at exactly the launch's size, so that a sanitizer sees an
// access past its end.
inline unsigned char *g_dynamic_smem = nullptr;
inline unsigned char *shim_dynamic_smem() { return g_dynamic_smem; }

inline unsigned shim_flat_thread() { return threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z); }
inline int shim_flat_thread_id() { return (int)shim_flat_thread(); }

// Warp exchanges of the threaded launch: each lane posts its value, the warp
// meets, each lane reads its partner's, the warp meets again.  Only full
// warps (mask 0xffffffff) are modelled, which is how the kernels call them.
inline unsigned long long __shfl_xor_sync(unsigned, unsigned long long v, int lane_mask)
{
    const unsigned t = shim_flat_thread(), w = t >> 5, lane = t & 31u;
    g_warp_lanes[w][lane] = v;
    g_warp_barrier[w].arrive_and_wait();
    const unsigned long long r = g_warp_lanes[w][lane ^ (unsigned)lane_mask];
    g_warp_barrier[w].arrive_and_wait();
    return r;
}
inline int __any_sync(unsigned, int pred)
{
    const unsigned t = shim_flat_thread(), w = t >> 5, lane = t & 31u;
    g_warp_lanes[w][lane] = pred ? 1ull : 0ull;
    g_warp_barrier[w].arrive_and_wait();
    int any = 0;
    for (unsigned l = 0; l < 32; ++l) any |= g_warp_lanes[w][l] != 0ull;
    g_warp_barrier[w].arrive_and_wait();
    return any;
}

inline std::mutex g_atomic_mutex;
inline unsigned long long atomicMax(unsigned long long *p, unsigned long long v)
{
    std::lock_guard<std::mutex> lk(g_atomic_mutex);
    const unsigned long long old = *p;
    if (v > old) *p = v;
    return old;
}
inline unsigned long long atomicAdd(unsigned long long *p, unsigned long long v)
{
    std::lock_guard<std::mutex> lk(g_atomic_mutex);
    const unsigned long long old = *p;
    *p = old + v;
    return old;
}
inline int atomicExch(int *p, int v)
{
    std::lock_guard<std::mutex> lk(g_atomic_mutex);
    const int old = *p;
    *p = v;
    return old;
}
inline void __threadfence() { std::atomic_thread_fence(std::memory_order_seq_cst); }
template <class T> inline T __ldcg(const T *p)
{
    std::lock_guard<std::mutex> lk(g_atomic_mutex);
    return *p;
}

inline ShimBarrier g_launch_barrier;   // between the blocks of one threaded launch

inline void shim_begin_block(size_t smem_bytes, unsigned n)
{
    void *smem = nullptr;
    if (smem_bytes && posix_memalign(&smem, 1024, smem_bytes) != 0) std::abort();
    if (smem) std::memset(smem, 0xFF, smem_bytes);
    g_dynamic_smem = static_cast<unsigned char *>(smem);
    g_block_or.store(0);
    g_block_barrier.reset(n);
    for (unsigned w = 0; w < (n + 31) / 32; ++w) g_warp_barrier[w].reset(n - 32 * w < 32 ? n - 32 * w : 32);
}

inline void shim_end_block()
{
    std::free(g_dynamic_smem);
    g_dynamic_smem = nullptr;
}

// One host thread per CUDA thread of a block; the same threads run the
// launch's blocks one after another, meeting between blocks while one of
// them sets up the next block's shared memory and barriers.
template <class F> void host_launch_threaded_now(dim3 grid, dim3 block, F &kernel_call, size_t smem_bytes);
template <class F> void host_launch_threaded(dim3 grid, dim3 block, F &&kernel_call, size_t smem_bytes = 0)
{
    std::decay_t<F> call = kernel_call;
    if (shim_record([=]() mutable { host_launch_threaded_now(grid, block, call, smem_bytes); })) return;
    host_launch_threaded_now(grid, block, call, smem_bytes);
}

template <class F> void host_launch_threaded_now(dim3 grid, dim3 block, F &kernel_call, size_t smem_bytes)
{
    gridDim = grid;
    blockDim = block;
    const unsigned n = block.x * block.y * block.z;
    const unsigned long long nblocks = (unsigned long long)grid.x * grid.y * grid.z;
    if (nblocks == 0 || n == 0) return;
    g_launch_barrier.reset(n);
    shim_begin_block(smem_bytes, n);
    std::vector<std::thread> threads;
    threads.reserve(n);
    for (unsigned t = 0; t < n; ++t)
        threads.emplace_back([&, t] {
            for (unsigned long long b = 0; b < nblocks; ++b) {
                blockIdx = dim3((unsigned)(b % grid.x), (unsigned)((b / grid.x) % grid.y),
                                (unsigned)(b / ((unsigned long long)grid.x * grid.y)));
                threadIdx = dim3(t % block.x, (t / block.x) % block.y, t / (block.x * block.y));
                kernel_call();
                g_warp_barrier[t >> 5].drop();
                g_block_barrier.drop();
                g_launch_barrier.arrive_and_wait();
                if (t == 0) {
                    shim_end_block();
                    if (b + 1 < nblocks) shim_begin_block(smem_bytes, n);
                }
                g_launch_barrier.arrive_and_wait();
            }
        });
    for (auto &th : threads) th.join();
}

// The runtime calls the kernels' host launchers make.
typedef int cudaError_t;
enum { cudaSuccess = 0, cudaErrorInvalidValue = 1, cudaErrorInvalidDevice = 101 };
enum cudaMemcpyKind { cudaMemcpyHostToHost, cudaMemcpyHostToDevice, cudaMemcpyDeviceToHost, cudaMemcpyDeviceToDevice };
inline cudaError_t cudaGetLastError() { return cudaSuccess; }
inline cudaError_t cudaMemsetAsync(void *p, int v, size_t n, cudaStream_t = nullptr)
{
    if (!shim_record([=] { std::memset(p, v, n); })) std::memset(p, v, n);
    return cudaSuccess;
}
inline cudaError_t cudaMemcpyAsync(void *d, const void *s, size_t n, cudaMemcpyKind, cudaStream_t = nullptr)
{
    if (!shim_record([=] { std::memcpy(d, s, n); })) std::memcpy(d, s, n);
    return cudaSuccess;
}
inline cudaError_t cudaStreamSynchronize(cudaStream_t) { return cudaSuccess; }
enum cudaFuncAttribute { cudaFuncAttributeMaxDynamicSharedMemorySize = 8, cudaFuncAttributePreferredSharedMemoryCarveout = 9 };
struct cudaFuncAttributes {
    int numRegs = 0;
};
template <class F> inline cudaError_t cudaFuncSetAttribute(F, cudaFuncAttribute, int) { return cudaSuccess; }
inline cudaError_t cudaFuncGetAttributes(cudaFuncAttributes *, const void *) { return cudaSuccess; }
template <class T> inline cudaError_t cudaGetSymbolAddress(void **p, T &symbol)
{
    *p = static_cast<void *>(&symbol);
    return cudaSuccess;
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

#include "cuda_host_runtime.h"
