// host_tma.cpp -- TEST INFRASTRUCTURE.  Host definitions of the stage
// kernel's staging primitives (resistivemhd_gpu_b200/csrc/tma_ptx.cuh) for
// its CPU build.  The mbarrier is modelled by two words: the number of
// completed phases and the bytes still expected in the current one
// (expect_tx sets them; each tensor load copies its box synchronously, with
// 0 for the elements outside the tensor as the maps' OOB fill gives, and
// counts its bytes off).  A wait tries until the phase it names has
// completed.  The stage kernel reserves 16 bytes for its barrier.
#include <atomic>
#include <chrono>
#include <new>
#include <thread>

#include "host_tma.h"
#include "tma_ptx.cuh"

namespace rmhd2d {

namespace {

std::atomic<unsigned long long> &phases(uint64_t *bar)
{
    return *reinterpret_cast<std::atomic<unsigned long long> *>(bar);
}

std::atomic<long long> &pending(uint64_t *bar)
{
    return *reinterpret_cast<std::atomic<long long> *>(bar + 1);
}

void complete_bytes(uint64_t *bar, long long bytes)
{
    if (pending(bar).fetch_sub(bytes) == bytes) phases(bar).fetch_add(1ull);
}

long long load_box(double *dst, const CUtensorMap *map, long long x, long long y, long long z)
{
    HostMap h;
    std::memcpy(&h, map, sizeof h);
    const unsigned nz = h.rank == 3 ? h.box[2] : 1;
    for (unsigned c = 0; c < nz; ++c)
        for (unsigned b = 0; b < h.box[1]; ++b)
            for (unsigned a = 0; a < h.box[0]; ++a) {
                const long long gx = x + a, gy = y + b, gz = z + c;
                double v = 0.0;
                if (gx >= 0 && gy >= 0 && gz >= 0 && gx < (long long)h.dims[0] && gy < (long long)h.dims[1] &&
                    (h.rank == 2 || gz < (long long)h.dims[2]))
                    v = h.base[(gz * (long long)h.strides[1] + gy * (long long)h.strides[0]) / 8 + gx];
                dst[((size_t)c * h.box[1] + b) * h.box[0] + a] = v;
            }
    return (long long)nz * h.box[1] * h.box[0] * 8;
}

}  // namespace

void mbar_init_tile(uint64_t *bar)
{
    new (bar) std::atomic<unsigned long long>(0ull);
    new (bar + 1) std::atomic<long long>(0);
}

// One try polls for up to 2 ms, so the kernel's bound of 50,000 tries (about
// a second on the device) becomes about 100 s here: loaded test machines
// and sanitizer builds stay well inside it.
bool mbar_try_wait(uint64_t *bar, uint32_t phase)
{
    const auto until = std::chrono::steady_clock::now() + std::chrono::milliseconds(2);
    do {
        if ((phases(bar).load() & 1ull) != phase) return true;
        std::this_thread::yield();
    } while (std::chrono::steady_clock::now() < until);
    return false;
}

void fence_proxy_async() {}

void mbar_expect_tx(uint64_t *bar, uint32_t bytes) { pending(bar).store((long long)bytes); }

void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y, int z)
{
    complete_bytes(bar, load_box(static_cast<double *>(dst), map, x, y, z));
}

void tma_load_2d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y)
{
    complete_bytes(bar, load_box(static_cast<double *>(dst), map, x, y, 0));
}

void prefetch_l2(const void *) {}

}  // namespace rmhd2d
