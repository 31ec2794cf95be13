// division_check.cu -- checks MdDiv (physics.cuh), the shared-reciprocal
// division of the exact arithmetic, against IEEE division on random and
// special operands.  Built by tests/test_division.py twice: with nvcc for
// sm_100a (the hardware reciprocal seed) and with g++ as host code under
// RMHD_HOST_EMULATION through the host shim (tests/host_build.py: shim_dir),
// with the emulated seed.
//
//   division_check <n_random> <seed>
// prints "checked <n> accepted <n_ok> mismatches <n_bad>"; a mismatch is an
// operand pair whose guard held but whose quotient's bits differ from a / b.
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "physics.cuh"

using namespace rmhd2d;

__host__ __device__ inline unsigned long long mix(unsigned long long z)
{
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Operand k of a sample: random sign and significand, exponent drawn from a
// range a little wider than the guard's, plus significands of all ones,
// powers of two, zeros of both signs and dividends close to the divisor.
__host__ __device__ inline void operands(unsigned long long seed, unsigned long long k, double &a, double &b)
{
    const unsigned long long r0 = mix(seed ^ (k * 2 + 1)), r1 = mix(r0), r2 = mix(r1), r3 = mix(r2);
    const int eb = (int)(r2 % 1000) - 500, ea = (int)(r3 % 1200) - 600;
    unsigned long long mb = r0 & 0xFFFFFFFFFFFFFull, ma = r1 & 0xFFFFFFFFFFFFFull;
    switch (k & 15) {
    case 0: mb = 0xFFFFFFFFFFFFFull; break;                 // all-ones divisor
    case 1: ma = 0; break;                                  // power-of-two dividend
    case 2: mb = 0; break;                                  // power-of-two divisor
    case 3: ma = mb ^ (r3 & 0x3F); break;                   // dividend near the divisor
    default: break;
    }
    unsigned long long ub = ((r2 >> 40) & 1ull) << 63 | (unsigned long long)(eb + 1023) << 52 | mb;
    unsigned long long ua = ((r3 >> 40) & 1ull) << 63 | (unsigned long long)(ea + 1023) << 52 | ma;
    if ((k & 255) == 4) ua = (r3 & 1ull) << 63;             // +-0 dividend
    if ((k & 15) == 3) ua = (ua & ~(0x7FFull << 52)) | (ub & (0x7FFull << 52));
    memcpy(&a, &ua, 8);
    memcpy(&b, &ub, 8);
}

__device__ inline void check_one(unsigned long long seed, unsigned long long k, unsigned long long &ok,
                                          unsigned long long &bad)
{
    double a, b;
    operands(seed, k, a, b);
    MdDiv md;
    const double y = md.recip(b);
    const double q = md.div(a, b, y);
    const double ref = a / b;
    if (md.ok) {
        ++ok;
        unsigned long long uq, ur;
        memcpy(&uq, &q, 8);
        memcpy(&ur, &ref, 8);
        if (uq != ur) ++bad;
    }
}

#ifdef __CUDACC__
__global__ void check_kernel(unsigned long long seed, unsigned long long n, unsigned long long *counts)
{
    unsigned long long ok = 0, bad = 0;
    for (unsigned long long k = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; k < n;
         k += (unsigned long long)gridDim.x * blockDim.x)
        check_one(seed, k, ok, bad);
    atomicAdd(&counts[0], ok);
    atomicAdd(&counts[1], bad);
}
#endif

int main(int argc, char **argv)
{
    const unsigned long long n = argc > 1 ? strtoull(argv[1], nullptr, 10) : 1000000ull;
    const unsigned long long seed = argc > 2 ? strtoull(argv[2], nullptr, 10) : 1ull;
    unsigned long long counts[2] = {0, 0};
#ifdef __CUDACC__
    unsigned long long *d = nullptr;
    if (cudaMalloc(&d, sizeof(counts)) != cudaSuccess) return 2;
    cudaMemset(d, 0, sizeof(counts));
    check_kernel<<<148 * 8, 256>>>(seed, n, d);
    if (cudaMemcpy(counts, d, sizeof(counts), cudaMemcpyDeviceToHost) != cudaSuccess) return 2;
    cudaFree(d);
#else
    for (unsigned long long k = 0; k < n; ++k) check_one(seed, k, counts[0], counts[1]);
#endif
    std::printf("checked %llu accepted %llu mismatches %llu\n", n, counts[0], counts[1]);
    return 0;
}
