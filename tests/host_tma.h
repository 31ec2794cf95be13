// host_tma.h -- TEST INFRASTRUCTURE.  The tensor map of the host build of the
// stage kernel (RMHD_HOST_EMULATION): what cuTensorMapEncodeTiled would
// encode for the library's maps (csrc/api.cu: encode_state_map,
// encode_eta_map), held in the bytes of a CUtensorMap.
#pragma once

#include <cstdint>
#include <cstring>

#include "cuda_host_shim.h"

struct HostMap {
    const double *base;
    unsigned long long dims[3];      // innermost first: j (ny), i (nx), field (8)
    unsigned long long strides[2];   // bytes between consecutive i, between fields
    unsigned box[3];                 // box extent per dimension
    int rank;                        // 2 or 3
};
static_assert(sizeof(HostMap) <= sizeof(CUtensorMap), "a host map fits a tensor map's bytes");

inline CUtensorMap host_map(const double *base, int rank, unsigned long long d0, unsigned long long d1,
                            unsigned long long d2, unsigned long long s0, unsigned long long s1, unsigned b0,
                            unsigned b1, unsigned b2)
{
    HostMap h{base, {d0, d1, d2}, {s0, s1}, {b0, b1, b2}, rank};
    CUtensorMap m{};
    std::memcpy(&m, &h, sizeof h);
    return m;
}
