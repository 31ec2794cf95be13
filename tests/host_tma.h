// host_tma.h -- TEST INFRASTRUCTURE.  Builds the tensor maps of the host
// build of the stage kernel (RMHD_HOST_EMULATION; HostMap in
// cuda_host_shim.h): what cuTensorMapEncodeTiled would encode for the
// library's maps (csrc/api.cu: encode_state_map, encode_eta_map).
#pragma once

#include <cstdint>
#include <cstring>

#include "cuda_host_shim.h"

inline CUtensorMap host_map(const double *base, int rank, unsigned long long d0, unsigned long long d1,
                            unsigned long long d2, unsigned long long s0, unsigned long long s1, unsigned b0,
                            unsigned b1, unsigned b2)
{
    HostMap h{base, {d0, d1, d2}, {s0, s1}, {b0, b1, b2}, rank};
    CUtensorMap m{};
    std::memcpy(&m, &h, sizeof h);
    return m;
}
