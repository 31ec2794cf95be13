// noalloc_dt.h -- the allocation-free CFL dt reduction (noalloc_dt.cu).
#pragma once

#include <cuda_runtime.h>

namespace rmhd2d {

// Device address of the file-scope scratch array on the current device,
// looked up with cudaGetSymbolAddress on every call (no cache that a context
// reset could leave dangling).
cudaError_t noalloc_scratch(unsigned long long **ptr);

// Enqueues on `st`: the clear of the completion counter, the reduction over
// ncell cells of the array-of-structures state `aos`, and the copy of the dt
// into *dt_host.  The caller synchronises `st` before reading *dt_host.
cudaError_t enqueue_dt_noalloc(const double *aos, long long ncell, double gm, double dx, double dy, double eps,
                               double eta, double cfl, unsigned long long *scratch, double *dt_host,
                               cudaStream_t st);

}  // namespace rmhd2d
