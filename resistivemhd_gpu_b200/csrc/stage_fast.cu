// Fast variant of the fused stage kernel: FMA contraction allowed and only the
// HLLD candidate fluxes whose indicator is set are formed.
#define RMHD_VARIANT fast
#define RMHD_ALL_CANDIDATES false
#include "stage_impl.cuh"
