// Exact variant of the fused stage kernel: compiled with -fmad=false and all
// six HLLD candidate fluxes formed, so every operation rounds exactly as the
// reference's functors do in IEEE binary64.
#define RMHD_VARIANT exact
#define RMHD_ALL_CANDIDATES true
#include "stage_impl.cuh"
