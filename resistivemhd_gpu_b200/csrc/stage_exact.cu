// Exact variant of the fused stage kernel: compiled with -fmad=false, every
// operation rounds exactly as the reference's functors do in IEEE binary64,
// and the HLLD flux has the bits of the reference's weighted sum of six
// candidate fluxes (physics.cuh hlld_flux_sel / hlld_flux_ieee).
#define RMHD_VARIANT exact
#include "stage_impl.cuh"
