// Fast variant of the fused stage kernel: FMA contraction, the HLLD flux with
// shared reciprocals and only the selected candidate fluxes
// (hlld_flux_fast), reciprocal multiplications for the primitive recovery,
// the current density and the CFL rate.  Differs from the exact variant by
// rounding only.
#define RMHD_VARIANT fast
#define RMHD_FAST_MATH 1
#include "stage_impl.cuh"
