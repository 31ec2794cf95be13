// FP32-bulk variant of the fused stage kernel: MUSCL reconstruction, the HLLD
// flux and the eta*J terms in single precision (hlld_flux_bulk),
// while the pressure recovery from the total energy, the corner-EMF
// accumulation, the flux-difference update and the CFL reduction stay in
// FP64 and the state is stored in FP64.  Compiled with --use_fast_math,
// which affects single-precision operations only.
#define RMHD_VARIANT bulk32
#define RMHD_FAST_MATH 1
#define RMHD_REAL float
#define RMHD_BULK 1
#include "stage_impl.cuh"
