// stage.cuh -- the fused RK2 stage kernel for sm_100a.
//
// One launch performs one stage of the reference's ResistiveMHD2D::oneStepRK2
// (lib_ResistiveMHD_2D_GPU_periodicXY/resistiveMHD_2D.cu:133-195) on the
// interior cells: face -> centre B, primitive recovery, MUSCL-minmod, HLLD
// fluxes in x and y, the resistive eta*J flux terms, the flux-difference
// update, and (stage 1) the corner EMF plus constrained transport of the
// face B.  The stage-2 launch also reduces the CFL rate of the new state for
// the next step's dt and raises the crash flag on a NaN energy.
//
// Data layout: 8 field planes of nx x pitch doubles (index i*pitch + j,
// y contiguous), one allocation per state.  Each CTA owns TI x TJ interior
// cells (one of the tile shapes of rmhd2d_internal.h, e.g. 8 x 32) and
// stages them with a 3-cell halo on every side by one 3-D TMA load
// (box TJ+6 x TI+6 x 8 fields) into shared memory, plus a 2-D TMA load of the
// eta table on the same cells; everything after those loads reads shared
// memory, except the update's read of its own cell of the stage's source
// state (and, in stage 2, of U^n).
//
// The kernel is compiled three times: an "exact" variant (-fmad=false, the
// bits of the reference's sum of six HLLD candidate fluxes), bit-identical to the reference
// evaluated in IEEE binary64; a "fast" FP64 variant (FMA contraction, shared
// reciprocals, only the selected HLLD candidate); and an "FP32-bulk" variant
// (reconstruction and fluxes in single precision, pressure recovery, EMF,
// update and dt in FP64).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>

#include "physics.cuh"
#include "rmhd2d_internal.h"

namespace rmhd2d {

struct StageArgs {
    Grid g;
    const double *src;   // state this stage reads (TMA source, and own cells in the update); stage 2: U*
    const double *un;    // stage 2: U^n (hydro fields read at own cells)
    double *dst;         // planes written (stage 1: U*; stage 2: U^n in place)
    const double *eta;   // cell-centred eta plane or nullptr (uniform g.eta)
    double *row2;        // symmetric boundaries: CT'd bY at j = 2, indexed by i
    Control *ctl;
    int parity;          // step parity: dt from ctl->amax[parity]
    double *dt_log;      // stage 1, or nullptr: the step's dt is also written here (a recorded run)
    const double *dt_in; // or nullptr: the step's dt is read from here (a replayed run), not reduced
};

// One set of launchers per variant (stage_exact.cu, stage_fast.cu, stage_bulk32.cu).
// Sweep of the stage kernel's flux phase (true: x sweep), as a compile-time
// constant (SweepC) or a run-time value (SweepRT).
template <bool F> struct SweepC {
    static constexpr bool value = F;
};
struct SweepRT {
    bool value;
};
// Whether an interface takes the exact variant's rare path (see flux_at).
template <bool B> struct FullC {
    static constexpr bool value = B;
};

namespace exact {
void launch_stage(int stage, int shape, const CUtensorMap *tmap, const CUtensorMap *emap, const StageArgs &args,
                  cudaStream_t stream);
void launch_stage_batch(int stage, int shape, const BatchRun *runs, const CUtensorMap *maps, const TileRef *tiles,
                        int ntiles, int ctas, int parity, cudaStream_t stream);
size_t stage_smem_bytes(int stage, int shape);
int stage_regs(int stage, int shape);
}  // namespace exact
namespace fast {
void launch_stage(int stage, int shape, const CUtensorMap *tmap, const CUtensorMap *emap, const StageArgs &args,
                  cudaStream_t stream);
void launch_stage_batch(int stage, int shape, const BatchRun *runs, const CUtensorMap *maps, const TileRef *tiles,
                        int ntiles, int ctas, int parity, cudaStream_t stream);
size_t stage_smem_bytes(int stage, int shape);
int stage_regs(int stage, int shape);
}  // namespace fast
namespace bulk32 {
void launch_stage(int stage, int shape, const CUtensorMap *tmap, const CUtensorMap *emap, const StageArgs &args,
                  cudaStream_t stream);
void launch_stage_batch(int stage, int shape, const BatchRun *runs, const CUtensorMap *maps, const TileRef *tiles,
                        int ntiles, int ctas, int parity, cudaStream_t stream);
size_t stage_smem_bytes(int stage, int shape);
int stage_regs(int stage, int shape);
}  // namespace bulk32

}  // namespace rmhd2d
