// rmhd2d_internal.h -- shared between the C-ABI host code and the CUDA
// kernels of librmhd2d.  Not part of the public interface (include/rmhd2d.h).
#pragma once

#include <cstddef>
#include <cstdint>

namespace rmhd2d {

// Field order of a cell, identical to the reference's ConservationParameter
// (lib_ResistiveMHD_2D_GPU_periodicXY/conservation_parameter_struct.hpp:5-27).
enum Field { RHO = 0, MX = 1, MY = 2, MZ = 3, BXF = 4, BYF = 5, BZF = 6, EN = 7, NFIELD = 8 };

// Wall kinds: the single-GPU libraries' periodic and mirror (symmetric)
// walls, and the multi-GPU library's zero-gradient copy, conducting wall (y)
// and flare wall (x).
enum Bc { BC_PERIODIC = 0, BC_SYMMETRIC = 1, BC_ZERO_GRADIENT = 2, BC_WALL = 3, BC_FLARE = 4 };

// Geometry and physics constants passed by value to every kernel.
struct Grid {
    int nx, ny;          // cells incl. 3 ghost layers per side
    int pitch;           // doubles between consecutive i rows of a plane (>= ny, multiple of 32)
    long long plane;     // doubles per field plane = nx * pitch
    double dx, dy;
    double gamma, cfl, eps, eta;
    int bc_x, bc_y;      // Bc of the x walls (i) and the y walls (j)
    // Slab of a decomposed domain: bit 0 (bit 1) set when the 3 columns
    // i < 3 (i >= nx-3) are the halo of the neighbouring slab, filled by the
    // host's exchange and read as interior columns; the x wall applies only
    // on the other sides.  0 for a whole domain.
    int x_halo;
};

// Device-side control block (one per solver), zero-initialised at create.
struct Control {
    unsigned long long amax[2];  // max over cells of |u|/dx + |v|/dy terms (raw bits, NaN skipped), per step parity
    int first_nan[2];            // cell k = 0 had a NaN dt candidate, per step parity
    double dt;                   // dt of the most recent step (reference's global dt)
    double total_time;           // sum of dt over the steps taken
    int crashed;                 // NaN energy seen in the newest state
    int error;                   // kernel-side error code (bounded wait expired, ...)
    double dt_fixed;             // dt of the next step when use_fixed_dt is set
    int use_fixed_dt;            // 1: steps take dt_fixed instead of the CFL dt (frozen-dt runs)
};

enum KernelError { KERR_NONE = 0, KERR_TMA_TIMEOUT = 1 };

// Tiles of the fused stage kernels: TI cells along x (i) by TJ along y (j).
// Stage 1 also computes the ring of fluxes its corner EMF needs, stage 2
// only the tile's own interfaces, so their best tile heights differ.
//   shape 0: stage 1  8 x 32 (636 interfaces), stage 2  9 x 32 (617); 320 threads, 2 CTAs per SM
//   shape 1: stage 1 16 x 16 (612 interfaces), stage 2 18 x 16 (610); 320 threads, 2 CTAs per SM
//   shape 2: stage 1 16 x 32 (1172),           stage 2 18 x 32 (1202); 640 threads, 1 CTA per SM
//   shape 3: stage 1  8 x 64 (1244),           stage 2  8 x 64 (1096); 512 threads, 1 CTA per SM
//   shape 4: stage 1  8 x 32 (636),            stage 2  8 x 32 (552);  256 threads, 3 CTAs per SM
//   shape 5: stage 1  6 x 32 (502),            stage 2  7 x 32 (487);  256 threads, 3 CTAs per SM
// Shape 2 forms 2.29 (stage 1) and 2.09 (stage 2) interfaces per cell
// against 2.48 and 2.14, at the same 20 warps per SM, but one CTA per SM
// leaves no second CTA to run while the first waits at a barrier.  Shape 3
// gives each thread 128 registers (16 warps per SM), shape 4 80 (24 warps
// in three CTAs).  Shape 5 is shape 4 with fewer rows: each stage's
// interfaces fit two passes of its 256 threads, where shape 4 needs a
// third pass that leaves most of its threads idle (stage 2: 40 of 256).
// Which is fastest for a variant and grid is the autotuners' question.
constexpr int HALO = 3;
constexpr int NSHAPE = 6;
constexpr int shape_tj(int shape) { return shape == 1 ? 16 : shape == 3 ? 64 : 32; }
constexpr int stage_ti(int stage, int shape)
{
    return shape == 0 ? (stage == 1 ? 8 : 9)
         : shape == 5 ? (stage == 1 ? 6 : 7)
         : shape >= 3 ? 8 : (stage == 1 ? 16 : 18);
}
constexpr int stage_ui(int stage, int shape) { return stage_ti(stage, shape) + 2 * HALO; }
constexpr int shape_uj(int shape) { return shape_tj(shape) + 2 * HALO; }  // TMA inner box: UJ * 8 B, a multiple of 16
constexpr int shape_threads(int shape) { return shape == 2 ? 640 : shape == 3 ? 512 : shape >= 4 ? 256 : 320; }
constexpr int shape_max_ctas(int shape) { return shape == 2 || shape == 3 ? 1 : shape >= 4 ? 3 : 2; }   // CTAs per SM that fit
constexpr bool shapes_have_a_thread_per_cell()
{
    for (int s = 0; s < NSHAPE; ++s)
        if (shape_threads(s) < stage_ti(2, s) * shape_tj(s) || shape_threads(s) < stage_ti(1, s) * shape_tj(s))
            return false;
    return true;
}
static_assert(shapes_have_a_thread_per_cell(), "one thread per tile cell in the update phase");

// Per-run record of a batch (device memory), and one entry of a batch's tile
// table.
struct BatchRun {
    Grid g;
    double *A, *B, *eta, *row2;
    Control *ctl;
};
struct TileRef {
    int run, ti, tj, pad;
};
// Tensor maps of one run in a batch: [stage-1 state A, stage-2 state B,
// stage-1 eta, stage-2 eta].
constexpr int MAPS_PER_RUN = 4;

}  // namespace rmhd2d
