// rmhd2d_internal.h -- shared between the C-ABI host code and the CUDA
// kernels of librmhd2d.  Not part of the public interface (include/rmhd2d.h).
#pragma once

#include <cstddef>
#include <cstdint>

namespace rmhd2d {

// Field order of a cell, identical to the reference's ConservationParameter
// (lib_ResistiveMHD_2D_GPU_periodicXY/conservation_parameter_struct.hpp:5-27).
enum Field { RHO = 0, MX = 1, MY = 2, MZ = 3, BXF = 4, BYF = 5, BZF = 6, EN = 7, NFIELD = 8 };

enum Bc { BC_PERIODIC = 0, BC_SYMMETRIC = 1 };

// Geometry and physics constants passed by value to every kernel.
struct Grid {
    int nx, ny;          // cells incl. 3 ghost layers per side
    int pitch;           // doubles between consecutive i rows of a plane (>= ny, multiple of 32)
    long long plane;     // doubles per field plane = nx * pitch
    double dx, dy;
    double gamma, cfl, eps, eta;
    int bc_x, bc_y;      // Bc of the x walls (i) and the y walls (j)
};

// Device-side control block (one per solver), zero-initialised at create.
struct Control {
    unsigned long long amax[2];  // max over cells of |u|/dx + |v|/dy terms (raw bits, NaN skipped), per step parity
    int first_nan[2];            // cell k = 0 had a NaN dt candidate, per step parity
    double dt;                   // dt of the most recent step (reference's global dt)
    double total_time;           // sum of dt over the steps taken
    int crashed;                 // NaN energy seen in the newest state
    int error;                   // kernel-side error code (bounded wait expired, ...)
};

enum KernelError { KERR_NONE = 0, KERR_TMA_TIMEOUT = 1 };

// Tiles of the fused stage kernels: TI cells along x (i) by TJ along y (j).
// Stage 1 also computes the ring of fluxes its corner EMF needs, stage 2
// only the tile's own interfaces, so their best tile heights differ: with
// 320 threads stage 1 (8 x 32) has 636 interfaces and stage 2 (9 x 32) 617,
// two nearly full rounds each.
constexpr int TJ = 32;
constexpr int HALO = 3;
constexpr int STAGE1_TI = 8;
constexpr int STAGE2_TI = 9;
constexpr int UJ = TJ + 2 * HALO;  // staged columns (TMA inner box: UJ * 8 bytes, multiple of 16)
constexpr int STAGE_THREADS = 320;
static_assert(STAGE_THREADS >= STAGE1_TI * TJ && STAGE_THREADS >= STAGE2_TI * TJ,
              "one thread per tile cell in the update phase");
constexpr int stage_ti(int stage) { return stage == 1 ? STAGE1_TI : STAGE2_TI; }
constexpr int stage_ui(int stage) { return stage_ti(stage) + 2 * HALO; }

}  // namespace rmhd2d
