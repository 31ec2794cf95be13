// adjoint.h -- launchers of the discrete-adjoint kernels (adjoint.cu).
#pragma once

#include <cuda_runtime.h>

#include "rmhd2d_internal.h"

namespace rmhd2d {

// One stage of the reverse sweep.  All arrays are pitched planes of the
// grid g (8 planes for states and their adjoints).
struct AdjStageArgs {
    Grid g;
    const double *W;       // the stage's input state (U^n for stage 1, U* for stage 2)
    const double *Ub;      // adjoint of the stage's output, boundary already transposed
    const double *UbStep;  // stage 1: adjoint of the step's output (its CT faces share the stage-1 EMF)
    const double *eta;     // eta plane, or nullptr for the uniform g.eta
    double *Q;             // 18 planes: interface primitives of each cell and its own b_n (x sweep, then y sweep)
    double *IF;            // 32 planes of per-interface adjoints (x sweep, then y sweep)
    double *RJ;            // 6 planes: adjoints of J_x, J_y, J_z and direct B adjoints of the eta*J terms
    double *tmp;           // 2 planes: adjoint of the cell-centred bX, bY
    double *etab;          // adjoint of the eta field, accumulated
    double *Ustage;        // stage 2: receives the adjoint of U*
    double *Uin;           // adjoint of U^n: set by stage 2, accumulated by stage 1
    double dt;             // the step's dt
    double s;              // weight of the flux difference: 1 (stage 1), 0.5 (stage 2)
    int stage;             // 1 or 2
};

void launch_adjoint_stage(const AdjStageArgs &a, cudaStream_t st);
// Transpose of the periodic x and y ghost fill, in place: ghost adjoints are
// added to the interior cells they were copied from and cleared.
void launch_boundary_transpose(const Grid &g, double *Ub, cudaStream_t st);
void launch_plane_to_table(const Grid &g, const double *plane, double *tab, cudaStream_t st);

}  // namespace rmhd2d
