// adjoint_common.cuh -- device helpers shared by the adjoint kernels
// (adjoint_prep.cu, adjoint.cu): indexing, the cell-centred B of a stage
// input, and the flux adjoints formed from the adjoint of a stage output.
#pragma once

#include "adjoint.h"
#include "rmhd2d_internal.h"

namespace rmhd2d {
namespace adjk {

constexpr int IF_PLANES = 16;   // per sweep: 7 left adjoints, b_n adjoint, 7 right adjoints, minmod branches
constexpr int Q_PLANES = 9;     // per sweep: the 8 interface primitives of the cell, and its own b_n

__device__ __forceinline__ long long at(const Grid &g, int i, int j) { return (long long)i * g.pitch + j; }

__device__ __forceinline__ bool hydro_field(int f) { return f != BXF && f != BYF; }

// Cell-centred B of W (resistiveMHD_2D.cu:313-368): the first row / column
// keeps its face value.
__device__ __forceinline__ double bx_c(const Grid &g, const double *W, int i, int j)
{
    const double *bX = W + BXF * g.plane;
    return i >= 1 ? __dmul_rn(0.5, __dadd_rn(bX[at(g, i, j)], bX[at(g, i - 1, j)])) : bX[at(g, i, j)];
}
__device__ __forceinline__ double by_c(const Grid &g, const double *W, int i, int j)
{
    const double *bY = W + BYF * g.plane;
    return j >= 1 ? __dmul_rn(0.5, __dadd_rn(bY[at(g, i, j)], bY[at(g, i, j - 1)])) : bY[at(g, i, j)];
}

// Sweep-order slot s -> natural field: x sweeps the cell as is, y as
// (rho, my, mz, mx, bY, bZ, bX, e) (hlld.cu:134-160); fluxes are permuted
// the same way (hlld.cu:200-233).
__device__ __forceinline__ int sweep_field(int dir, int s)
{
    if (dir == 0) return s;
    return s == 1 ? MY : s == 2 ? MZ : s == 3 ? MX : s == 4 ? BYF : s == 5 ? BZF : s == 6 ? BXF : s;
}

// Adjoint of the stage-1 corner EMF Ez(i, j): both CT results (the stage-1
// state and the step output) use it (ct.cu:44-59).
__device__ __forceinline__ double ez_bar(const AdjStageArgs &a, int i, int j)
{
    const Grid &g = a.g;
    if (i < 0 || j < 0 || i > g.nx - 2 || j > g.ny - 2) return 0.0;
    auto b = [&](int f, int ii, int jj) -> double {
        if (ii < 1 || jj < 1 || ii > g.nx - 1 || jj > g.ny - 1) return 0.0;
        const long long k = f * g.plane + at(g, ii, jj);
        return a.Ub[k] + a.UbStep[k];
    };
    return a.dt / g.dy * (b(BXF, i, j + 1) - b(BXF, i, j)) + a.dt / g.dx * (b(BYF, i, j) - b(BYF, i + 1, j));
}

// Adjoint of the x flux F at interface (i, j) (between cells i and i+1),
// natural field order; i + 1 <= nx - 1.  The update
// (resistiveMHD_2D.cu:53-130) subtracts s dt/dx (F_i - F_{i-1}).
__device__ __forceinline__ void f_bar(const AdjStageArgs &a, int i, int j, double *fb)
{
    const Grid &g = a.g;
    const double c = -a.s * a.dt / g.dx;
    const long long k0 = at(g, i, j), k1 = at(g, i + 1, j);
#pragma unroll
    for (int f = 0; f < NFIELD; ++f) fb[f] = hydro_field(f) ? c * (a.Ub[f * g.plane + k0] - a.Ub[f * g.plane + k1]) : 0.0;
    if (a.stage == 1) fb[BYF] = -0.25 * (ez_bar(a, i, j) + ez_bar(a, i, j - 1));
}

// Adjoint of the y flux G at interface (i, j) (between cells j and j+1).
__device__ __forceinline__ void g_bar(const AdjStageArgs &a, int i, int j, double *gb)
{
    const Grid &g = a.g;
    const double c = -a.s * a.dt / g.dy;
    const long long k0 = at(g, i, j), k1 = at(g, i, j + 1);
#pragma unroll
    for (int f = 0; f < NFIELD; ++f) gb[f] = hydro_field(f) ? c * (a.Ub[f * g.plane + k0] - a.Ub[f * g.plane + k1]) : 0.0;
    if (a.stage == 1) gb[BXF] = 0.25 * (ez_bar(a, i, j) + ez_bar(a, i - 1, j));
}

// Interfaces whose flux adjoint can be non-zero: they touch an interior
// cell's update or an interior face's CT.
__device__ __forceinline__ bool iface_live(const Grid &g, int dir, int i, int j)
{
    return dir == 0 ? (i >= 2 && i <= g.nx - 4 && j >= 2 && j <= g.ny - 3)
                    : (i >= 2 && i <= g.nx - 3 && j >= 2 && j <= g.ny - 4);
}

}  // namespace adjk
}  // namespace rmhd2d
