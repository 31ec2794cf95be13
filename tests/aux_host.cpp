// aux_host.cpp -- TEST INFRASTRUCTURE.  Entry points over the host builds of
// aux_kernels.cu (ghost fill, CFL rate and crash flag, layout conversions)
// and noalloc_dt.cu (the allocation-free dt), compiled through
// cuda_host_shim.h, for tests/test_aux_host.py.  Each mirrors what the C ABI
// does with these launchers (resistivemhd_gpu_b200/csrc/api.cu): set_state
// with the boundary applied, the CFL reduction of refresh_rate and
// rmhd2d_calculate_dt, and rmhd2d_calculate_dt_noalloc.
#include <cstring>
#include <vector>

#include "aux_kernels.h"
#include "noalloc_dt.h"
#include "physics.cuh"
#include "rmhd2d_internal.h"

using namespace rmhd2d;

namespace {

Grid make_grid(int nx, int ny, double dx, double dy, double gamma, double cfl, double eps, double eta, int bc_x,
               int bc_y)
{
    Grid g{};
    g.nx = nx;
    g.ny = ny;
    g.pitch = (ny + 31) / 32 * 32;
    g.plane = (long long)nx * g.pitch;
    g.dx = dx;
    g.dy = dy;
    g.gamma = gamma;
    g.cfl = cfl;
    g.eps = eps;
    g.eta = eta;
    g.bc_x = bc_x;
    g.bc_y = bc_y < 0 ? bc_x : bc_y;
    return g;
}

}  // namespace

extern "C" {

// The state (reference layout, in place) through the library's layout
// conversion and ghost fill, as rmhd2d_set_state(apply_boundary = 1) leaves
// it, then the CFL reduction over every cell: *dt is rmhd2d_calculate_dt's
// value and *crashed its crash flag.  With `ghost_rates`, the ghost fill
// also folds the ghosts' rates into a second control block, whose maximum
// is returned in *ghost_amax.
int host_set_state_dt(int nx, int ny, double dx, double dy, double gamma, double cfl, double eps, double eta, int bc_x,
                      int bc_y, double *state, double *dt, int *crashed, int ghost_rates,
                      unsigned long long *ghost_amax)
{
    const Grid g = make_grid(nx, ny, dx, dy, gamma, cfl, eps, eta, bc_x, bc_y);
    const size_t sd = (size_t)g.plane * NFIELD;
    std::vector<double> A(sd, 0.0), row2((size_t)nx, 0.0);
    launch_aos_to_planes(g, state, A.data(), nullptr);
    Control gc{};
    if (g.bc_x == BC_SYMMETRIC) launch_snapshot_row2(g, A.data(), row2.data(), nullptr);
    launch_boundary(g, A.data(), row2.data(), ghost_rates ? &gc : nullptr, 0, nullptr);
    if (ghost_amax) *ghost_amax = gc.amax[0];
    Control ctl{};
    launch_rate(g, A.data(), &ctl, 0, 1, nullptr);
    *dt = step_dt(ctl.amax[0], ctl.first_nan[0], g.dx, g.dy, g.eps, g.eta, g.cfl);
    *crashed = ctl.crashed;
    launch_planes_to_aos(g, A.data(), state, nullptr);
    return 0;
}

// rmhd2d_calculate_dt_noalloc's reduction over a reference-layout state.
int host_dt_noalloc(int nx, int ny, double dx, double dy, double gamma, double cfl, double eps, double eta,
                    const double *state, double *dt)
{
    unsigned long long *scratch = nullptr;
    if (noalloc_scratch(&scratch) != cudaSuccess) return 1;
    double out = 0.0;
    if (enqueue_dt_noalloc(state, (long long)nx * ny, gamma, dx, dy, eps, eta, cfl, scratch, &out, nullptr) !=
        cudaSuccess)
        return 2;
    *dt = out;
    return 0;
}

}  // extern "C"
