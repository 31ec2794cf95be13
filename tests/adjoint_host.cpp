// adjoint_host.cpp -- TEST INFRASTRUCTURE.  The reverse sweep of the C
// ABI's rmhd2d_adjoint_backward (resistivemhd_gpu_b200/csrc/api.cu), run on
// the CPU over the adjoint kernels' own source (adjoint.cu, adjoint_prep.cu,
// compiled for the host through cuda_host_shim.h), with the forward
// trajectory supplied by the caller (the oracle's, which is bit-identical to
// the FP64-exact CUDA step) instead of checkpoints and recomputation.
#include <cstring>
#include <vector>

#include "adjoint.h"
#include "rmhd2d_internal.h"

using namespace rmhd2d;

namespace {

Grid make_grid(int nx, int ny, double dx, double dy, double gamma, double eps, double eta, int bc_x, int bc_y)
{
    Grid g{};
    g.nx = nx;
    g.ny = ny;
    g.pitch = (ny + 31) / 32 * 32;
    g.plane = (long long)nx * g.pitch;
    g.dx = dx;
    g.dy = dy;
    g.gamma = gamma;
    g.cfl = 0.0;
    g.eps = eps;
    g.eta = eta;
    g.bc_x = bc_x;
    g.bc_y = bc_y < 0 ? bc_x : bc_y;
    return g;
}

// Reference layout (cell k = j + i*ny, 8 doubles) -> 8 pitched planes.
void aos_to_planes(const Grid &g, const double *aos, double *planes)
{
    for (int f = 0; f < NFIELD; ++f)
        for (int i = 0; i < g.nx; ++i)
            for (int j = 0; j < g.ny; ++j)
                planes[f * g.plane + (long long)i * g.pitch + j] = aos[((long long)j + (long long)i * g.ny) * NFIELD + f];
}

void planes_to_aos(const Grid &g, const double *planes, double *aos)
{
    for (int f = 0; f < NFIELD; ++f)
        for (int i = 0; i < g.nx; ++i)
            for (int j = 0; j < g.ny; ++j)
                aos[((long long)j + (long long)i * g.ny) * NFIELD + f] = planes[f * g.plane + (long long)i * g.pitch + j];
}

}  // namespace

extern "C" {

// dJ/dU_0 and dJ/d eta of nsteps frozen-dt steps for the seed dJ/dU_N.
// un, ustar: nsteps states each (reference layout), the state step s starts
// from and its stage-1 state after the boundary pass; dts: the steps' dts;
// eta_table: nx*ny cell-centred eta or NULL for the uniform eta; grad_eta:
// nx*ny.  Mirrors the reverse loop of rmhd2d_adjoint_backward.
int host_adjoint_backward(int nx, int ny, double dx, double dy, double gamma, double eps, double eta, int bc_x,
                          int bc_y, const double *eta_table, int nsteps, const double *un, const double *ustar,
                          const double *dts, const double *seed, double *grad_state, double *grad_eta)
{
    const Grid g = make_grid(nx, ny, dx, dy, gamma, eps, eta, bc_x, bc_y);
    const size_t P = (size_t)g.plane, sd = P * NFIELD, naos = (size_t)nx * ny * NFIELD;
    std::vector<double> eta_plane, W0(sd, 0.0), W1(sd, 0.0), Q(18 * P, 0.0), IF(32 * P, 0.0), RJ(6 * P, 0.0),
        tmp(2 * P, 0.0), etab(P, 0.0);
    std::vector<double> ub[3] = {std::vector<double>(sd, 0.0), std::vector<double>(sd, 0.0),
                                 std::vector<double>(sd, 0.0)};
    if (eta_table) {
        eta_plane.assign(P, 0.0);
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) eta_plane[(size_t)i * g.pitch + j] = eta_table[(size_t)j + (size_t)i * ny];
    }
    aos_to_planes(g, seed, ub[0].data());
    cudaStream_t st = nullptr;
    int cur = 0;
    for (int n = nsteps - 1; n >= 0; --n) {
        aos_to_planes(g, un + (size_t)n * naos, W0.data());
        aos_to_planes(g, ustar + (size_t)n * naos, W1.data());
        const int mid = (cur + 1) % 3, nxt = (cur + 2) % 3;
        AdjStageArgs a{};
        a.g = g;
        a.eta = eta_table ? eta_plane.data() : nullptr;
        a.Q = Q.data();
        a.IF = IF.data();
        a.RJ = RJ.data();
        a.tmp = tmp.data();
        a.etab = etab.data();
        a.dt = dts[n];
        launch_boundary_transpose(g, ub[cur].data(), st);
        a.W = W1.data();
        a.Ub = ub[cur].data();
        a.UbStep = ub[cur].data();
        a.Ustage = ub[mid].data();
        a.Uin = ub[nxt].data();
        a.s = 0.5;
        a.stage = 2;
        launch_adjoint_stage(a, st);
        launch_boundary_transpose(g, ub[mid].data(), st);
        a.W = W0.data();
        a.Ub = ub[mid].data();
        a.UbStep = ub[cur].data();
        a.Ustage = nullptr;
        a.s = 1.0;
        a.stage = 1;
        launch_adjoint_stage(a, st);
        cur = nxt;
    }
    // the boundary applied when the initial state was set
    launch_boundary_transpose(g, ub[cur].data(), st);
    planes_to_aos(g, ub[cur].data(), grad_state);
    if (grad_eta) {
        std::vector<double> tab((size_t)nx * ny);
        launch_plane_to_table(g, etab.data(), tab.data(), st);
        std::memcpy(grad_eta, tab.data(), tab.size() * sizeof(double));
    }
    return 0;
}

}  // extern "C"
