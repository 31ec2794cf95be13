// stage_host.cpp -- TEST INFRASTRUCTURE.  The stage-1-EMF RK2 step of the C
// ABI run on the CPU over the fused stage kernel's own source (the exact
// variant, stage_exact.cu) and the ghost-fill / CFL kernels
// (aux_kernels.cu), compiled for the host through cuda_host_shim.h with the
// tile staging of host_tma.cpp.  The set-up mirrors rmhd2d_create +
// rmhd2d_set_state(apply_boundary = 1), the tensor maps those of
// encode_state_map / encode_eta_map, and each step enqueue_step
// (resistivemhd_gpu_b200/csrc/api.cu).
#include <vector>

#include "aux_kernels.h"
#include "host_tma.h"
#include "physics.cuh"
#include "rmhd2d_internal.h"
#include "stage.cuh"

using namespace rmhd2d;

extern "C" {

// nsteps steps from the reference-layout state (updated in place; the
// boundary is applied first), each step's dt in dts, with the stage kernels'
// tile shape `shape`.  Returns 0, or 1 + the step whose output raised the
// crash flag.
int host_stage_run(int nx, int ny, double dx, double dy, double gamma, double cfl, double eps, double eta, int bc_x,
                   int bc_y, const double *eta_table, int shape, double *state, int nsteps, double *dts)
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
    const size_t P = (size_t)g.plane, sd = P * NFIELD;
    std::vector<double> A(sd, 0.0), B(sd, 0.0), row2((size_t)nx, 0.0), eta_plane;
    if (eta_table) {
        eta_plane.assign(P, 0.0);
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) eta_plane[(size_t)i * g.pitch + j] = eta_table[(size_t)j + (size_t)i * ny];
    }
    const unsigned long long st0 = (unsigned long long)g.pitch * 8, st1 = (unsigned long long)P * 8;
    const unsigned uj = (unsigned)shape_uj(shape), ui1 = (unsigned)stage_ui(1, shape), ui2 = (unsigned)stage_ui(2, shape);
    const CUtensorMap mapA = host_map(A.data(), 3, ny, nx, NFIELD, st0, st1, uj, ui1, NFIELD);
    const CUtensorMap mapB = host_map(B.data(), 3, ny, nx, NFIELD, st0, st1, uj, ui2, NFIELD);
    const double *ep = eta_table ? eta_plane.data() : nullptr;
    const CUtensorMap mapE1 = host_map(ep, 2, ny, nx, 1, st0, 0, uj, ui1, 1);
    const CUtensorMap mapE2 = host_map(ep, 2, ny, nx, 1, st0, 0, uj, ui2, 1);

    Control ctl{};
    launch_aos_to_planes(g, state, A.data(), nullptr);
    if (g.bc_x == BC_SYMMETRIC) launch_snapshot_row2(g, A.data(), row2.data(), nullptr);
    launch_boundary(g, A.data(), row2.data(), nullptr, 0, nullptr);
    int parity = 0;
    launch_rate(g, A.data(), &ctl, parity, 1, nullptr);
    int rc = 0;
    for (int n = 0; n < nsteps; ++n) {
        StageArgs a{};
        a.g = g;
        a.eta = ep;
        a.row2 = g.bc_x == BC_SYMMETRIC ? row2.data() : nullptr;
        a.ctl = &ctl;
        a.parity = parity;
        a.src = A.data();
        a.un = A.data();
        a.dst = B.data();
        exact::launch_stage(1, shape, &mapA, &mapE1, a, nullptr);
        launch_boundary(g, B.data(), row2.data(), nullptr, 0, nullptr);
        a.src = B.data();
        a.un = A.data();
        a.dst = A.data();
        exact::launch_stage(2, shape, &mapB, &mapE2, a, nullptr);
        launch_boundary(g, A.data(), row2.data(), &ctl, parity ^ 1, nullptr);
        dts[n] = ctl.dt;
        parity ^= 1;
        if (ctl.error) return -1;
        if (ctl.crashed) {
            rc = 1 + n;
            break;
        }
    }
    launch_planes_to_aos(g, A.data(), state, nullptr);
    return rc;
}

}  // extern "C"
