// stage_host.cpp -- TEST INFRASTRUCTURE.  The stage-1-EMF RK2 step of the C
// ABI run on the CPU over the fused stage kernel's own source (the variant
// STAGE_VARIANT names: stage_exact.cu, stage_fast.cu or stage_bulk32.cu)
// and the ghost-fill / CFL kernels
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

// The kernel variant this driver steps (exact, fast or bulk32).
#ifndef STAGE_VARIANT
#define STAGE_VARIANT exact
#endif

using namespace rmhd2d;

extern "C" {

// nsteps steps from the reference-layout state (updated in place; with
// apply_boundary the boundary is applied first, as set_state does), each
// step's dt in dts, with the stage kernels' tile shape `shape`.  With
// fixed_dts the steps take those dts (rmhd2d_run_fixed_dt) instead of the
// CFL dt.  Returns 0, or 1 + the step whose output raised the crash flag.
int host_stage_run(int nx, int ny, double dx, double dy, double gamma, double cfl, double eps, double eta, int bc_x,
                   int bc_y, const double *eta_table, int shape, double *state, int nsteps, double *dts,
                   int apply_boundary, const double *fixed_dts)
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
    if (apply_boundary) {
        if (g.bc_x == BC_SYMMETRIC) launch_snapshot_row2(g, A.data(), row2.data(), nullptr);
        launch_boundary(g, A.data(), row2.data(), nullptr, 0, nullptr);
    }
    int parity = 0;
    launch_rate(g, A.data(), &ctl, parity, 1, nullptr);
    int rc = 0;
    for (int n = 0; n < nsteps; ++n) {
        ctl.use_fixed_dt = fixed_dts ? 1 : 0;
        if (fixed_dts) ctl.dt_fixed = fixed_dts[n];
        StageArgs a{};
        a.g = g;
        a.eta = ep;
        a.row2 = g.bc_x == BC_SYMMETRIC ? row2.data() : nullptr;
        a.ctl = &ctl;
        a.parity = parity;
        a.src = A.data();
        a.un = A.data();
        a.dst = B.data();
        STAGE_VARIANT::launch_stage(1, shape, &mapA, &mapE1, a, nullptr);
        launch_boundary(g, B.data(), row2.data(), nullptr, 0, nullptr);
        a.src = B.data();
        a.un = A.data();
        a.dst = A.data();
        STAGE_VARIANT::launch_stage(2, shape, &mapB, &mapE2, a, nullptr);
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

// A batch of `nruns` runs (per run: nx, ny, dx, dy, eta, bc_x, bc_y; the
// states concatenated in `states`, updated in place) stepped nsteps times
// as rmhd2d_batch_run steps them, with `ctas` persistent CTAs per stage
// launch; dts[r * nsteps + n] is run r's dt of step n.  gamma, cfl and eps
// are shared.  Returns 0, or -1 when a tile's staging wait expired.
int host_batch_run(int nruns, const int *nx, const int *ny, const double *dx, const double *dy, const double *eta,
                   const int *bc_x, const int *bc_y, double gamma, double cfl, double eps, int shape, int ctas,
                   double *states, int nsteps, double *dts)
{
    std::vector<Grid> grids(nruns);
    std::vector<std::vector<double>> A(nruns), B(nruns), row2(nruns);
    std::vector<Control> ctl(nruns);
    std::vector<BatchRun> runs(nruns);
    std::vector<CUtensorMap> maps((size_t)nruns * MAPS_PER_RUN);
    std::vector<TileRef> tiles[2];
    long long max_ghost = 0;
    size_t off = 0;
    for (int r = 0; r < nruns; ++r) {
        Grid &g = grids[r];
        g = Grid{};
        g.nx = nx[r];
        g.ny = ny[r];
        g.pitch = (g.ny + 31) / 32 * 32;
        g.plane = (long long)g.nx * g.pitch;
        g.dx = dx[r];
        g.dy = dy[r];
        g.gamma = gamma;
        g.cfl = cfl;
        g.eps = eps;
        g.eta = eta[r];
        g.bc_x = bc_x[r];
        g.bc_y = bc_y[r] < 0 ? bc_x[r] : bc_y[r];
        const size_t P = (size_t)g.plane;
        A[r].assign(P * NFIELD, 0.0);
        B[r].assign(P * NFIELD, 0.0);
        row2[r].assign((size_t)g.nx, 0.0);
        launch_aos_to_planes(g, states + off, A[r].data(), nullptr);
        if (g.bc_x == BC_SYMMETRIC) launch_snapshot_row2(g, A[r].data(), row2[r].data(), nullptr);
        launch_boundary(g, A[r].data(), row2[r].data(), nullptr, 0, nullptr);
        launch_rate(g, A[r].data(), &ctl[r], 0, 1, nullptr);
        off += (size_t)g.nx * g.ny * NFIELD;
        runs[r] = BatchRun{g, A[r].data(), B[r].data(), nullptr, row2[r].data(), &ctl[r]};
        const unsigned long long st0 = (unsigned long long)g.pitch * 8, st1 = (unsigned long long)P * 8;
        const unsigned uj = (unsigned)shape_uj(shape);
        for (int st = 1; st <= 2; ++st)
            maps[(size_t)r * MAPS_PER_RUN + st - 1] = host_map(st == 1 ? A[r].data() : B[r].data(), 3, g.ny, g.nx,
                                                               NFIELD, st0, st1, uj, (unsigned)stage_ui(st, shape), NFIELD);
        const long long ng = 6LL * g.ny + 6LL * (g.nx - 6);
        max_ghost = ng > max_ghost ? ng : max_ghost;
        for (int st = 1; st <= 2; ++st) {
            const int ti = stage_ti(st, shape), tj = shape_tj(shape);
            const int nti = (g.nx - 2 * HALO + ti - 1) / ti, ntj = (g.ny - 2 * HALO + tj - 1) / tj;
            for (int a = 0; a < nti; ++a)
                for (int c = 0; c < ntj; ++c) tiles[st - 1].push_back(TileRef{r, a, c, 0});
        }
    }
    int parity = 0;
    for (int n = 0; n < nsteps; ++n) {
        STAGE_VARIANT::launch_stage_batch(1, shape, runs.data(), maps.data(), tiles[0].data(), (int)tiles[0].size(), ctas,
                                  parity, nullptr);
        launch_boundary_batch(runs.data(), nruns, max_ghost, 0, 0, nullptr);
        STAGE_VARIANT::launch_stage_batch(2, shape, runs.data(), maps.data(), tiles[1].data(), (int)tiles[1].size(), ctas,
                                  parity, nullptr);
        launch_boundary_batch(runs.data(), nruns, max_ghost, 1, parity ^ 1, nullptr);
        for (int r = 0; r < nruns; ++r) {
            if (ctl[r].error) return -1;
            dts[(size_t)r * nsteps + n] = ctl[r].dt;
        }
        parity ^= 1;
    }
    off = 0;
    for (int r = 0; r < nruns; ++r) {
        launch_planes_to_aos(grids[r], A[r].data(), states + off, nullptr);
        off += (size_t)grids[r].nx * grids[r].ny * NFIELD;
    }
    return 0;
}

}  // extern "C"
