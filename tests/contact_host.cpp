// contact_host.cpp -- TEST INFRASTRUCTURE.  The CT-Contact step of the C ABI
// (enqueue_contact_step, resistivemhd_gpu_b200/csrc/contact.cu) run on the
// CPU over its kernels' own source, compiled for the host through
// cuda_host_shim.h.  The three launchers contact.cu takes from
// aux_kernels.cu are supplied here: the ghost fill is the oracle's
// (orc_boundary, which the CUDA fill matches bit for bit on the GPU), and the
// CFL reduction evaluates the library's per-cell rate (physics.cuh:
// cfl_rate, rate_bits) as rate_kernel does, cell by cell.  The set-up
// mirrors rmhd2d_create + rmhd2d_set_state(apply_boundary = 1), and each step
// rmhd2d_step_rk2 with ct_scheme = RMHD2D_CT_CONTACT.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "aux_kernels.h"
#include "contact.h"
#include "physics.cuh"
#include "rmhd2d_internal.h"
#include "rmhd2d_oracle.h"

namespace rmhd2d {

namespace {

orc_params g_params;

void to_aos(const Grid &g, const double *planes, double *aos)
{
    for (int f = 0; f < NFIELD; ++f)
        for (int i = 0; i < g.nx; ++i)
            for (int j = 0; j < g.ny; ++j)
                aos[((long long)j + (long long)i * g.ny) * NFIELD + f] = planes[f * g.plane + (long long)i * g.pitch + j];
}

void to_planes(const Grid &g, const double *aos, double *planes)
{
    for (int f = 0; f < NFIELD; ++f)
        for (int i = 0; i < g.nx; ++i)
            for (int j = 0; j < g.ny; ++j)
                planes[f * g.plane + (long long)i * g.pitch + j] = aos[((long long)j + (long long)i * g.ny) * NFIELD + f];
}

}  // namespace

void launch_snapshot_row2(const Grid &g, const double *s, double *row2, cudaStream_t)
{
    for (int i = 0; i < g.nx; ++i) row2[i] = s[BYF * g.plane + (long long)i * g.pitch + 2];
}

// The contact step applies the boundary after a fresh row2 snapshot and with
// no control block: the plain ghost fill of the configured walls.
void launch_boundary(const Grid &g, double *s, const double *, Control *ctl, int, cudaStream_t)
{
    if (ctl) {
        std::fprintf(stderr, "contact_host: launch_boundary with a control block is not modelled\n");
        std::abort();
    }
    std::vector<double> aos((size_t)g.nx * g.ny * NFIELD);
    to_aos(g, s, aos.data());
    orc_boundary(&g_params, aos.data());
    to_planes(g, aos.data(), s);
}

void launch_rate(const Grid &g, const double *s, Control *ctl, int slot, int set_crash, cudaStream_t)
{
    const long long n = (long long)g.nx * g.ny, P = g.plane;
    unsigned long long bits = 0ull;
    int nan_e = 0;
    for (long long t = 0; t < n; ++t) {
        const int i = (int)(t / g.ny), j = (int)(t - (long long)i * g.ny);
        const long long k = (long long)i * g.pitch + j;
        const double e = s[EN * P + k];
        const double r = cfl_rate(s[RHO * P + k], s[MX * P + k], s[MY * P + k], s[MZ * P + k], s[BXF * P + k],
                                  s[BYF * P + k], s[BZF * P + k], e, g.gamma, g.dx, g.dy);
        const unsigned long long b = rate_bits(r);
        bits = b > bits ? b : bits;
        if (t == 0 && r != r) ctl->first_nan[slot] = 1;
        nan_e |= (e != e);
    }
    if (bits > ctl->amax[slot]) ctl->amax[slot] = bits;
    if (set_crash && nan_e) ctl->crashed = 1;
}

}  // namespace rmhd2d

using namespace rmhd2d;

extern "C" {

// nsteps CT-Contact steps from the reference-layout state (updated in place;
// the boundary is applied first, as set_state does), each step's dt in dts.
// Returns 0, or 1 + the step whose output raised the crash flag.
int host_contact_run(int nx, int ny, double dx, double dy, double gamma, double cfl, double eps, double eta, int bc_x,
                     int bc_y, const double *eta_table, double *state, int nsteps, double *dts)
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
    g_params = orc_params{};
    g_params.nx = nx;
    g_params.ny = ny;
    g_params.dx = dx;
    g_params.dy = dy;
    g_params.gamma = gamma;
    g_params.cfl = cfl;
    g_params.eps = eps;
    g_params.eta = eta;
    g_params.eta_table = eta_table;
    g_params.bc = bc_x;
    g_params.bc_y = g.bc_y;
    g_params.ct_contact = 1;

    const size_t P = (size_t)g.plane, sd = P * NFIELD;
    std::vector<double> A(sd, 0.0), B(sd, 0.0), C(sd, 0.0), F1(sd, 0.0), G1(sd, 0.0), F2(sd, 0.0), G2(sd, 0.0),
        R1(P, 0.0), R2(P, 0.0), E(P, 0.0), row2((size_t)nx, 0.0), eta_plane;
    if (eta_table) {
        eta_plane.assign(P, 0.0);
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) eta_plane[(size_t)i * g.pitch + j] = eta_table[(size_t)j + (size_t)i * ny];
    }
    Control ctl{};
    to_planes(g, state, A.data());
    if (g.bc_x == BC_SYMMETRIC) launch_snapshot_row2(g, A.data(), row2.data(), nullptr);
    launch_boundary(g, A.data(), row2.data(), nullptr, 0, nullptr);
    int parity = 0;
    launch_rate(g, A.data(), &ctl, parity, 1, nullptr);
    int rc = 0;
    for (int n = 0; n < nsteps; ++n) {
        ContactStep c{};
        c.g = g;
        c.A = A.data();
        c.B = B.data();
        c.C = C.data();
        c.F1 = F1.data();
        c.G1 = G1.data();
        c.F2 = F2.data();
        c.G2 = G2.data();
        c.R1 = R1.data();
        c.R2 = R2.data();
        c.E = E.data();
        c.eta = eta_table ? eta_plane.data() : nullptr;
        c.row2 = row2.data();
        c.ctl = &ctl;
        c.parity = parity;
        enqueue_contact_step(c, nullptr);
        dts[n] = ctl.dt;
        parity ^= 1;
        if (ctl.crashed) {
            rc = 1 + n;
            break;
        }
    }
    to_aos(g, A.data(), state);
    return rc;
}

}  // extern "C"
