// contact.cu -- the step with the CT-Contact EMF (cfg.ct_scheme =
// RMHD2D_CT_CONTACT), compiled with -fmad=false: FP64 in the reference's
// evaluation order, bit-identical to the oracle's orc_step_contact.
//
// The step follows the multi-GPU library's ordering
// (ResistiveMHD_multiGPU_cuda/ResistiveMHD2D_GPU/resistiveMHD2D.cu:147-221)
// with its corner EMF (ct.cu:26-257), on this library's fluxes, update ranges
// and dt:
//   begin        dt (CFL or the fixed dt), the control block's step fields
//   flux         F, G of the cell-centred U^n (HLLD, MUSCL, resistive hook)
//   ref (old)    per-cell reference EMF u bY - v bX - eta jZ of U^n with the
//                face B that shift + back-to-face leave (smoothed)
//   update 1     U* = U^n - dt div(F, G) for all 8 fields (smoothed face B)
//   boundary     U*
//   flux         F, G of the cell-centred U*
//   update 2     C = (U^n + U* - dt div(F, G)) / 2 (both with smoothed face B)
//   boundary     C
//   ref (now)    per-cell reference EMF of C
//   corners      Ez of every corner, the mean of the two stages' contact EMFs
//   CT           A = C with face B = U^n's faces - dt curl(Ez)
//   boundary     A, then the CFL rate and NaN test of every cell
// Flux entries whose stencil leaves the grid, and the EMF inputs outside
// 0 < i < nx-1, 0 < j < ny-1, are NaN, as the oracle leaves them: they reach
// only ghost cells, which the boundary passes overwrite.
#include <cuda_runtime.h>

#include "adjoint_core.cuh"
#include "aux_kernels.h"
#include "contact.h"
#include "physics.cuh"
#include "rmhd2d_internal.h"

namespace rmhd2d {

namespace {

__device__ __forceinline__ long long at(const Grid &g, int i, int j) { return (long long)i * g.pitch + j; }

__device__ __forceinline__ double qnan() { return bits_to_double(0x7FF8000000000000ull); }

// shiftUToCenterForCT (resistiveMHD_2D.cu:313-368)
__device__ __forceinline__ double bx_c(const Grid &g, const double *U, int i, int j)
{
    const double *b = U + BXF * g.plane;
    return i >= 1 ? 0.5 * (b[at(g, i, j)] + b[at(g, i - 1, j)]) : b[at(g, i, j)];
}
__device__ __forceinline__ double by_c(const Grid &g, const double *U, int i, int j)
{
    const double *b = U + BYF * g.plane;
    return j >= 1 ? 0.5 * (b[at(g, i, j)] + b[at(g, i, j - 1)]) : b[at(g, i, j)];
}
// then backUToCenterHalfForCT (resistiveMHD_2D.cu:371-426): the face value
// the two leave in U
__device__ __forceinline__ double bx_s(const Grid &g, const double *U, int i, int j)
{
    return i < g.nx - 1 ? 0.5 * (bx_c(g, U, i, j) + bx_c(g, U, i + 1, j)) : bx_c(g, U, i, j);
}
__device__ __forceinline__ double by_s(const Grid &g, const double *U, int i, int j)
{
    return j < g.ny - 1 ? 0.5 * (by_c(g, U, i, j) + by_c(g, U, i, j + 1)) : by_c(g, U, i, j);
}

// A cell of the cell-centred state in sweep order (hlld.cu:134-160 shuffles
// the y sweep's cell to rho, rhoV, rhoW, rhoU, bY, bZ, bX, e).
template <int DIR>
__device__ __forceinline__ void sweep_cell(const Grid &g, const double *U, int i, int j, double *c)
{
    const long long k = at(g, i, j), P = g.plane;
    if (DIR == 0) {
        c[0] = U[RHO * P + k]; c[1] = U[MX * P + k]; c[2] = U[MY * P + k]; c[3] = U[MZ * P + k];
        c[4] = bx_c(g, U, i, j); c[5] = by_c(g, U, i, j); c[6] = U[BZF * P + k]; c[7] = U[EN * P + k];
    } else {
        c[0] = U[RHO * P + k]; c[1] = U[MY * P + k]; c[2] = U[MZ * P + k]; c[3] = U[MX * P + k];
        c[4] = by_c(g, U, i, j); c[5] = U[BZF * P + k]; c[6] = bx_c(g, U, i, j); c[7] = U[EN * P + k];
    }
}

// F and G of every interface: HLLD::calculateFluxF / G (hlld.cu:110-233)
// of the cell-centred state plus the resistive hook
// (main_plasmoid.cu:175-290).  The x sweep is defined for 1 <= i <= nx-4,
// the y sweep for 1 <= j <= ny-3 (the ranges the reference's buffers hold
// current values in), NaN elsewhere.  One CTA stages the primitives of
// (CT_TI + 3) x (CT_TJ + 3) cells in shared memory once -- the x and y
// sweeps' pressures sum their squares in different orders, so both are
// kept -- then the hook's eta*J of the (CT_TI + 1) x (CT_TJ + 1) cells its
// interfaces read, once per cell, and forms the x and y interfaces (i, j)
// of its CT_TI x CT_TJ cells from there, in the reference's order of
// operations.  Divisions go through shared correctly rounded reciprocals
// (MdDiv, with IEEE division where its guard fails), which give the
// reference's quotients bit for bit.
constexpr int CT_TI = 16, CT_TJ = 32, CT_THREADS = 256;
constexpr int CT_SI = CT_TI + 3, CT_SJ = CT_TJ + 3, CT_SC = CT_SI * CT_SJ;
constexpr int CT_JI = CT_TI + 1, CT_JJ = CT_TJ + 1, CT_JC = CT_JI * CT_JJ;
enum { S_RHO = 0, S_U, S_V, S_W, S_BXC, S_BYC, S_BZ, S_PX, S_PY, S_NF };
enum { J_X = 0, J_Y, J_Z, J_NF };   // eta*Jx, eta*Jy, eta*Jz
constexpr size_t CT_SMEM = (size_t)(S_NF * CT_SC + J_NF * CT_JC) * sizeof(double);

__global__ void __launch_bounds__(CT_THREADS, 2) contact_flux_tiled_kernel(Grid g, const double *U, const double *eta,
                                                                         double *F, double *G)
{
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    double (*S)[CT_SC] = reinterpret_cast<double (*)[CT_SC]>(smem_raw);
    double (*J)[CT_JC] = reinterpret_cast<double (*)[CT_JC]>(smem_raw + S_NF * CT_SC * sizeof(double));
    const int i0 = blockIdx.y * CT_TI, j0 = blockIdx.x * CT_TJ;
    const long long P = g.plane;
    const double gm1 = g.gamma - 1.0;
    // staged cell (si, sj) is cell (i0 - 1 + si, j0 - 1 + sj)
    for (int c = threadIdx.x; c < CT_SC; c += CT_THREADS) {
        const int si = c / CT_SJ, sj = c - si * CT_SJ;
        const int i = i0 - 1 + si, j = j0 - 1 + sj;
        if (i < 0 || j < 0 || i >= g.nx || j >= g.ny) continue;   // read by no defined interface
        const long long k = at(g, i, j);
        const double rho = U[RHO * P + k], mx = U[MX * P + k], my = U[MY * P + k], mz = U[MZ * P + k];
        // calculate_half_Q.cu:4-38 in both sweeps' orders
        MdDiv md;
        const double yr = md.recip(rho);
        double u = md.div(mx, rho, yr), v = md.div(my, rho, yr), w = md.div(mz, rho, yr);
        if (!md.ok) {
            u = mx / rho;
            v = my / rho;
            w = mz / rho;
        }
        const double bxc = bx_c(g, U, i, j), byc = by_c(g, U, i, j), bz = U[BZF * P + k], e = U[EN * P + k];
        S[S_RHO][c] = rho;
        S[S_U][c] = u;
        S[S_V][c] = v;
        S[S_W][c] = w;
        S[S_BXC][c] = bxc;
        S[S_BYC][c] = byc;
        S[S_BZ][c] = bz;
        S[S_PX][c] = gm1 * ((e - 0.5 * (rho * (u * u + v * v + w * w))) - 0.5 * (bxc * bxc + byc * byc + bz * bz));
        S[S_PY][c] = gm1 * ((e - 0.5 * (rho * (v * v + w * w + u * u))) - 0.5 * (byc * byc + bz * bz + bxc * bxc));
    }
    __syncthreads();

    auto at_s = [](int si, int sj) { return si * CT_SJ + sj; };
    auto bz = [&](int a, int b) { return S[S_BZ][at_s(a, b)]; };
    auto byc = [&](int a, int b) { return S[S_BYC][at_s(a, b)]; };
    auto bxc = [&](int a, int b) { return S[S_BXC][at_s(a, b)]; };
    const double two_dx = 2.0 * g.dx, two_dy = 2.0 * g.dy;
    MdDiv cd;
    const double y2dx = cd.recip(two_dx), y2dy = cd.recip(two_dy);
    // eta*J of cell (i0 + ci, j0 + cj), staged at (ci + 1, cj + 1), where
    // all its neighbours exist (the hook reads it only there)
    for (int c = threadIdx.x; c < CT_JC; c += CT_THREADS) {
        const int ci = c / CT_JJ, cj = c - ci * CT_JJ;
        const int i = i0 + ci, j = j0 + cj;
        if (i < 1 || j < 1 || i > g.nx - 2 || j > g.ny - 2) continue;
        const int si = ci + 1, sj = cj + 1;
        const double nX = bz(si, sj + 1) - bz(si, sj - 1);
        const double nY = -(bz(si + 1, sj) - bz(si - 1, sj));
        const double nZx = byc(si + 1, sj) - byc(si - 1, sj), nZy = bxc(si, sj + 1) - bxc(si, sj - 1);
        MdDiv md;
        md.ok = cd.ok;
        double jX = md.div(nX, two_dy, y2dy), jY = md.div(nY, two_dx, y2dx);
        double jZ = md.div(nZx, two_dx, y2dx) - md.div(nZy, two_dy, y2dy);
        if (!md.ok) {
            jX = nX / two_dy;
            jY = nY / two_dx;
            jZ = nZx / two_dx - nZy / two_dy;
        }
        const double e = eta ? eta[at(g, i, j)] : g.eta;
        J[J_X][c] = e * jX;
        J[J_Y][c] = e * jY;
        J[J_Z][c] = e * jZ;
    }
    __syncthreads();

    for (int t = threadIdx.x; t < 2 * CT_TI * CT_TJ; t += CT_THREADS) {
        const int dir = t >= CT_TI * CT_TJ;
        const int r = t - dir * CT_TI * CT_TJ;
        const int li = r / CT_TJ, lj = r - li * CT_TJ;
        const int i = i0 + li, j = j0 + lj;
        if (i >= g.nx || j >= g.ny) continue;
        const int si = li + 1, sj = lj + 1;
        double out[8];
        const bool ok = dir == 0 ? (i >= 1 && i <= g.nx - 4) : (j >= 1 && j <= g.ny - 3);
        if (!ok) {
#pragma unroll
            for (int c = 0; c < 8; ++c) out[c] = qnan();
        } else {
            // sweep-order primitives of the four cells along the sweep
            double q[4][8];
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                const int c = dir == 0 ? at_s(si - 1 + m, sj) : at_s(si, sj - 1 + m);
                if (dir == 0) {
                    q[m][0] = S[S_RHO][c]; q[m][1] = S[S_U][c]; q[m][2] = S[S_V][c]; q[m][3] = S[S_W][c];
                    q[m][5] = S[S_BYC][c]; q[m][6] = S[S_BZ][c]; q[m][7] = S[S_PX][c];
                } else {
                    q[m][0] = S[S_RHO][c]; q[m][1] = S[S_V][c]; q[m][2] = S[S_W][c]; q[m][3] = S[S_U][c];
                    q[m][5] = S[S_BZ][c]; q[m][6] = S[S_BXC][c]; q[m][7] = S[S_PY][c];
                }
                q[m][4] = 0.0;
            }
            // basic_param's interface-normal B of the left cell and its neighbour
            {
                const int nb = dir == 0 ? S_BXC : S_BYC;
                const int c1 = at_s(si, sj), c2 = dir == 0 ? at_s(si + 1, sj) : at_s(si, sj + 1);
                q[1][4] = XMUL(0.5, XADD(S[nb][c1], S[nb][c2]));
            }
            double L[8], R[8], f[8];
            adj::muscl_states(q[0], q[1], q[2], q[3], g.eps, L, R);
            const Prim PL{L[0], L[1], L[2], L[3], L[4], L[5], L[6], L[7]};
            const Prim PR{R[0], R[1], R[2], R[3], R[4], R[5], R[6], R[7]};
            hlld_flux<true>(PL, PR, g.gamma, g.eps, f);
            if (dir == 0) {
#pragma unroll
                for (int c = 0; c < 8; ++c) out[c] = f[c];
            } else {
                out[0] = f[0]; out[1] = f[3]; out[2] = f[1]; out[3] = f[2];
                out[4] = f[6]; out[5] = f[4]; out[6] = f[5]; out[7] = f[7];
            }
            // the resistive hook (the reference's 0 < i < nx-2, 0 < j < ny-2)
            if (i >= 1 && i <= g.nx - 3 && j >= 1 && j <= g.ny - 3) {
                const int c0 = li * CT_JJ + lj;                         // eta*J of cell (i, j)
                if (dir == 0) {
                    const int c1 = c0 + CT_JJ;                          // (i + 1, j)
                    const double etaJY = J[J_Y][c0], etaJZ = J[J_Z][c0];
                    const double etaJYBZ = etaJY * bz(si, sj), etaJZBY = etaJZ * byc(si, sj);
                    const double etaJYPlus1 = J[J_Y][c1], etaJZPlus1 = J[J_Z][c1];
                    const double etaJYBZPlus1 = etaJYPlus1 * bz(si + 1, sj), etaJZBYPlus1 = etaJZPlus1 * byc(si + 1, sj);
                    out[5] -= 0.5 * (etaJZ + etaJZPlus1);
                    out[6] += 0.5 * (etaJY + etaJYPlus1);
                    out[7] += 0.5 * (etaJYBZ + etaJYBZPlus1) - 0.5 * (etaJZBY + etaJZBYPlus1);
                } else {
                    const int c1 = c0 + 1;                              // (i, j + 1)
                    const double etaJX = J[J_X][c0], etaJZ = J[J_Z][c0];
                    const double etaJXBZ = etaJX * bz(si, sj), etaJZBX = etaJZ * bxc(si, sj);
                    const double etaJXPlus1 = J[J_X][c1], etaJZPlus1 = J[J_Z][c1];
                    const double etaJXBZPlus1 = etaJXPlus1 * bz(si, sj + 1), etaJZBXPlus1 = etaJZPlus1 * bxc(si, sj + 1);
                    out[4] += 0.5 * (etaJZ + etaJZPlus1);
                    out[6] -= 0.5 * (etaJX + etaJXPlus1);
                    out[7] += 0.5 * (etaJZBX + etaJZBXPlus1) - 0.5 * (etaJXBZ + etaJXBZPlus1);
                }
            }
        }
        double *o = (dir == 0 ? F : G) + at(g, i, j);
#pragma unroll
        for (int c = 0; c < 8; ++c) o[c * P] = out[c];
    }
}

__global__ void contact_begin_kernel(Grid g, Control *ctl, int parity)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double dt = ctl->use_fixed_dt
                          ? ctl->dt_fixed
                          : step_dt(ctl->amax[parity], ctl->first_nan[parity], g.dx, g.dy, g.eps, g.eta, g.cfl);
    ctl->dt = dt;
    ctl->total_time = ctl->total_time + dt;
    ctl->amax[parity ^ 1] = 0ull;
    ctl->first_nan[parity ^ 1] = 0;
    ctl->crashed = 0;
}

// ct.cu:45-61: reference EMF u bY - v bX - eta jZ of cell (i, j) for
// 0 < i < nx-1, 0 < j < ny-1, from U's face B, smoothed (stage 1) or as
// stored (stage 2).
template <bool SMOOTHED>
__global__ void contact_ref_kernel(Grid g, const double *U, const double *eta, double *ref)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)g.nx * g.ny) return;
    const int i = (int)(t / g.ny), j = (int)(t - (long long)i * g.ny);
    const long long k = at(g, i, j), P = g.plane;
    if (!(i > 0 && i < g.nx - 1 && j > 0 && j < g.ny - 1)) {
        ref[k] = qnan();
        return;
    }
    auto BX = [&](int ii, int jj) { return SMOOTHED ? bx_s(g, U, ii, jj) : U[BXF * P + at(g, ii, jj)]; };
    auto BY = [&](int ii, int jj) { return SMOOTHED ? by_s(g, U, ii, jj) : U[BYF * P + at(g, ii, jj)]; };
    const double dx = g.dx, dy = g.dy;
    const double rho = U[RHO * P + k], mx = U[MX * P + k], my = U[MY * P + k];
    const double bX = 0.5 * (BX(i, j) + BX(i - 1, j));
    const double bY = 0.5 * (BY(i, j) + BY(i, j - 1));
    // the differences of the current's eight terms, in the reference's order
    const double nb[8] = {BY(i + 1, j) - BY(i, j),         BX(i, j + 1) - BX(i, j),
                          BY(i + 1, j - 1) - BY(i, j - 1), BX(i, j) - BX(i, j - 1),
                          BY(i, j - 1) - BY(i - 1, j - 1), BX(i - 1, j) - BX(i - 1, j - 1),
                          BY(i, j) - BY(i - 1, j),         BX(i - 1, j + 1) - BX(i - 1, j)};
    const double e = eta ? eta[k] : g.eta;
    // divisions through shared correctly rounded reciprocals (MdDiv), or
    // IEEE division where its guard fails: the same quotients
    auto ref_of = [&](auto &dv) {
        const double yr = dv.recip(rho), ydx = dv.recip(dx), ydy = dv.recip(dy);
        const double u = dv.div(mx, rho, yr), v = dv.div(my, rho, yr);
        const double jZ = 0.25 * (dv.div(nb[0], dx, ydx) - dv.div(nb[1], dy, ydy)
                                + dv.div(nb[2], dx, ydx) - dv.div(nb[3], dy, ydy)
                                + dv.div(nb[4], dx, ydx) - dv.div(nb[5], dy, ydy)
                                + dv.div(nb[6], dx, ydx) - dv.div(nb[7], dy, ydy));
        return u * bY - v * bX - e * jZ;
    };
    MdDiv md;
    double r = ref_of(md);
    if (!md.ok) {
        IeeeDiv id;
        r = ref_of(id);
    }
    ref[k] = r;
}

// The stage updates (resistiveMHD_2D.cu:53-130 functors, over k >= ny), all
// 8 fields, face B as shift + back-to-face leave it.
template <int STAGE>
__global__ void contact_update_kernel(Grid g, const double *Un, const double *Ub, const double *F, const double *G,
                                      const Control *ctl, double *dst)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)g.nx * g.ny) return;
    const int i = (int)(t / g.ny), j = (int)(t - (long long)i * g.ny);
    const long long k = at(g, i, j), P = g.plane;
    if (i == 0) {
        // outside the update range: stage 1 keeps U^n (copied before the
        // smoothing); stage 2 keeps U^n as the smoothing left it
#pragma unroll
        for (int c = 0; c < NFIELD; ++c) {
            double v = Un[c * P + k];
            if (STAGE == 2 && c == BXF) v = bx_s(g, Un, i, j);
            if (STAGE == 2 && c == BYF) v = by_s(g, Un, i, j);
            dst[c * P + k] = v;
        }
        return;
    }
    const double dt = ctl->dt;
    const double rdx = dt / g.dx, rdy = dt / g.dy;
    const long long km = at(g, i - 1, j);
#pragma unroll
    for (int c = 0; c < NFIELD; ++c) {
        // the flat k - 1 neighbour of j = 0 is the previous column's last
        // cell, whose G entry is NaN
        const double gm = j >= 1 ? G[c * P + k - 1] : qnan();
        const double div = rdx * (F[c * P + k] - F[c * P + km]);
        const double dvg = rdy * (G[c * P + k] - gm);
        double u = Un[c * P + k];
        if (c == BXF) u = bx_s(g, Un, i, j);
        if (c == BYF) u = by_s(g, Un, i, j);
        if (STAGE == 1) {
            dst[c * P + k] = u - div - dvg;
        } else {
            double ub = Ub[c * P + k];
            if (c == BXF) ub = bx_s(g, Ub, i, j);
            if (c == BYF) ub = by_s(g, Ub, i, j);
            dst[c * P + k] = 0.5 * (u + ub - div - dvg);
        }
    }
}

__device__ __forceinline__ int isgn(double x) { return (x > 0.0) - (x < 0.0); }

// One stage's inputs of the contact EMF (ct.cu:26-65), NaN outside
// 0 < i < nx-1, 0 < j < ny-1.
struct StageEmf {
    const double *F, *G, *ref;
    __device__ __forceinline__ bool in(const Grid &g, int i, int j) const
    {
        return i > 0 && i < g.nx - 1 && j > 0 && j < g.ny - 1;
    }
    __device__ __forceinline__ double NF5(const Grid &g, int i, int j) const
    {
        return in(g, i, j) ? F[BYF * g.plane + at(g, i, j)] : qnan();
    }
    __device__ __forceinline__ double NG4(const Grid &g, int i, int j) const
    {
        return in(g, i, j) ? G[BXF * g.plane + at(g, i, j)] : qnan();
    }
    __device__ __forceinline__ double NF0(const Grid &g, int i, int j) const
    {
        return in(g, i, j) ? F[RHO * g.plane + at(g, i, j)] : qnan();
    }
    __device__ __forceinline__ double NG0(const Grid &g, int i, int j) const
    {
        return in(g, i, j) ? G[RHO * g.plane + at(g, i, j)] : qnan();
    }
    __device__ __forceinline__ double CF5(const Grid &g, int i, int j) const
    {
        return in(g, i, j) ? ref[at(g, i, j)] : qnan();
    }
    __device__ __forceinline__ double CG4(const Grid &g, int i, int j) const
    {
        return in(g, i, j) ? -(ref[at(g, i, j)]) : qnan();
    }
};

// ct.cu:147-169: the corner (i+1/2, j+1/2) EMF of one stage.
__device__ double contact_corner(const Grid &g, const StageEmf &s, int i, int j)
{
    const double avg = 0.25 * (-s.NF5(g, i, j) - s.NF5(g, i, j + 1) + s.NG4(g, i, j) + s.NG4(g, i + 1, j));
    const int sF0 = isgn(s.NF0(g, i, j)), sF0n = isgn(s.NF0(g, i, j + 1));
    const int sG0 = isgn(s.NG0(g, i, j)), sG0e = isgn(s.NG0(g, i + 1, j));
    const double eS = (1.0 + sF0) * (s.NG4(g, i, j) - s.CG4(g, i, j))
                    + (1.0 - sF0) * (s.NG4(g, i + 1, j) - s.CG4(g, i + 1, j));
    const double eN = (1.0 + sF0n) * (s.CG4(g, i, j + 1) - s.NG4(g, i, j))
                    + (1.0 - sF0n) * (s.CG4(g, i + 1, j + 1) - s.NG4(g, i + 1, j));
    const double eW = -(1.0 + sG0) * (s.NF5(g, i, j) - s.CF5(g, i, j))
                    - (1.0 - sG0) * (s.NF5(g, i, j + 1) - s.CF5(g, i, j + 1));
    const double eE = -(1.0 + sG0e) * (s.CF5(g, i + 1, j) - s.NF5(g, i, j))
                    - (1.0 - sG0e) * (s.CF5(g, i + 1, j + 1) - s.NF5(g, i, j + 1));
    return avg + 0.125 * (eS - eN + eW - eE);
}

// ct.cu:195: the mean of the two stages' EMFs, defined for i < nx-1,
// j < ny-1.
__device__ __forceinline__ double corner_ez(const Grid &g, const StageEmf &o, const StageEmf &n, int i, int j)
{
    if (i < 0 || j < 0 || i >= g.nx - 1 || j >= g.ny - 1) return qnan();
    return 0.5 * (contact_corner(g, o, i, j) + contact_corner(g, n, i, j));
}

// Every corner EMF once (corner_ez), NaN where it is undefined.
__global__ void contact_corner_kernel(Grid g, StageEmf o, StageEmf n, double *E)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)g.nx * g.ny) return;
    const int i = (int)(t / g.ny), j = (int)(t - (long long)i * g.ny);
    E[at(g, i, j)] = corner_ez(g, o, n, i, j);
}

// ct.cu:200-218 CT_kernel on the step input's faces (A), the rest of the
// state from the stage-2 result C; E holds the corner EMFs.
__global__ void contact_ct_kernel(Grid g, const double *E, const double *C, const Control *ctl, double *A)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)g.nx * g.ny) return;
    const int i = (int)(t / g.ny), j = (int)(t - (long long)i * g.ny);
    const long long k = at(g, i, j), P = g.plane;
#pragma unroll
    for (int c = 0; c < NFIELD; ++c)
        if (c != BXF && c != BYF) A[c * P + k] = C[c * P + k];
    if (i > 0 && j > 0) {
        const double dt = ctl->dt;
        const double ez = E[k];
        A[BXF * P + k] = A[BXF * P + k] - dt / g.dy * (ez - E[at(g, i, j - 1)]);
        A[BYF * P + k] = A[BYF * P + k] + dt / g.dx * (ez - E[at(g, i - 1, j)]);
    } else {
        A[BXF * P + k] = C[BXF * P + k];
        A[BYF * P + k] = C[BYF * P + k];
    }
}

int blocks_for(long long n, int threads) { return (int)((n + threads - 1) / threads); }

}  // namespace

void enqueue_contact_step(const ContactStep &c, cudaStream_t st)
{
    const Grid &g = c.g;
    const long long n = (long long)g.nx * g.ny;
    const int b256 = blocks_for(n, 256);
    const dim3 flux_grid((g.ny + CT_TJ - 1) / CT_TJ, (g.nx + CT_TI - 1) / CT_TI);
    auto boundary = [&](double *state) {
        if (g.bc_x == BC_SYMMETRIC) launch_snapshot_row2(g, state, c.row2, st);
        launch_boundary(g, state, c.row2, nullptr, 0, st);
    };
    cudaFuncSetAttribute(contact_flux_tiled_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CT_SMEM);
    contact_begin_kernel<<<1, 32, 0, st>>>(g, c.ctl, c.parity);
    // stage 1
    contact_flux_tiled_kernel<<<flux_grid, CT_THREADS, CT_SMEM, st>>>(g, c.A, c.eta, c.F1, c.G1);
    contact_ref_kernel<true><<<b256, 256, 0, st>>>(g, c.A, c.eta, c.R1);
    contact_update_kernel<1><<<b256, 256, 0, st>>>(g, c.A, nullptr, c.F1, c.G1, c.ctl, c.B);
    boundary(c.B);
    // stage 2
    contact_flux_tiled_kernel<<<flux_grid, CT_THREADS, CT_SMEM, st>>>(g, c.B, c.eta, c.F2, c.G2);
    contact_update_kernel<2><<<b256, 256, 0, st>>>(g, c.A, c.B, c.F2, c.G2, c.ctl, c.C);
    boundary(c.C);
    contact_ref_kernel<false><<<b256, 256, 0, st>>>(g, c.C, c.eta, c.R2);
    // CT with the two stages' mean contact EMF, then the boundary and the
    // next step's CFL rate and crash flag
    contact_corner_kernel<<<b256, 256, 0, st>>>(g, StageEmf{c.F1, c.G1, c.R1}, StageEmf{c.F2, c.G2, c.R2}, c.E);
    contact_ct_kernel<<<b256, 256, 0, st>>>(g, c.E, c.C, c.ctl, c.A);
    boundary(c.A);
    launch_rate(g, c.A, c.ctl, c.parity ^ 1, 1, st);
}

}  // namespace rmhd2d
