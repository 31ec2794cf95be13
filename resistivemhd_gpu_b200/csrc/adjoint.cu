// adjoint.cu -- discrete adjoint of the RK2 step (dt of each step held
// fixed): the reverse of one stage as three kernels, and the transpose of
// the periodic boundary.
//
// Forward stage (resistiveMHD_2D.cu:133-195), W the stage input:
//   Wc  = W with cell-centred bX, bY            (shiftUToCenterForCT)
//   F,G = HLLD(MUSCL(prim(Wc))) + eta*J terms   (flux_solver.cu, hlld.cu,
//                                                main_plasmoid.cu:175-290)
//   Ez  = (G4 + G4[i+1] - F5 - F5[j+1]) / 4     (stage 1 only, ct.cu:22-41)
//   hydro out = s_in*U0 + s*(W - dt div(F,G))   (s = 1 stage 1, 1/2 stage 2)
//   bX, bY out = CT of the step input's faces with the stage-1 Ez
// Reverse, given Ub = adjoint of the stage output after the boundary
// transpose (so every ghost entry is 0):
//   adj_iface_kernel  per interface: F-bar, G-bar from Ub (and the corner
//                     EMF adjoint in stage 1), the recomputed interface
//                     states and the HLLD reverse -> adjoints of the left
//                     and right states + the minmod branches; per cell the
//                     eta*J reverse -> J-bar, direct B adjoints, eta-bar
//   adj_gather_kernel per cell: MUSCL and primitive-recovery transposes over
//                     the four interfaces of each sweep that read the cell
//                     -> adjoint of Wc (hydro part written out, centred B
//                     parked for the next kernel)
//   adj_center_kernel per cell: transpose of the face->centre averaging and
//                     of the CT copy of the step input's faces
#include <cuda_runtime.h>

#include "adjoint.h"
#include "adjoint_core.cuh"
#include "rmhd2d_internal.h"

namespace rmhd2d {

namespace {

using adj::recon_comp;

constexpr int IF_PLANES = 16;   // per sweep: 7 left adjoints, b_n adjoint, 7 right adjoints, minmod branches
constexpr int ADJ_THREADS = 128;

__device__ __forceinline__ long long at(const Grid &g, int i, int j) { return (long long)i * g.pitch + j; }

__device__ __forceinline__ bool hydro_field(int f) { return f != BXF && f != BYF; }

// Cell-centred B of W (resistiveMHD_2D.cu:313-368): the first row / column
// keeps its face value.
__device__ __forceinline__ double bx_c(const Grid &g, const double *W, int i, int j)
{
    const double *bX = W + BXF * g.plane;
    return i >= 1 ? 0.5 * (bX[at(g, i, j)] + bX[at(g, i - 1, j)]) : bX[at(g, i, j)];
}
__device__ __forceinline__ double by_c(const Grid &g, const double *W, int i, int j)
{
    const double *bY = W + BYF * g.plane;
    return j >= 1 ? 0.5 * (bY[at(g, i, j)] + bY[at(g, i, j - 1)]) : bY[at(g, i, j)];
}

// A centred cell in sweep order: x (rho, mx, my, mz, bXc, bYc, bZ, e),
// y (rho, my, mz, mx, bYc, bZ, bXc, e) as shuffleForTmpUForFluxG_kernel
// (hlld.cu:134-160) arranges it.
template <int DIR>
__device__ __forceinline__ void sweep_cell(const Grid &g, const double *W, int i, int j, double *c)
{
    const long long k = at(g, i, j), P = g.plane;
    if (DIR == 0) {
        c[0] = W[RHO * P + k]; c[1] = W[MX * P + k]; c[2] = W[MY * P + k]; c[3] = W[MZ * P + k];
        c[4] = bx_c(g, W, i, j); c[5] = by_c(g, W, i, j); c[6] = W[BZF * P + k]; c[7] = W[EN * P + k];
    } else {
        c[0] = W[RHO * P + k]; c[1] = W[MY * P + k]; c[2] = W[MZ * P + k]; c[3] = W[MX * P + k];
        c[4] = by_c(g, W, i, j); c[5] = W[BZF * P + k]; c[6] = bx_c(g, W, i, j); c[7] = W[EN * P + k];
    }
}

// Sweep-order slot s of DIR -> natural field.
template <int DIR> __device__ __forceinline__ int sweep_field(int s)
{
    if (DIR == 0) return s;
    constexpr int map[8] = {RHO, MY, MZ, MX, BYF, BZF, BXF, EN};
    return map[s];
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
// natural field order; i + 1 <= nx - 1.
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
__device__ __forceinline__ bool x_iface_live(const Grid &g, int i, int j)
{
    return i >= 2 && i <= g.nx - 4 && j >= 2 && j <= g.ny - 3;
}
__device__ __forceinline__ bool y_iface_live(const Grid &g, int i, int j)
{
    return i >= 2 && i <= g.nx - 3 && j >= 2 && j <= g.ny - 4;
}

template <int DIR>
__device__ void iface_reverse(const AdjStageArgs &a, int i, int j)
{
    const Grid &g = a.g;
    const long long k = at(g, i, j);
    double *out = a.IF + (long long)DIR * IF_PLANES * g.plane + k;
    const bool live = DIR == 0 ? x_iface_live(g, i, j) : y_iface_live(g, i, j);
    if (!live) {
#pragma unroll
        for (int p = 0; p < IF_PLANES; ++p) out[p * g.plane] = 0.0;
        return;
    }
    // flux adjoint in sweep order (hlld.cu:200-233 un-shuffles the y flux)
    double nat[8], fb[8];
    if (DIR == 0) f_bar(a, i, j, nat); else g_bar(a, i, j, nat);
    // (the flux components are permuted like the cell: G = f[0,3,1,2,6,4,5,7])
#pragma unroll
    for (int s = 0; s < 8; ++s) fb[s] = nat[sweep_field<DIR>(s)];
    // interface states from cells m = -1..2 (and b_n of m = 3's neighbour)
    double cell[5][8], q[4][8];
#pragma unroll
    for (int m = 0; m < 5; ++m) {
        const int ii = DIR == 0 ? i + m - 1 : i, jj = DIR == 0 ? j : j + m - 1;
        sweep_cell<DIR>(g, a.W, ii, jj, cell[m]);
    }
#pragma unroll
    for (int m = 0; m < 4; ++m) adj::basic_param(cell[m], cell[m + 1][4], g.gamma, q[m]);
    double L[8], R[8], Lb[8], Rb[8];
    const unsigned bits = adj::muscl_states(q[0], q[1], q[2], q[3], g.eps, L, R);
#pragma unroll
    for (int c = 0; c < 8; ++c) { Lb[c] = 0.0; Rb[c] = 0.0; }
    adj::hlld_flux_adj(L, R, g.gamma, g.eps, fb, Lb, Rb);
#pragma unroll
    for (int n = 0; n < 7; ++n) {
        out[n * g.plane] = Lb[recon_comp(n)];
        out[(8 + n) * g.plane] = Rb[recon_comp(n)];
    }
    out[7 * g.plane] = Lb[adj::QBX] + Rb[adj::QBX];
    out[15 * g.plane] = __longlong_as_double((long long)bits);
}

// Reverse of the resistive hook (main_plasmoid.cu:175-290) at cell (i, j):
// the cell's eta*J enters F at interfaces i-1, i and G at j-1, j.
__device__ void resistive_reverse(const AdjStageArgs &a, int i, int j)
{
    const Grid &g = a.g;
    const long long k = at(g, i, j);
    double JXb = 0.0, JYb = 0.0, JZb = 0.0, dbX = 0.0, dbY = 0.0, dbZ = 0.0;
    if (i >= 2 && i <= g.nx - 3 && j >= 2 && j <= g.ny - 3) {
        const double *W = a.W;
        const long long P = g.plane;
        const double bXc = bx_c(g, W, i, j), bYc = by_c(g, W, i, j), bZ = W[BZF * P + k];
        const double two_dx = 2.0 * g.dx, two_dy = 2.0 * g.dy;
        const double JX = (W[BZF * P + at(g, i, j + 1)] - W[BZF * P + at(g, i, j - 1)]) / two_dy;
        const double JY = -(W[BZF * P + at(g, i + 1, j)] - W[BZF * P + at(g, i - 1, j)]) / two_dx;
        const double JZ = (by_c(g, W, i + 1, j) - by_c(g, W, i - 1, j)) / two_dx
                        - (bx_c(g, W, i, j + 1) - bx_c(g, W, i, j - 1)) / two_dy;
        const double eta = a.eta ? a.eta[k] : g.eta;
        const double ea = eta * JZ, eb = eta * JY, ec = eta * JX;
        double ab = 0.0, bb = 0.0, cb = 0.0;
        double fb[8];
        for (int ii = i - 1; ii <= i; ++ii) {
            if (ii < 1 || ii > g.nx - 3 || j < 1 || j > g.ny - 3) continue;   // hook guard
            f_bar(a, ii, j, fb);
            ab += -0.5 * fb[BYF] - 0.5 * fb[EN] * bYc;
            bb += 0.5 * fb[BZF] + 0.5 * fb[EN] * bZ;
            dbY += -0.5 * fb[EN] * ea;
            dbZ += 0.5 * fb[EN] * eb;
        }
        for (int jj = j - 1; jj <= j; ++jj) {
            if (i < 1 || i > g.nx - 3 || jj < 1 || jj > g.ny - 3) continue;
            g_bar(a, i, jj, fb);
            ab += 0.5 * fb[BXF] + 0.5 * fb[EN] * bXc;
            cb += -0.5 * fb[BZF] - 0.5 * fb[EN] * bZ;
            dbX += 0.5 * fb[EN] * ea;
            dbZ += -0.5 * fb[EN] * ec;
        }
        a.etab[k] += ab * JZ + bb * JY + cb * JX;
        JZb = eta * ab;
        JYb = eta * bb;
        JXb = eta * cb;
    }
    double *rj = a.RJ + k;
    rj[0] = JXb;
    rj[g.plane] = JYb;
    rj[2 * g.plane] = JZb;
    rj[3 * g.plane] = dbX;
    rj[4 * g.plane] = dbY;
    rj[5 * g.plane] = dbZ;
}

__global__ void __launch_bounds__(ADJ_THREADS) adj_iface_kernel(AdjStageArgs a)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)a.g.nx * a.g.ny) return;
    const int i = (int)(t / a.g.ny), j = (int)(t - (long long)i * a.g.ny);
    iface_reverse<0>(a, i, j);
    iface_reverse<1>(a, i, j);
    resistive_reverse(a, i, j);
}

// MUSCL transpose of one sweep at cell c = (i, j): the adjoint of dQ[c]
// from interfaces m = c+1 (left state, qm), c (left q, right q), c-1 (left
// qp, right qp) and c-2 (right qpp).
template <int DIR>
__device__ void gather_sweep(const AdjStageArgs &a, int i, int j, double *nat_bar)
{
    const Grid &g = a.g;
    const int n_along = DIR == 0 ? g.nx : g.ny;
    const int c = DIR == 0 ? i : j;
    const double *IFd = a.IF + (long long)DIR * IF_PLANES * g.plane;
    auto idx = [&](int m) -> long long { return DIR == 0 ? at(g, m, j) : at(g, i, m); };
    auto sel = [](unsigned bits, int n, int right) -> int { return (int)((bits >> (2 * n + (right ? 14 : 0))) & 3u); };
    double qb[8];
#pragma unroll
    for (int s = 0; s < 8; ++s) qb[s] = 0.0;
#pragma unroll
    for (int d = -2; d <= 1; ++d) {
        const int m = c + d;
        if (m < 0 || m >= n_along) continue;
        const long long km = idx(m);
        const unsigned bits = (unsigned)__double_as_longlong(IFd[15 * g.plane + km]);
#pragma unroll
        for (int n = 0; n < 7; ++n) {
            const double Lb = IFd[n * g.plane + km], Rb = IFd[(8 + n) * g.plane + km];
            const int sl = sel(bits, n, 0), sr = sel(bits, n, 1);
            double v = 0.0;
            if (d == 1) {                       // c = m - 1: qm of the left state
                if (sl == 1) v -= 0.5 * Lb;
            } else if (d == 0) {                // c = m: q of both states
                v += Lb * (1.0 + (sl == 1 ? 0.5 : 0.0) - (sl == 2 ? 0.5 : 0.0));
                if (sr == 1) v += 0.5 * Rb;
            } else if (d == -1) {               // c = m + 1: qp of both states
                if (sl == 2) v += 0.5 * Lb;
                v += Rb * (1.0 - (sr == 1 ? 0.5 : 0.0) + (sr == 2 ? 0.5 : 0.0));
            } else {                            // c = m + 2: qpp of the right state
                if (sr == 2) v -= 0.5 * Rb;
            }
            qb[recon_comp(n)] += v;
        }
        if (d == 0) qb[adj::QBX] = IFd[7 * g.plane + km];
    }
    double cell[8], cb[8];
    sweep_cell<DIR>(g, a.W, i, j, cell);
#pragma unroll
    for (int s = 0; s < 8; ++s) cb[s] = 0.0;
    adj::basic_param_adj(cell, g.gamma, qb, cb);
    // b_n of dQ[c - 1] is the average of cells c-1 and c
    if (c - 1 >= 0) cb[4] += 0.5 * IFd[7 * g.plane + idx(c - 1)];
#pragma unroll
    for (int s = 0; s < 8; ++s) nat_bar[sweep_field<DIR>(s)] += cb[s];
}

__global__ void __launch_bounds__(ADJ_THREADS) adj_gather_kernel(AdjStageArgs a)
{
    const Grid &g = a.g;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)g.nx * g.ny) return;
    const int i = (int)(t / g.ny), j = (int)(t - (long long)i * g.ny);
    const long long k = at(g, i, j), P = g.plane;
    double wb[8];
#pragma unroll
    for (int f = 0; f < 8; ++f) wb[f] = 0.0;
    if (i >= 1 && i <= g.nx - 2 && j >= 1 && j <= g.ny - 2) {
        gather_sweep<0>(a, i, j, wb);
        gather_sweep<1>(a, i, j, wb);
        // eta*J: direct B terms, and J of the neighbours (centred differences)
        const double *RJ = a.RJ;
        auto rj = [&](int p, int ii, int jj) -> double {
            if (ii < 0 || jj < 0 || ii >= g.nx || jj >= g.ny) return 0.0;
            return RJ[p * P + at(g, ii, jj)];
        };
        wb[BXF] += RJ[3 * P + k] + (rj(2, i, j + 1) - rj(2, i, j - 1)) / (2.0 * g.dy);
        wb[BYF] += RJ[4 * P + k] + (rj(2, i - 1, j) - rj(2, i + 1, j)) / (2.0 * g.dx);
        wb[BZF] += RJ[5 * P + k] + (rj(1, i + 1, j) - rj(1, i - 1, j)) / (2.0 * g.dx)
                 + (rj(0, i, j - 1) - rj(0, i, j + 1)) / (2.0 * g.dy);
    }
#pragma unroll
    for (int f = 0; f < 8; ++f) {
        if (!hydro_field(f)) continue;
        const long long kf = f * P + k;
        if (a.stage == 2) {
            a.Ustage[kf] = 0.5 * a.Ub[kf] + wb[f];   // adjoint of the stage-1 state
            a.Uin[kf] = 0.5 * a.Ub[kf];              // adjoint of the step input (U^n term)
        } else {
            a.Uin[kf] += a.Ub[kf] + wb[f];
        }
    }
    a.tmp[k] = wb[BXF];
    a.tmp[P + k] = wb[BYF];
}

__global__ void __launch_bounds__(256) adj_center_kernel(AdjStageArgs a)
{
    const Grid &g = a.g;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)g.nx * g.ny) return;
    const int i = (int)(t / g.ny), j = (int)(t - (long long)i * g.ny);
    const long long k = at(g, i, j), P = g.plane;
    const double *tx = a.tmp, *ty = a.tmp + P;
    const double cbx = (i >= 1 ? 0.5 : 1.0) * tx[k] + (i + 1 < g.nx ? 0.5 * tx[at(g, i + 1, j)] : 0.0);
    const double cby = (j >= 1 ? 0.5 : 1.0) * ty[k] + (j + 1 < g.ny ? 0.5 * ty[at(g, i, j + 1)] : 0.0);
    const long long kx = BXF * P + k, ky = BYF * P + k;
    if (a.stage == 2) {
        a.Ustage[kx] = cbx;
        a.Ustage[ky] = cby;
        a.Uin[kx] = a.Ub[kx];      // CT copies the step input's faces
        a.Uin[ky] = a.Ub[ky];
    } else {
        a.Uin[kx] += a.Ub[kx] + cbx;
        a.Uin[ky] += a.Ub[ky] + cby;
    }
}

// Transpose of periodicBoundaryY2nd (boundary.cu:73-141): the y pass ran
// last, so it is undone first.
__global__ void periodic_y_transpose(Grid g, double *Ub)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)g.nx * NFIELD) return;
    const int i = (int)(t / NFIELD), f = (int)(t - (long long)i * NFIELD);
    double *row = Ub + f * g.plane + (long long)i * g.pitch;
    for (int q = 0; q < 3; ++q) {
        row[g.ny - 6 + q] += row[q];
        row[q] = 0.0;
        row[3 + q] += row[g.ny - 3 + q];
        row[g.ny - 3 + q] = 0.0;
    }
}

// Transpose of periodicBoundaryX2nd (boundary.cu:4-57).
__global__ void periodic_x_transpose(Grid g, double *Ub)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)g.ny * NFIELD) return;
    const int j = (int)(t / NFIELD), f = (int)(t - (long long)j * NFIELD);
    double *col = Ub + f * g.plane + j;
    for (int q = 0; q < 3; ++q) {
        col[(long long)(g.nx - 6 + q) * g.pitch] += col[(long long)q * g.pitch];
        col[(long long)q * g.pitch] = 0.0;
        col[(long long)(3 + q) * g.pitch] += col[(long long)(g.nx - 3 + q) * g.pitch];
        col[(long long)(g.nx - 3 + q) * g.pitch] = 0.0;
    }
}

// Pitched plane -> dense (nx, ny) table.
__global__ void plane_to_table_kernel(Grid g, const double *plane, double *tab)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)g.nx * g.ny) return;
    const int i = (int)(t / g.ny), j = (int)(t - (long long)i * g.ny);
    tab[t] = plane[at(g, i, j)];
}

int blocks_for(long long n, int threads) { return (int)((n + threads - 1) / threads); }

}  // namespace

void launch_adjoint_stage(const AdjStageArgs &a, cudaStream_t st)
{
    const long long n = (long long)a.g.nx * a.g.ny;
    adj_iface_kernel<<<blocks_for(n, ADJ_THREADS), ADJ_THREADS, 0, st>>>(a);
    adj_gather_kernel<<<blocks_for(n, ADJ_THREADS), ADJ_THREADS, 0, st>>>(a);
    adj_center_kernel<<<blocks_for(n, 256), 256, 0, st>>>(a);
}

void launch_boundary_transpose(const Grid &g, double *Ub, cudaStream_t st)
{
    periodic_y_transpose<<<blocks_for((long long)g.nx * NFIELD, 128), 128, 0, st>>>(g, Ub);
    periodic_x_transpose<<<blocks_for((long long)g.ny * NFIELD, 128), 128, 0, st>>>(g, Ub);
}

void launch_plane_to_table(const Grid &g, const double *plane, double *tab, cudaStream_t st)
{
    plane_to_table_kernel<<<blocks_for((long long)g.nx * g.ny, 256), 256, 0, st>>>(g, plane, tab);
}

}  // namespace rmhd2d
