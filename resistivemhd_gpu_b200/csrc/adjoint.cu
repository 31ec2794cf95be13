// adjoint.cu -- discrete adjoint of the RK2 step (dt of each step held
// fixed): the reverse of one stage, and the transpose of the periodic
// boundary.
//
// Forward stage (resistiveMHD_2D.cu:133-195), W the stage input:
//   Wc  = W with cell-centred bX, bY            (shiftUToCenterForCT)
//   F,G = HLLD(MUSCL(prim(Wc))) + eta*J terms   (flux_solver.cu, hlld.cu,
//                                                main_plasmoid.cu:175-290)
//   Ez  = (G4 + G4[i+1] - F5 - F5[j+1]) / 4     (stage 1 only, ct.cu:22-41)
//   hydro out = s_in*U0 + s*(W - dt div(F,G))   (s = 1 stage 1, 1/2 stage 2)
//   bX, bY out = CT of the step input's faces with the stage-1 Ez
// Reverse, given Ub = adjoint of the stage output after the boundary
// transpose (so every ghost entry is 0), four launches:
//   adj_prep_kernel   (adjoint_prep.cu) per cell: interface primitives of
//                     both sweeps; reverse of the eta*J terms
//   adj_iface_kernel  per interface (grid.y = sweep): F-bar or G-bar, the
//                     MUSCL states and the HLLD reverse -> adjoints of the
//                     left and right states + the minmod branches
//   adj_gather_kernel per cell: MUSCL and primitive-recovery transposes over
//                     the four interfaces of each sweep that read the cell
//                     -> adjoint of Wc (hydro part written out, centred B
//                     parked for the next kernel)
//   adj_center_kernel per cell: transpose of the face->centre averaging and
//                     of the CT copy of the step input's faces
// Compiled with fused multiply-add: the branch-deciding forward values are
// formed with explicitly rounded operations (adjoint_core.cuh).
#include <cuda_runtime.h>

#include "adjoint.h"
#include "adjoint_common.cuh"
#include "adjoint_core.cuh"

namespace rmhd2d {

void launch_adjoint_prep(const AdjStageArgs &a, cudaStream_t st);

namespace {

using namespace adjk;
using adj::recon_comp;

constexpr int ADJ_THREADS = 128;

__global__ void __launch_bounds__(ADJ_THREADS, 3) adj_iface_kernel(AdjStageArgs a)
{
    const Grid &g = a.g;
    const int dir = blockIdx.y;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)g.nx * g.ny) return;
    const int i = (int)(t / g.ny), j = (int)(t - (long long)i * g.ny);
    const long long k = at(g, i, j), P = g.plane;
    double *out = a.IF + (long long)dir * IF_PLANES * P + k;
    if (!iface_live(g, dir, i, j)) {
#pragma unroll
        for (int p = 0; p < IF_PLANES; ++p) out[p * P] = 0.0;
        return;
    }
    // flux adjoint in sweep order
    double nat[8], fb[8];
    if (dir == 0) f_bar(a, i, j, nat); else g_bar(a, i, j, nat);
#pragma unroll
    for (int s = 0; s < 8; ++s) fb[s] = nat[sweep_field(dir, s)];
    // interface primitives of cells m-1 .. m+2 along the sweep
    const double *Q = a.Q + (long long)dir * Q_PLANES * P + k;
    const long long step = dir == 0 ? g.pitch : 1;
    double q[4][8];
#pragma unroll
    for (int m = 0; m < 4; ++m)
#pragma unroll
        for (int s = 0; s < 8; ++s) q[m][s] = Q[s * P + (m - 1) * step];
    double L[8], R[8], Lb[8], Rb[8];
    const unsigned bits = adj::muscl_states(q[0], q[1], q[2], q[3], g.eps, L, R);
#pragma unroll
    for (int c = 0; c < 8; ++c) { Lb[c] = 0.0; Rb[c] = 0.0; }
    adj::hlld_flux_adj(L, R, g.gamma, g.eps, fb, Lb, Rb);
#pragma unroll
    for (int n = 0; n < 7; ++n) {
        out[n * P] = Lb[recon_comp(n)];
        out[(8 + n) * P] = Rb[recon_comp(n)];
    }
    out[7 * P] = Lb[adj::QBX] + Rb[adj::QBX];
    out[15 * P] = __longlong_as_double((long long)bits);
}

// MUSCL transpose of one sweep at cell c: the adjoint of dQ[c] from
// interfaces m = c+1 (left state, qm), c (left q, right q), c-1 (left qp,
// right qp) and c-2 (right qpp), then the primitive-recovery transpose.
// Every load is issued unconditionally (indices clamped into the grid,
// contributions from outside it masked to 0).
__device__ __forceinline__ void gather_sweep(const AdjStageArgs &a, int dir, int i, int j, double *nat_bar)
{
    const Grid &g = a.g;
    const long long P = g.plane, k = at(g, i, j);
    const int n_along = dir == 0 ? g.nx : g.ny;
    const int c = dir == 0 ? i : j;
    const long long step = dir == 0 ? g.pitch : 1;
    const double *IFd = a.IF + (long long)dir * IF_PLANES * P + k;
    const double mp1 = c + 1 < n_along ? 1.0 : 0.0, mm1 = c >= 1 ? 1.0 : 0.0, mm2 = c >= 2 ? 1.0 : 0.0;
    const double *s1 = IFd + (c + 1 < n_along ? step : 0);
    const double *s0 = IFd;
    const double *sm1 = IFd - (c >= 1 ? step : 0);
    const double *sm2 = IFd - (c >= 2 ? 2 * step : 0);
    const unsigned b1 = (unsigned)__double_as_longlong(s1[15 * P]);
    const unsigned b0 = (unsigned)__double_as_longlong(s0[15 * P]);
    const unsigned bm1 = (unsigned)__double_as_longlong(sm1[15 * P]);
    const unsigned bm2 = (unsigned)__double_as_longlong(sm2[15 * P]);
    double qb[8];
#pragma unroll
    for (int n = 0; n < 7; ++n) {
        const double L1 = s1[n * P], L0 = s0[n * P], R0 = s0[(8 + n) * P];
        const double Lm1 = sm1[n * P], Rm1 = sm1[(8 + n) * P], Rm2 = sm2[(8 + n) * P];
        auto sel = [n](unsigned bits, int right) -> unsigned { return (bits >> (2 * n + (right ? 14 : 0))) & 3u; };
        const unsigned l1 = sel(b1, 0), l0 = sel(b0, 0), r0 = sel(b0, 1), lm1 = sel(bm1, 0), rm1 = sel(bm1, 1),
                       rm2 = sel(bm2, 1);
        double v = mp1 * (l1 == 1 ? -0.5 * L1 : 0.0);
        v += L0 * (l0 == 1 ? 1.5 : (l0 == 2 ? 0.5 : 1.0)) + (r0 == 1 ? 0.5 * R0 : 0.0);
        v += mm1 * ((lm1 == 2 ? 0.5 * Lm1 : 0.0) + Rm1 * (rm1 == 1 ? 0.5 : (rm1 == 2 ? 1.5 : 1.0)));
        v += mm2 * (rm2 == 2 ? -0.5 * Rm2 : 0.0);
        qb[recon_comp(n)] = v;
    }
    qb[adj::QBX] = s0[7 * P];
    const double *Q = a.Q + (long long)dir * Q_PLANES * P + k;
    double q[8], cb[8];
#pragma unroll
    for (int s = 0; s < 8; ++s) { q[s] = Q[s * P]; cb[s] = 0.0; }
    adj::basic_param_adj(q, Q[8 * P], g.gamma, qb, cb);
    // b_n of dQ[c - 1] is the average of cells c-1 and c
    cb[4] += mm1 * 0.5 * sm1[7 * P];
#pragma unroll
    for (int s = 0; s < 8; ++s) nat_bar[sweep_field(dir, s)] += cb[s];
}

__global__ void __launch_bounds__(ADJ_THREADS, 6) adj_gather_kernel(AdjStageArgs a)
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
        gather_sweep(a, 0, i, j, wb);
        gather_sweep(a, 1, i, j, wb);
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

// Transpose of the periodic boundary (periodicBoundaryX2nd then
// periodicBoundaryY2nd, boundary.cu:4-141).  After both passes every ghost
// cell holds the interior cell (wrap(i), wrap(j)), so its adjoint moves onto
// that cell and the ghost's becomes 0.  One thread per interior cell of the
// 3-wide bands along the walls and per field gathers its images -- the
// y-wall image Jg, the x-wall image Ig and the corner (Ig, Jg) -- and zeroes
// them, summing in the order the two passes' transposes (y first, then x)
// would: (U(I,J) + U(I,Jg)) + (U(Ig,J) + U(Ig,Jg)).  Each ghost has one
// image, so no two threads touch the same entry.
__global__ void periodic_transpose_kernel(Grid g, double *Ub)
{
    const long long nrow = 6LL * (g.nx - 6);    // rows 3..5 and ny-6..ny-4, interior columns
    const long long ncol = 6LL * (g.ny - 12);   // columns 3..5 and nx-6..nx-4, rows 6..ny-7
    const long long per_field = nrow + ncol;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= per_field * NFIELD) return;
    const int f = (int)(t / per_field);
    long long u = t - (long long)f * per_field;
    int I, J;
    if (u < nrow) {
        const int r = (int)(u / (g.nx - 6));
        I = 3 + (int)(u - (long long)r * (g.nx - 6));
        J = r < 3 ? 3 + r : g.ny - 9 + r;
    } else {
        u -= nrow;
        const int c = (int)(u / (g.ny - 12));
        J = 6 + (int)(u - (long long)c * (g.ny - 12));
        I = c < 3 ? 3 + c : g.nx - 9 + c;
    }
    const int Ig = I < 6 ? I + g.nx - 6 : (I >= g.nx - 6 ? I - (g.nx - 6) : -1);
    const int Jg = J < 6 ? J + g.ny - 6 : (J >= g.ny - 6 ? J - (g.ny - 6) : -1);
    double *p = Ub + (long long)f * g.plane;
    double v = p[at(g, I, J)];
    if (Jg >= 0) {
        v = v + p[at(g, I, Jg)];
        p[at(g, I, Jg)] = 0.0;
    }
    if (Ig >= 0) {
        double w = p[at(g, Ig, J)];
        if (Jg >= 0) {
            w = w + p[at(g, Ig, Jg)];
            p[at(g, Ig, Jg)] = 0.0;
        }
        p[at(g, Ig, J)] = 0.0;
        v = v + w;
    }
    p[at(g, I, J)] = v;
}

// Transpose of the symmetric walls and of mixed periodic / symmetric walls.
// The forward (TS boundary.cu:4-205, as the oracle's tangent restates it)
// runs the x pass over every row, then the y pass over every column.  Each
// pass copies every field but the wall-normal B from the mirror cells
// (ghost 2 <- 3, 1 <- 4, 0 <- 5 and their upper twins) and integrates the
// normal B into the wall from its neighbours' tangential B, e.g. at the
// lower y wall, for column i > 0,
//   bY(i,2) = bY(i,3) + (bX(i,3) - bX(i-1,3)) dy/dx
//   bY(i,1) = bY(i,2) + (bX(i,2) - bX(i-1,2)) dy/dx      (bX(.,2) a copy of row 3)
//   bY(i,0) = bY(i,1) + (bX(i,1) - bX(i-1,1)) dy/dx      (bX(.,1) a copy of row 4)
// The transposes run in the opposite order, y then x, in gather form: a
// thread owns one column (y) or one row (x), takes the chain adjoints of
// its own and of the next column or row, and writes only its own entries;
// the ghost entries it reads are zeroed by a separate launch after it.  The
// x pass at row 3 reads the lower wall face bY(c,2) before the y pass
// replaces it -- in the step, the stage-1 CT result (row2) -- so the x
// transpose leaves that adjoint in the ghost entry (c,2) of the interior
// columns, where the stage-1 reverse takes it as the CT'd face's.

// Running sums of a lower and an upper chain's output adjoints: t1 = the
// sum of all three, t2 = the outer two, t3 = the outermost.
struct ChainAdj {
    double t1, t2, t3;
};

__device__ __forceinline__ ChainAdj chain_adj(double inner, double middle, double outer)
{
    return ChainAdj{inner + middle + outer, middle + outer, outer};
}

template <int BY> __global__ void ytrans_kernel(Grid g, double *Ub)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.nx) return;
    const long long P = g.plane;
    const int ny = g.ny;
    auto L = [&](int f, int ii, int jj) -> double & { return Ub[f * P + at(g, ii, jj)]; };
    if (BY == BC_PERIODIC) {
#pragma unroll
        for (int f = 0; f < NFIELD; ++f)
            for (int q = 0; q < 3; ++q) {
                L(f, i, ny - 6 + q) += L(f, i, q);
                L(f, i, 3 + q) += L(f, i, ny - 3 + q);
            }
        return;
    }
    const double c = g.dy / g.dx;
    auto lower = [&](int col) { return chain_adj(L(BYF, col, 2), L(BYF, col, 1), L(BYF, col, 0)); };
    auto upper = [&](int col) { return chain_adj(L(BYF, col, ny - 3), L(BYF, col, ny - 2), L(BYF, col, ny - 1)); };
    const ChainAdj lo = lower(i), up = upper(i);
    // chain terms on bX: this column's (i > 0) and the next column's
    const ChainAdj z{0.0, 0.0, 0.0};
    const ChainAdj lo_own = i > 0 ? lo : z, up_own = i > 0 ? up : z;
    const ChainAdj lo_nxt = i + 1 < g.nx ? lower(i + 1) : z, up_nxt = i + 1 < g.nx ? upper(i + 1) : z;
    L(BYF, i, 3) += lo.t1;
    L(BYF, i, ny - 4) += up.t1;
    L(BXF, i, 3) += L(BXF, i, 2) + c * (lo_own.t1 - lo_nxt.t1) + c * (lo_own.t2 - lo_nxt.t2);
    L(BXF, i, 4) += L(BXF, i, 1) + c * (lo_own.t3 - lo_nxt.t3);
    L(BXF, i, 5) += L(BXF, i, 0);
    L(BXF, i, ny - 4) += L(BXF, i, ny - 3) - c * (up_own.t1 - up_nxt.t1);
    L(BXF, i, ny - 5) += L(BXF, i, ny - 2) - c * (up_own.t2 - up_nxt.t2);
    L(BXF, i, ny - 6) += L(BXF, i, ny - 1) - c * (up_own.t3 - up_nxt.t3);
#pragma unroll
    for (int f = 0; f < NFIELD; ++f) {
        if (f == BXF || f == BYF) continue;
        L(f, i, 3) += L(f, i, 2);
        L(f, i, 4) += L(f, i, 1);
        L(f, i, 5) += L(f, i, 0);
        L(f, i, ny - 4) += L(f, i, ny - 3);
        L(f, i, ny - 5) += L(f, i, ny - 2);
        L(f, i, ny - 6) += L(f, i, ny - 1);
    }
}

// Zeroes ghost rows (ROWS) or the ghost columns of the interior rows.
template <bool ROWS> __global__ void zero_ghosts_kernel(Grid g, double *Ub)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long per_field = ROWS ? 6LL * g.nx : 6LL * (g.ny - 6);
    if (t >= per_field * NFIELD) return;
    const int f = (int)(t / per_field);
    const long long u = t - (long long)f * per_field;
    int i, j;
    if (ROWS) {
        i = (int)(u / 6);
        const int q = (int)(u - (long long)i * 6);
        j = q < 3 ? q : g.ny - 6 + q;
    } else {
        j = 3 + (int)(u / 6);
        const int q = (int)(u - (long long)(j - 3) * 6);
        i = q < 3 ? q : g.nx - 6 + q;
    }
    Ub[(long long)f * g.plane + at(g, i, j)] = 0.0;
}

// x transpose for rows 2 .. ny-4 (row 2 only gathers the lower wall face's
// adjoint from row 3's chains; every ghost row is zero by now).
template <int BX> __global__ void xtrans_kernel(Grid g, double *Ub)
{
    const int j = 2 + blockIdx.x * blockDim.x + threadIdx.x;
    if (j > g.ny - 4) return;
    const long long P = g.plane;
    const int nx = g.nx;
    auto L = [&](int f, int ii, int jj) -> double & { return Ub[f * P + at(g, ii, jj)]; };
    if (BX == BC_PERIODIC) {
        if (j < 3) return;
#pragma unroll
        for (int f = 0; f < NFIELD; ++f)
            for (int q = 0; q < 3; ++q) {
                L(f, nx - 6 + q, j) += L(f, q, j);
                L(f, 3 + q, j) += L(f, nx - 3 + q, j);
            }
        return;
    }
    const double c = g.dx / g.dy;
    auto lower = [&](int row) { return chain_adj(L(BXF, 2, row), L(BXF, 1, row), L(BXF, 0, row)); };
    auto upper = [&](int row) { return chain_adj(L(BXF, nx - 3, row), L(BXF, nx - 2, row), L(BXF, nx - 1, row)); };
    const ChainAdj z{0.0, 0.0, 0.0};
    const ChainAdj lo = j >= 3 ? lower(j) : z, up = j >= 3 ? upper(j) : z;
    const ChainAdj lo_nxt = lower(j + 1), up_nxt = upper(j + 1);
    // the chains' bY terms at this row: + from its own chain, - from the next
    // row's (its j-1), through the copies 2 <- 3 and 1 <- 4
    L(BYF, 3, j) += c * (lo.t1 - lo_nxt.t1) + c * (lo.t2 - lo_nxt.t2);
    L(BYF, 4, j) += c * (lo.t3 - lo_nxt.t3);
    L(BYF, nx - 4, j) -= c * (up.t1 - up_nxt.t1);
    L(BYF, nx - 5, j) -= c * (up.t2 - up_nxt.t2);
    L(BYF, nx - 6, j) -= c * (up.t3 - up_nxt.t3);
    if (j < 3) return;
    L(BXF, 3, j) += lo.t1;
    L(BXF, nx - 4, j) += up.t1;
#pragma unroll
    for (int f = 0; f < NFIELD; ++f) {
        if (f == BXF) continue;
        L(f, 3, j) += L(f, 2, j);
        L(f, 4, j) += L(f, 1, j);
        L(f, 5, j) += L(f, 0, j);
        L(f, nx - 4, j) += L(f, nx - 3, j);
        L(f, nx - 5, j) += L(f, nx - 2, j);
        L(f, nx - 6, j) += L(f, nx - 1, j);
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
    launch_adjoint_prep(a, st);
    adj_iface_kernel<<<dim3(blocks_for(n, ADJ_THREADS), 2), ADJ_THREADS, 0, st>>>(a);
    adj_gather_kernel<<<blocks_for(n, ADJ_THREADS), ADJ_THREADS, 0, st>>>(a);
    adj_center_kernel<<<blocks_for(n, 256), 256, 0, st>>>(a);
}

void launch_boundary_transpose(const Grid &g, double *Ub, cudaStream_t st)
{
    if (g.bc_x == BC_PERIODIC && g.bc_y == BC_PERIODIC) {
        const long long n = (6LL * (g.nx - 6) + 6LL * (g.ny - 12)) * NFIELD;
        periodic_transpose_kernel<<<blocks_for(n, 256), 256, 0, st>>>(g, Ub);
        return;
    }
    if (g.bc_y == BC_PERIODIC)
        ytrans_kernel<BC_PERIODIC><<<blocks_for(g.nx, 128), 128, 0, st>>>(g, Ub);
    else
        ytrans_kernel<BC_SYMMETRIC><<<blocks_for(g.nx, 128), 128, 0, st>>>(g, Ub);
    zero_ghosts_kernel<true><<<blocks_for(6LL * g.nx * NFIELD, 256), 256, 0, st>>>(g, Ub);
    if (g.bc_x == BC_PERIODIC)
        xtrans_kernel<BC_PERIODIC><<<blocks_for(g.ny - 5, 128), 128, 0, st>>>(g, Ub);
    else
        xtrans_kernel<BC_SYMMETRIC><<<blocks_for(g.ny - 5, 128), 128, 0, st>>>(g, Ub);
    zero_ghosts_kernel<false><<<blocks_for(6LL * (g.ny - 6) * NFIELD, 256), 256, 0, st>>>(g, Ub);
}

void launch_plane_to_table(const Grid &g, const double *plane, double *tab, cudaStream_t st)
{
    plane_to_table_kernel<<<blocks_for((long long)g.nx * g.ny, 256), 256, 0, st>>>(g, plane, tab);
}

}  // namespace rmhd2d
