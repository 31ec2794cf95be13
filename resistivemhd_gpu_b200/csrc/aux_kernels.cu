// aux_kernels.cu -- boundary fill, CFL reduction and layout conversion for
// librmhd2d.  Compiled with -fmad=false: the symmetric boundary's div-B
// integration and the CFL rate must round exactly as the reference does.
#include <cuda_runtime.h>

#include "aux_kernels.h"
#include "physics.cuh"

namespace rmhd2d {

namespace {

__device__ __forceinline__ long long at(const Grid &g, int i, int j) { return (long long)i * g.pitch + j; }

// Mirror index of the symmetric boundary (TS boundary.cu:9-52): ghost 0,1,2
// take cells 5,4,3 and ghost n-1,n-2,n-3 take n-6,n-5,n-4.
__device__ __forceinline__ int mirror(int c, int n)
{
    if (c < 3) return 5 - c;
    if (c >= n - 3) return 2 * n - 7 - c;
    return c;
}

// A column that holds cells of the domain's interior: the interior columns
// of the array and, in a slab of a decomposed domain, its halo columns
// (copies of the neighbouring slab's own columns).
__device__ __forceinline__ bool x_inner(const Grid &g, int i)
{
    return (i >= 3 || (g.x_halo & 1)) && (i < g.nx - 3 || (g.x_halo & 2));
}

// A halo column of a slab (filled by the exchange, never by the ghost fill).
__device__ __forceinline__ bool halo_col(const Grid &g, int i)
{
    return (i < 3 && (g.x_halo & 1)) || (i >= g.nx - 3 && (g.x_halo & 2));
}

// Periodic wrap (boundary.cu:9-57, period n-6).
__device__ __forceinline__ int wrap(int c, int n)
{
    if (c < 3) return c + n - 6;
    if (c >= n - 3) return c - (n - 6);
    return c;
}


// bY seen by the x-wall integration at interior column c and row r: the
// lower-wall face row (r = 2) holds the stage's constrained-transport value
// (row2), which the symmetric y pass replaces only afterwards.
__device__ __forceinline__ double bY_prewall(const Grid &g, const double *bY, const double *row2, int c, int r)
{
    return r == 2 ? row2[c] : bY[at(g, c, r)];
}

// x-wall ghost bX at ghost column c, interior row r
// (TS boundary.cu:56-88 symmetricBoundaryX2ndBX_kernel, 0 < j branch).
__device__ double bX_xghost(const Grid &g, const double *bX, const double *bY, const double *row2, int c, int r)
{
    const double dx = g.dx, dy = g.dy;
    const int nx = g.nx;
    if (c < 3) {
        const double d3 = (bY_prewall(g, bY, row2, 3, r) - bY_prewall(g, bY, row2, 3, r - 1)) / dy * dx;
        double b = bX[at(g, 3, r)] + d3;          // column 2
        if (c == 2) return b;
        b = b + (bY_prewall(g, bY, row2, 3, r) - bY_prewall(g, bY, row2, 3, r - 1)) / dy * dx;  // column 1 (bY copied from 3)
        if (c == 1) return b;
        return b + (bY_prewall(g, bY, row2, 4, r) - bY_prewall(g, bY, row2, 4, r - 1)) / dy * dx;  // column 0 (bY from 4)
    }
    double b = bX[at(g, nx - 4, r)]
             - (bY_prewall(g, bY, row2, nx - 4, r) - bY_prewall(g, bY, row2, nx - 4, r - 1)) / dy * dx;  // nx-3
    if (c == nx - 3) return b;
    b = b - (bY_prewall(g, bY, row2, nx - 5, r) - bY_prewall(g, bY, row2, nx - 5, r - 1)) / dy * dx;       // nx-2
    if (c == nx - 2) return b;
    return b - (bY_prewall(g, bY, row2, nx - 6, r) - bY_prewall(g, bY, row2, nx - 6, r - 1)) / dy * dx;    // nx-1
}

// The multi-GPU library's wall states (ResistiveMHD_multiGPU_cuda/
// ResistiveMHD2D_GPU/boundary.cu:63-84, 212-229): from cell c, density,
// normal B and bZ kept, tangential bY 0, velocity 0 (the conducting wall)
// or only v kept (the flare's line-tied wall), energy rebuilt from the
// cell's pressure (computed with its face B).
template <bool KEEP_V>
__device__ __forceinline__ void mc_wall_state(const double *c, double gm, double *out)
{
    const double rho = c[RHO];
    const double u = c[MX] / rho, v = c[MY] / rho, w = c[MZ] / rho;
    const double bX = c[BXF], bY = c[BYF], bZ = c[BZF], e = c[EN];
    const double p = (gm - 1.0) * (e - 0.5 * rho * (u * u + v * v + w * w) - 0.5 * (bX * bX + bY * bY + bZ * bZ));
    const double vk = KEEP_V ? v : 0.0;
    out[RHO] = rho;
    out[MX] = rho * 0.0;
    out[MY] = KEEP_V ? rho * v : rho * 0.0;
    out[MZ] = rho * 0.0;
    out[BXF] = bX;
    out[BYF] = 0.0;
    out[BZF] = bZ;
    out[EN] = p / (gm - 1.0) + 0.5 * rho * (0.0 * 0.0 + vk * vk + 0.0 * 0.0) + 0.5 * (bX * bX + 0.0 * 0.0 + bZ * bZ);
}

__device__ __forceinline__ void load_cell(const Grid &g, const double *s, int i, int j, double *v)
{
#pragma unroll
    for (int f = 0; f < NFIELD; ++f) v[f] = s[f * g.plane + at(g, i, j)];
}

// The cell (i, j) after the x pass (any column, an interior row j): the cell
// itself in interior columns, else the x wall's rule -- periodic copy
// (boundary.cu:4-57), mirror copy with the integrated bX (TS
// boundary.cu:4-104), copy of the nearest interior column (zero gradient,
// the multi-GPU library's boundary.cu:231-243), or the flare's line-tied
// state at x = xmin and a copy at x = xmax (boundary.cu:196-245).
// BX is the x wall kind, or -1 to read it from g (batches of mixed walls).
template <int BX>
__device__ void after_x_cell(const Grid &g, const double *s, const double *row2, int i, int j, double *v)
{
    if (x_inner(g, i)) {
        load_cell(g, s, i, j, v);
        return;
    }
    switch (BX >= 0 ? BX : g.bc_x) {
    case BC_PERIODIC:
        load_cell(g, s, wrap(i, g.nx), j, v);
        return;
    case BC_SYMMETRIC:
        load_cell(g, s, mirror(i, g.nx), j, v);
        v[BXF] = bX_xghost(g, s + BXF * g.plane, s + BYF * g.plane, row2, i, j);
        return;
    case BC_FLARE:
        if (i < 3) {
            double c[NFIELD];
            load_cell(g, s, 3, j, c);
            mc_wall_state<true>(c, g.gamma, v);
            return;
        }
        load_cell(g, s, g.nx - 4, j, v);
        return;
    default:   // BC_ZERO_GRADIENT
        load_cell(g, s, i < 3 ? 3 : g.nx - 4, j, v);
        return;
    }
}

template <int BX>
__device__ __forceinline__ double after_x_field(const Grid &g, const double *s, const double *row2, int f, int i,
                                                int j)
{
    const int kx = BX >= 0 ? BX : g.bc_x;
    if (x_inner(g, i)) return s[f * g.plane + at(g, i, j)];
    if (kx == BC_PERIODIC) return s[f * g.plane + at(g, wrap(i, g.nx), j)];
    if (kx == BC_SYMMETRIC)
        return f == BXF ? bX_xghost(g, s + BXF * g.plane, s + BYF * g.plane, row2, i, j)
                        : s[f * g.plane + at(g, mirror(i, g.nx), j)];
    double v[NFIELD];
    after_x_cell<BX>(g, s, row2, i, j, v);
    return v[f];
}

// y-wall ghost bY at column i, ghost row j of the mirror wall, from the x
// pass's result (TS boundary.cu:159-188 symmetricBoundaryY2ndBY_kernel).
template <int BX>
__device__ double bY_yghost(const Grid &g, const double *s, const double *row2, int i, int j)
{
    const double dx = g.dx, dy = g.dy;
    const int ny = g.ny;
    auto bx = [&](int c, int r) { return after_x_field<BX>(g, s, row2, BXF, c, r); };
    if (j < 3) {
        double b = after_x_field<BX>(g, s, row2, BYF, i, 3);
        if (i == 0) return b;
        const double s3 = (bx(i, 3) - bx(i - 1, 3)) / dx * dy;
        b = b + s3;                                   // row 2
        if (j == 2) return b;
        b = b + (bx(i, 3) - bx(i - 1, 3)) / dx * dy;  // row 1
        if (j == 1) return b;
        return b + (bx(i, 4) - bx(i - 1, 4)) / dx * dy;  // row 0
    }
    double b = after_x_field<BX>(g, s, row2, BYF, i, ny - 4);
    if (i == 0) return b;
    b = b - (bx(i, ny - 4) - bx(i - 1, ny - 4)) / dx * dy;  // ny-3
    if (j == ny - 3) return b;
    b = b - (bx(i, ny - 5) - bx(i - 1, ny - 5)) / dx * dy;  // ny-2
    if (j == ny - 2) return b;
    return b - (bx(i, ny - 6) - bx(i - 1, ny - 6)) / dx * dy;  // ny-1
}

// Maps a linear ghost-cell index to (i, j): first the 6 ghost columns
// (all rows, j contiguous), then the 6 ghost rows of the interior columns.
__device__ __forceinline__ void ghost_cell(const Grid &g, long long t, int &i, int &j)
{
    const long long ncol = 6LL * g.ny;
    if (t < ncol) {
        const int c = (int)(t / g.ny);
        j = (int)(t - (long long)c * g.ny);
        i = c < 3 ? c : g.nx - 6 + c;
    } else {
        const long long u = t - ncol;
        const int w = g.nx - 6;
        const int r = (int)(u / w);
        i = 3 + (int)(u - (long long)r * w);
        j = r < 3 ? r : g.ny - 6 + r;
    }
}

// Fills ghost cell number t of `s` from its interior (and, for mirror x
// walls, the CT'd lower-wall bY row), with the exact results of the
// reference's x pass followed by its y pass.  Every ghost's value reads only
// interior rows of the x pass's result, which reads only interior columns,
// so no ghost cell is read and the in-place fill is race free.  Returns the
// cell's CFL rate bits and NaN-energy flag when `rate` is set.
template <int BX, int BY>
__device__ __forceinline__ void fill_ghost(const Grid &g, double *s, const double *row2, long long t, bool rate,
                                           unsigned long long &bits, int &nan_e, bool &cell0_nan)
{
    int i, j;
    ghost_cell(g, t, i, j);
    if (halo_col(g, i)) return;   // a slab's halo comes from its neighbour
    const long long P = g.plane;
    const long long k = at(g, i, j);
    double v[8];
    if (j >= 3 && j < g.ny - 3) {
        after_x_cell<BX>(g, s, row2, i, j, v);
    } else {
        switch (BY >= 0 ? BY : g.bc_y) {
        case BC_PERIODIC:                       // boundary.cu:73-141
            after_x_cell<BX>(g, s, row2, i, wrap(j, g.ny), v);
            break;
        case BC_SYMMETRIC:                      // TS boundary.cu:107-205
            after_x_cell<BX>(g, s, row2, i, mirror(j, g.ny), v);
            v[BYF] = bY_yghost<BX>(g, s, row2, i, j);
            break;
        case BC_WALL: {                         // boundary.cu:48-119
            double c[NFIELD];
            after_x_cell<BX>(g, s, row2, i, j < 3 ? 3 : g.ny - 4, c);
            mc_wall_state<false>(c, g.gamma, v);
            break;
        }
        default:                                // BC_ZERO_GRADIENT, boundary.cu:292-337
            after_x_cell<BX>(g, s, row2, i, j < 3 ? 3 : g.ny - 4, v);
            break;
        }
    }
#pragma unroll
    for (int f = 0; f < 8; ++f) s[f * P + k] = v[f];
    if (rate) {
        const double r = cfl_rate(v[RHO], v[MX], v[MY], v[MZ], v[BXF], v[BYF], v[BZF], v[EN], g.gamma, g.dx, g.dy);
        bits = rate_bits(r);
        nan_e = v[EN] != v[EN];
        cell0_nan = (i == 0 && j == 0 && r != r);
    }
}

__device__ __forceinline__ void reduce_ghost_rates(Control *ctl, int slot, unsigned long long bits, int nan_e,
                                                   bool cell0_nan)
{
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const unsigned long long o = __shfl_xor_sync(0xffffffffu, bits, off);
        bits = o > bits ? o : bits;
    }
    const int any_nan = __any_sync(0xffffffffu, nan_e);
    if (cell0_nan) ctl->first_nan[slot] = 1;
    if ((threadIdx.x & 31) == 0) {
        if (bits) atomicMax(&ctl->amax[slot], bits);
        if (any_nan) atomicExch(&ctl->crashed, 1);
    }
}

// Field f of ghost cell (i, j): fill_ghost's value of that field alone.
template <int BX, int BY>
__device__ __forceinline__ double ghost_field(const Grid &g, const double *s, const double *row2, int i, int j, int f)
{
    if (j >= 3 && j < g.ny - 3) return after_x_field<BX>(g, s, row2, f, i, j);
    switch (BY >= 0 ? BY : g.bc_y) {
    case BC_PERIODIC:
        return after_x_field<BX>(g, s, row2, f, i, wrap(j, g.ny));
    case BC_SYMMETRIC:
        return f == BYF ? bY_yghost<BX>(g, s, row2, i, j) : after_x_field<BX>(g, s, row2, f, i, mirror(j, g.ny));
    case BC_WALL: {
        const int r = j < 3 ? 3 : g.ny - 4;
        if (f == RHO || f == BXF || f == BZF) return after_x_field<BX>(g, s, row2, f, i, r);
        if (f != EN) return f == BYF ? 0.0 : after_x_field<BX>(g, s, row2, RHO, i, r) * 0.0;
        double c[NFIELD], v[NFIELD];
        after_x_cell<BX>(g, s, row2, i, r, c);
        mc_wall_state<false>(c, g.gamma, v);
        return v[EN];
    }
    default:   // BC_ZERO_GRADIENT
        return after_x_field<BX>(g, s, row2, f, i, j < 3 ? 3 : g.ny - 4);
    }
}

// Every ghost cell of one run, one thread per (ghost cell, field): a block
// of GHOST_CELLS x 8 threads holds GHOST_CELLS consecutive ghost cells, warp
// f their field f, so that each thread follows only its own field's
// dependences (a copy, or one wall-normal B integration chain) and the
// launch spreads over every SM.  With `ctl` set the block's first warp also
// folds the ghost cells' CFL rate and NaN-energy test into the reductions of
// the stage-2 kernel (slot = the next step's parity), from the 8 values the
// block staged in shared memory.  The values are fill_ghost's, bit for bit.
constexpr int GHOST_CELLS = 32;
template <int BX, int BY>
__global__ void __launch_bounds__(GHOST_CELLS * NFIELD)
boundary_kernel(Grid g, double *s, const double *row2, Control *ctl, int slot)
{
    __shared__ double sv[NFIELD][GHOST_CELLS];
    const long long nghost = 6LL * g.ny + 6LL * (g.nx - 6);
    const int lane = threadIdx.x & 31, f = threadIdx.x >> 5;
    const long long t = (long long)blockIdx.x * GHOST_CELLS + lane;
    int i = 0, j = 0;
    bool live = false;
    if (t < nghost) {
        ghost_cell(g, t, i, j);
        live = !halo_col(g, i);   // a slab's halo comes from its neighbour
    }
    if (live) {
        const double v = ghost_field<BX, BY>(g, s, row2, i, j, f);
        s[f * g.plane + at(g, i, j)] = v;
        if (ctl) sv[f][lane] = v;
    }
    if (!ctl) return;
    __syncthreads();
    if (f != 0) return;
    unsigned long long bits = 0ull;
    int nan_e = 0;
    bool c0 = false;
    if (live) {
        const double r = cfl_rate(sv[RHO][lane], sv[MX][lane], sv[MY][lane], sv[MZ][lane], sv[BXF][lane],
                                  sv[BYF][lane], sv[BZF][lane], sv[EN][lane], g.gamma, g.dx, g.dy);
        bits = rate_bits(r);
        nan_e = sv[EN][lane] != sv[EN][lane];
        c0 = (i == 0 && j == 0 && r != r);
    }
    reduce_ghost_rates(ctl, slot, bits, nan_e, c0);
}

// Every ghost cell of every run of a batch (blockIdx.y = run); `which`
// selects the state (0: B after stage 1, 1: A after stage 2 with the CFL
// and NaN reductions).
__global__ void boundary_batch_kernel(const BatchRun *runs, int which, int slot)
{
    const BatchRun &r = runs[blockIdx.y];
    const Grid &g = r.g;
    const long long nghost = 6LL * g.ny + 6LL * (g.nx - 6);
    const long long first = (long long)blockIdx.x * blockDim.x;
    if (first >= nghost) return;   // whole warp-aligned block beyond this run
    const long long t = first + threadIdx.x;
    unsigned long long bits = 0ull;
    int nan_e = 0;
    bool c0 = false;
    const bool rate = which == 1;
    if (t < nghost) fill_ghost<-1, -1>(g, which == 1 ? r.A : r.B, r.row2, t, rate, bits, nan_e, c0);
    if (rate) reduce_ghost_rates(r.ctl, slot, bits, nan_e, c0);
}

// Copies the lower-wall face row bY(i, 2) into row2 (used when the boundary
// is applied to a state that did not come from a stage, e.g. after set_state).
__global__ void snapshot_row2_kernel(Grid g, const double *s, double *row2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < g.nx) row2[i] = s[BYF * g.plane + at(g, i, 2)];
}

// CFL rate over every cell (resistiveMHD_2D.cu:247-291) and the NaN-energy
// test (resistiveMHD_2D.cu:294-309).
__global__ void rate_kernel(Grid g, const double *s, Control *ctl, int slot, int set_crash)
{
    const long long n = (long long)g.nx * g.ny;
    unsigned long long bits = 0ull;
    int nan_e = 0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t / g.ny), j = (int)(t - (long long)i * g.ny);
        if (halo_col(g, i)) continue;   // a slab's halo cells are reduced by their owner
        const long long k = at(g, i, j);
        const long long P = g.plane;
        const double e = s[EN * P + k];
        const double r = cfl_rate(s[RHO * P + k], s[MX * P + k], s[MY * P + k], s[MZ * P + k],
                                  s[BXF * P + k], s[BYF * P + k], s[BZF * P + k], e, g.gamma, g.dx, g.dy);
        const unsigned long long b = rate_bits(r);
        bits = b > bits ? b : bits;
        if (t == 0 && r != r) ctl->first_nan[slot] = 1;
        nan_e |= (e != e);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const unsigned long long o = __shfl_xor_sync(0xffffffffu, bits, off);
        bits = o > bits ? o : bits;
    }
    const int any_nan = __any_sync(0xffffffffu, nan_e);
    if ((threadIdx.x & 31) == 0) {
        atomicMax(&ctl->amax[slot], bits);
        if (set_crash && any_nan) atomicExch(&ctl->crashed, 1);
    }
}

// AoS (reference layout, cell k = j + i*ny, 8 doubles) <-> SoA planes.
__global__ void aos_to_planes_kernel(Grid g, const double *aos, double *s)
{
    const long long n = (long long)g.nx * g.ny;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n * 8; t += (long long)gridDim.x * blockDim.x) {
        const long long cell = t >> 3;
        const int f = (int)(t & 7);
        const int i = (int)(cell / g.ny), j = (int)(cell - (long long)i * g.ny);
        s[f * g.plane + at(g, i, j)] = aos[t];
    }
}

__global__ void planes_to_aos_kernel(Grid g, const double *s, double *aos)
{
    const long long n = (long long)g.nx * g.ny;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n * 8; t += (long long)gridDim.x * blockDim.x) {
        const long long cell = t >> 3;
        const int f = (int)(t & 7);
        const int i = (int)(cell / g.ny), j = (int)(cell - (long long)i * g.ny);
        aos[t] = s[f * g.plane + at(g, i, j)];
    }
}

// Dense (nx, ny) table -> pitched plane.
__global__ void table_to_plane_kernel(Grid g, const double *tab, double *plane)
{
    const long long n = (long long)g.nx * g.ny;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t / g.ny), j = (int)(t - (long long)i * g.ny);
        plane[at(g, i, j)] = tab[t];
    }
}

// Slab halo exchange: the 3 columns starting at col0 (all rows, all fields)
// to (to_buf) or from a packed buffer laid out [field][3 columns][pitch].
__global__ void slab_halo_kernel(Grid g, double *s, double *buf, int col0, int to_buf)
{
    const long long per_field = 3LL * g.pitch;
    const long long n = NFIELD * per_field;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const long long f = t / per_field;
        double *p = s + f * g.plane + (long long)col0 * g.pitch + (t - f * per_field);
        if (to_buf) buf[t] = *p;
        else *p = buf[t];
    }
}

// The first slab of a periodic-x decomposition holds the domain's ghost
// column 0 in its low halo, copied from the last slab's column nx-6.  A
// mirror y wall fills column 0's ghost bY without the div-B integration, for
// want of a column to its left (TS boundary.cu:159-188 at i = 0), where the
// copied column integrated: restore those 6 values.  The copies' CFL rates
// were reduced by their owner, these 6 cells' are reduced here, with cell
// (0, 0)'s NaN test for first_nan.  One thread per ghost row.
__global__ void slab_origin_column_kernel(Grid g, double *s, Control *ctl, int slot)
{
    const int t = threadIdx.x;
    if (t >= 6) return;
    const int j = t < 3 ? t : g.ny - 6 + t;
    const long long P = g.plane;
    const long long k = at(g, 0, j);
    if (g.bc_y == BC_SYMMETRIC) s[BYF * P + k] = s[BYF * P + at(g, 0, j < 3 ? 3 : g.ny - 4)];
    const double r = cfl_rate(s[RHO * P + k], s[MX * P + k], s[MY * P + k], s[MZ * P + k], s[BXF * P + k],
                              s[BYF * P + k], s[BZF * P + k], s[EN * P + k], g.gamma, g.dx, g.dy);
    const unsigned long long b = rate_bits(r);
    if (b) atomicMax(&ctl->amax[slot], b);
    if (j == 0 && r != r) ctl->first_nan[slot] = 1;
}

// The reductions a decomposed domain combines across slabs: w = [amax bits
// of slot, first_nan of slot, crashed], to (to_buf) or from the buffer.
__global__ void slab_words_kernel(Control *ctl, int slot, long long *w, int to_buf)
{
    if (to_buf) {
        w[0] = (long long)ctl->amax[slot];
        w[1] = ctl->first_nan[slot];
        w[2] = ctl->crashed;
    } else {
        ctl->amax[slot] = (unsigned long long)w[0];
        ctl->first_nan[slot] = (int)w[1];
        ctl->crashed = (int)w[2];
    }
}

int grid_for(long long n, int threads)
{
    long long b = (n + threads - 1) / threads;
    if (b > 148LL * 32) b = 148LL * 32;
    return (int)(b < 1 ? 1 : b);
}

}  // namespace

void launch_boundary(const Grid &g, double *s, const double *row2, Control *ctl, int slot, cudaStream_t st)
{
    const long long nghost = 6LL * g.ny + 6LL * (g.nx - 6);
    const int threads = GHOST_CELLS * NFIELD;
    const int blocks = (int)((nghost + GHOST_CELLS - 1) / GHOST_CELLS);
    // one instantiation per (x, y) wall pair; the y kind is a template
    // argument under each x kind
    auto launch = [&](auto kernel) { kernel<<<blocks, threads, 0, st>>>(g, s, row2, ctl, slot); };
#define RMHD_BY(BXK)                                                                                   \
    switch (g.bc_y) {                                                                                  \
    case BC_PERIODIC: launch(boundary_kernel<BXK, BC_PERIODIC>); break;                                \
    case BC_SYMMETRIC: launch(boundary_kernel<BXK, BC_SYMMETRIC>); break;                              \
    case BC_WALL: launch(boundary_kernel<BXK, BC_WALL>); break;                                        \
    default: launch(boundary_kernel<BXK, BC_ZERO_GRADIENT>); break;                                    \
    }
    switch (g.bc_x) {
    case BC_PERIODIC: RMHD_BY(BC_PERIODIC) break;
    case BC_SYMMETRIC: RMHD_BY(BC_SYMMETRIC) break;
    case BC_FLARE: RMHD_BY(BC_FLARE) break;
    default: RMHD_BY(BC_ZERO_GRADIENT) break;
    }
#undef RMHD_BY
}

void launch_boundary_batch(const BatchRun *runs, int nruns, long long max_ghost, int which, int slot, cudaStream_t st)
{
    const int threads = 256;
    const dim3 grid((unsigned)((max_ghost + threads - 1) / threads), (unsigned)nruns);
    boundary_batch_kernel<<<grid, threads, 0, st>>>(runs, which, slot);
}

void launch_snapshot_row2(const Grid &g, const double *s, double *row2, cudaStream_t st)
{
    snapshot_row2_kernel<<<(g.nx + 255) / 256, 256, 0, st>>>(g, s, row2);
}

void launch_rate(const Grid &g, const double *s, Control *ctl, int slot, int set_crash, cudaStream_t st)
{
    rate_kernel<<<grid_for((long long)g.nx * g.ny, 256), 256, 0, st>>>(g, s, ctl, slot, set_crash);
}

void launch_slab_halo(const Grid &g, double *s, double *buf, int col0, int to_buf, cudaStream_t st)
{
    slab_halo_kernel<<<grid_for(8LL * 3 * g.pitch, 256), 256, 0, st>>>(g, s, buf, col0, to_buf);
}

void launch_slab_origin_column(const Grid &g, double *s, Control *ctl, int slot, cudaStream_t st)
{
    slab_origin_column_kernel<<<1, 32, 0, st>>>(g, s, ctl, slot);
}

void launch_slab_words(Control *ctl, int slot, long long *w, int to_buf, cudaStream_t st)
{
    slab_words_kernel<<<1, 1, 0, st>>>(ctl, slot, w, to_buf);
}

void launch_aos_to_planes(const Grid &g, const double *aos, double *s, cudaStream_t st)
{
    aos_to_planes_kernel<<<grid_for((long long)g.nx * g.ny * 8, 256), 256, 0, st>>>(g, aos, s);
}

void launch_planes_to_aos(const Grid &g, const double *s, double *aos, cudaStream_t st)
{
    planes_to_aos_kernel<<<grid_for((long long)g.nx * g.ny * 8, 256), 256, 0, st>>>(g, s, aos);
}

void launch_table_to_plane(const Grid &g, const double *tab, double *plane, cudaStream_t st)
{
    table_to_plane_kernel<<<grid_for((long long)g.nx * g.ny, 256), 256, 0, st>>>(g, tab, plane);
}

}  // namespace rmhd2d
