// adjoint_prep.cu -- first kernel of a stage's reverse sweep, compiled with
// -fmad=false: per cell, the interface primitives of both sweeps
// (calculate_half_Q.cu:4-38 on the cell-centred stage input, rounded as the
// forward step rounds them, so the reverse takes the forward's branches),
// and the reverse of the resistive hook (main_plasmoid.cu:175-290).
#include <cuda_runtime.h>

#include "adjoint_common.cuh"
#include "adjoint_core.cuh"

namespace rmhd2d {

namespace {

using namespace adjk;

// The cell's eta*J enters F at interfaces i-1, i and G at j-1, j; returns
// the adjoints of J (through eta) and the direct B adjoints of the eta*J*B
// products, and accumulates the eta adjoint.
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
            if (ii < 1 || ii > g.nx - 3 || j < 1 || j > g.ny - 3) continue;   // the hook's guard
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

__global__ void __launch_bounds__(128, 8) adj_prep_kernel(AdjStageArgs a)
{
    const Grid &g = a.g;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)g.nx * g.ny) return;
    const int i = (int)(t / g.ny), j = (int)(t - (long long)i * g.ny);
    const long long k = at(g, i, j), P = g.plane;
    if (i >= 1 && i <= g.nx - 2 && j >= 1 && j <= g.ny - 2) {
        const double *W = a.W;
        const double bxo = bx_c(g, W, i, j), byo = by_c(g, W, i, j);
        double c[8], q[8];
        c[0] = W[RHO * P + k]; c[1] = W[MX * P + k]; c[2] = W[MY * P + k]; c[3] = W[MZ * P + k];
        c[4] = bxo; c[5] = byo; c[6] = W[BZF * P + k]; c[7] = W[EN * P + k];
        adj::basic_param(c, bx_c(g, W, i + 1, j), g.gamma, q);
        double *Qx = a.Q + k;
#pragma unroll
        for (int s = 0; s < 8; ++s) Qx[s * P] = q[s];
        Qx[8 * P] = bxo;
        c[1] = W[MY * P + k]; c[2] = W[MZ * P + k]; c[3] = W[MX * P + k];
        c[4] = byo; c[5] = W[BZF * P + k]; c[6] = bxo;
        adj::basic_param(c, by_c(g, W, i, j + 1), g.gamma, q);
        double *Qy = a.Q + Q_PLANES * P + k;
#pragma unroll
        for (int s = 0; s < 8; ++s) Qy[s * P] = q[s];
        Qy[8 * P] = byo;
    }
    resistive_reverse(a, i, j);
}

}  // namespace

void launch_adjoint_prep(const AdjStageArgs &a, cudaStream_t st)
{
    const long long n = (long long)a.g.nx * a.g.ny;
    adj_prep_kernel<<<(int)((n + 127) / 128), 128, 0, st>>>(a);
}

}  // namespace rmhd2d
