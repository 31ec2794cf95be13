// stage_impl.cuh -- body of the fused stage kernel (see stage.cuh).  Included
// once per variant by stage_exact.cu and stage_fast.cu, which define
// RMHD_VARIANT and RMHD_ALL_CANDIDATES.
#pragma once

#include "stage.cuh"

#ifndef RMHD_FAST_MATH
#define RMHD_FAST_MATH 0
#endif

#ifndef RMHD_VARIANT
#error "define RMHD_VARIANT (exact or fast) before including stage_impl.cuh"
#endif

namespace rmhd2d {
namespace RMHD_VARIANT {

// ---- shared-memory carve-up (doubles) ----
// Ut [8][UI][UJ]        TMA destination: U at i0-3..i0+TI+2, j0-3..j0+TJ+2
// Rs [7][TI+2][TJ+2]    per-cell eta*J terms (reuses Ut after primitives)
// Ez [TI+1][TJ+1]       corner EMF (reuses Rs after the flux phase)
// Ps [9][TI+4][TJ+4]    primitives + centred B + both sweep pressures
// Fs [7][TI+1][TJ+2]    x fluxes f0 f1 f2 f3 f5 f6 f7 at i+1/2
// Gs [7][TI+2][TJ+1]    y fluxes g0 g1 g2 g3 g4 g6 g7 at j+1/2
constexpr int PI_ = TI + 4, PJ_ = TJ + 4;
constexpr int RI_ = TI + 2, RJ_ = TJ + 2;
constexpr int FI_ = TI + 1, FJ_ = TJ + 2;
constexpr int GI_ = TI + 2, GJ_ = TJ + 1;
constexpr int EI_ = TI + 1, EJ_ = TJ + 1;
constexpr int U_DOUBLES = NFIELD * UI * UJ;
constexpr int P_DOUBLES = 9 * PI_ * PJ_;
constexpr int F_DOUBLES = 7 * FI_ * FJ_;
constexpr int G_DOUBLES = 7 * GI_ * GJ_;
constexpr int R_DOUBLES = 7 * RI_ * RJ_;
static_assert(R_DOUBLES <= U_DOUBLES, "eta*J terms must fit in the staged-U region");
static_assert(EI_ * EJ_ <= U_DOUBLES, "corner EMF must fit in the staged-U region");
constexpr size_t SMEM_BYTES = (size_t)(U_DOUBLES + P_DOUBLES + F_DOUBLES + G_DOUBLES) * 8 + 16;
constexpr unsigned TMA_BYTES = (unsigned)(U_DOUBLES * 8);

// primitive planes in Ps
enum { P_RHO = 0, P_U, P_V, P_W, P_BXC, P_BYC, P_BZ, P_PX, P_PY };
// eta*J planes in Rs
enum { R_JX = 0, R_JY, R_JZ, R_JYBZ, R_JZBY, R_JXBZ, R_JZBX };

__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Waits for phase `phase` of the mbarrier with a bounded number of tries;
// returns false when the bound expired.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t phase)
{
    const uint32_t a = smem_addr(bar);
    for (int tries = 0; tries < 50000; ++tries) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(a), "r"(phase), "r"(20000u)
            : "memory");
        if (ok) return true;
    }
    return false;
}

template <int STAGE>
__global__ void __launch_bounds__(STAGE_THREADS, 1)
stage_kernel(const __grid_constant__ CUtensorMap tmap, const StageArgs a)
{
    extern __shared__ __align__(1024) double smem[];
    double *Ut = smem;
    double *Rs = smem;
    double *Ez = smem;
    double *Ps = smem + U_DOUBLES;
    double *Fs = Ps + P_DOUBLES;
    double *Gs = Fs + F_DOUBLES;
    uint64_t *bar = reinterpret_cast<uint64_t *>(Gs + G_DOUBLES);

    const Grid &g = a.g;
    const int tid = threadIdx.x;
    const int j0 = HALO + blockIdx.x * TJ;
    const int i0 = HALO + blockIdx.y * TI;

    // ---- stage the tile + halo: one 3-D TMA load of all 8 field planes ----
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    if (tid == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                     ::"r"(smem_addr(bar)), "r"(TMA_BYTES) : "memory");
        // x coordinate (j) = j0 - 3 = blockIdx.x * TJ: a multiple of TJ, so
        // 16-byte aligned in the global tensor as TMA requires.
        asm volatile(
            "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
            " [%0], [%1, {%3, %4, %5}], [%2];"
            ::"r"(smem_addr(Ut)), "l"(reinterpret_cast<uint64_t>(&tmap)), "r"(smem_addr(bar)),
              "r"(j0 - HALO), "r"(i0 - HALO), "r"(0)
            : "memory");
    }

    // dt of this step from the CFL reduction of the previous state
    // (resistiveMHD_2D.cu:277-291), identical in every thread.
    const double dt = step_dt(a.ctl->amax[a.parity], a.ctl->first_nan[a.parity], g.dx, g.dy, g.eps, g.eta, g.cfl);
    if (STAGE == 1 && blockIdx.x == 0 && blockIdx.y == 0 && tid == 0) {
        a.ctl->dt = dt;
        a.ctl->total_time = a.ctl->total_time + dt;
        a.ctl->amax[a.parity ^ 1] = 0ull;
        a.ctl->first_nan[a.parity ^ 1] = 0;
        a.ctl->crashed = 0;
    }

    // Every thread waits (bounded) for the staged tile; the CTA gives up as a
    // whole if any wait expired, after one more bounded wait for the copy in
    // flight, and reports it in the control block.
    const bool staged = mbar_wait_bounded(bar, 0);
    if (__syncthreads_or(!staged)) {
        if (tid == 0) {
            atomicExch(&a.ctl->error, (int)KERR_TMA_TIMEOUT);
            mbar_wait_bounded(bar, 0);
        }
        return;
    }

    const double gm = g.gamma, EPS = g.eps;
#if RMHD_FAST_MATH
    const double inv_gm1 = 1.0 / (gm - 1.0);
#endif

    // ---- primitives on (TI+4) x (TJ+4) cells ----
    // calculate_half_Q.cu:4-38 on the centred state (shift kernels,
    // resistiveMHD_2D.cu:313-337), once for the x sweep and once for the
    // permuted y sweep (hlld.cu:134-152), whose pressure sums in another order.
    for (int c = tid; c < PI_ * PJ_; c += STAGE_THREADS) {
        const int pi = c / PJ_, pj = c - pi * PJ_;
        const int ui = pi + 1, uj = pj + 1;
        const double *u0 = Ut + ui * UJ + uj;
        const int F = UI * UJ;
        const double rho = u0[RHO * F];
#if RMHD_FAST_MATH
        const double irho = __drcp_rn(rho);
        const double u = u0[MX * F] * irho;
        const double v = u0[MY * F] * irho;
        const double w = u0[MZ * F] * irho;
#else
        const double u = u0[MX * F] / rho;
        const double v = u0[MY * F] / rho;
        const double w = u0[MZ * F] / rho;
#endif
        const double bXc = 0.5 * (u0[BXF * F] + u0[BXF * F - UJ]);
        const double bYc = 0.5 * (u0[BYF * F] + u0[BYF * F - 1]);
        const double bZ = u0[BZF * F];
        const double e = u0[EN * F];
        const double px = (gm - 1.0) * (e - 0.5 * (rho * (u * u + v * v + w * w))
                        - 0.5 * (bXc * bXc + bYc * bYc + bZ * bZ));
        const double py = (gm - 1.0) * (e - 0.5 * (rho * (v * v + w * w + u * u))
                        - 0.5 * (bYc * bYc + bZ * bZ + bXc * bXc));
        double *p0 = Ps + c;
        const int PF = PI_ * PJ_;
        p0[P_RHO * PF] = rho;
        p0[P_U * PF] = u;
        p0[P_V * PF] = v;
        p0[P_W * PF] = w;
        p0[P_BXC * PF] = bXc;
        p0[P_BYC * PF] = bYc;
        p0[P_BZ * PF] = bZ;
        p0[P_PX * PF] = px;
        p0[P_PY * PF] = py;
    }
    __syncthreads();

    // ---- per-cell eta*J terms on (TI+2) x (TJ+2) cells (driver hook,
    // examples2D/plasmoid/main_plasmoid.cu:175-274) ----
    {
        const int PF = PI_ * PJ_, RF = RI_ * RJ_;
        const double two_dx = 2.0 * g.dx, two_dy = 2.0 * g.dy;
#if RMHD_FAST_MATH
        const double i2dx = 1.0 / two_dx, i2dy = 1.0 / two_dy;
#endif
        for (int c = tid; c < RF; c += STAGE_THREADS) {
            const int ri = c / RJ_, rj = c - ri * RJ_;
            const double *p0 = Ps + (ri + 1) * PJ_ + (rj + 1);
#if RMHD_FAST_MATH
            const double jY = -(p0[P_BZ * PF + PJ_] - p0[P_BZ * PF - PJ_]) * i2dx;
            const double jX = (p0[P_BZ * PF + 1] - p0[P_BZ * PF - 1]) * i2dy;
            const double jZ = (p0[P_BYC * PF + PJ_] - p0[P_BYC * PF - PJ_]) * i2dx
                            - (p0[P_BXC * PF + 1] - p0[P_BXC * PF - 1]) * i2dy;
#else
            const double jY = -(p0[P_BZ * PF + PJ_] - p0[P_BZ * PF - PJ_]) / two_dx;
            const double jX = (p0[P_BZ * PF + 1] - p0[P_BZ * PF - 1]) / two_dy;
            const double jZ = (p0[P_BYC * PF + PJ_] - p0[P_BYC * PF - PJ_]) / two_dx
                            - (p0[P_BXC * PF + 1] - p0[P_BXC * PF - 1]) / two_dy;
#endif
            const int gi = i0 - 1 + ri, gj = j0 - 1 + rj;
            double eta = g.eta;
            if (a.eta) {
                const bool in = gi < g.nx && gj < g.ny;
                eta = in ? a.eta[(long long)gi * g.pitch + gj] : 0.0;
            }
            const double eJX = eta * jX, eJY = eta * jY, eJZ = eta * jZ;
            double *r0 = Rs + c;
            r0[R_JX * RF] = eJX;
            r0[R_JY * RF] = eJY;
            r0[R_JZ * RF] = eJZ;
            r0[R_JYBZ * RF] = eJY * p0[P_BZ * PF];
            r0[R_JZBY * RF] = eJZ * p0[P_BYC * PF];
            r0[R_JXBZ * RF] = eJX * p0[P_BZ * PF];
            r0[R_JZBX * RF] = eJZ * p0[P_BXC * PF];
        }
    }
    __syncthreads();

    // ---- HLLD fluxes: F on (TI+1) x (TJ+2) x-interfaces, G on (TI+2) x (TJ+1)
    // y-interfaces (hlld.cu:110-233, muscl.cu:6-126, flux_solver.cu:10-33) ----
    {
        const int PF = PI_ * PJ_, RF = RI_ * RJ_;
        constexpr int NF = FI_ * FJ_, NG = GI_ * GJ_;
        for (int it = tid; it < NF + NG; it += STAGE_THREADS) {
            const bool isF = it < NF;
            int li, lj, step;
            const double *pc;  // cell on the left / below the interface
            if (isF) {
                li = it / FJ_; lj = it - li * FJ_;
                pc = Ps + (li + 1) * PJ_ + (lj + 1);
                step = PJ_;
            } else {
                const int t = it - NF;
                li = t / GJ_; lj = t - li * GJ_;
                pc = Ps + (li + 1) * PJ_ + (lj + 1);
                step = 1;
            }
            // sweep-frame component planes (the y sweep is the x-sweep
            // arithmetic on (rho, v, w, u, bY, bZ, bX, e), hlld.cu:134-152)
            const int cU = isF ? P_U : P_V, cV = isF ? P_V : P_W, cW = isF ? P_W : P_U;
            const int cN = isF ? P_BXC : P_BYC;   // normal B (centred)
            const int cT1 = isF ? P_BYC : P_BZ, cT2 = isF ? P_BZ : P_BXC;
            const int cP = isF ? P_PX : P_PY;
            const int comp[7] = {P_RHO, cU, cV, cW, cT1, cT2, cP};
            double qL[7], qR[7];
#pragma unroll
            for (int n = 0; n < 7; ++n) {
                const double *q = pc + comp[n] * PF;
                const double qm = q[-step], q0 = q[0], qp = q[step], qpp = q[2 * step];
                qL[n] = q0 + 0.5 * minmod(q0 - qm, qp - q0, EPS);
                qR[n] = qp - 0.5 * minmod(qp - q0, qpp - qp, EPS);
            }
            const double bn = 0.5 * (pc[cN * PF] + pc[cN * PF + step]);
            Prim L{qL[0], qL[1], qL[2], qL[3], bn, qL[4], qL[5], qL[6]};
            Prim R{qR[0], qR[1], qR[2], qR[3], bn, qR[4], qR[5], qR[6]};
            double f[8];
#if RMHD_FAST_MATH
            hlld_flux_fast(L, R, gm, inv_gm1, EPS, f);
#else
            hlld_flux<RMHD_ALL_CANDIDATES>(L, R, gm, EPS, f);
#endif
            const double *r0 = Rs + li * RJ_ + lj;   // cell (i, j) of the interface
            const int rs = isF ? RJ_ : 1;            // its neighbour across the interface
            if (isF) {
                const double f5 = f[5] - 0.5 * (r0[R_JZ * RF] + r0[R_JZ * RF + rs]);
                const double f6 = f[6] + 0.5 * (r0[R_JY * RF] + r0[R_JY * RF + rs]);
                const double f7 = f[7] + (0.5 * (r0[R_JYBZ * RF] + r0[R_JYBZ * RF + rs])
                                        - 0.5 * (r0[R_JZBY * RF] + r0[R_JZBY * RF + rs]));
                double *o = Fs + it;
                constexpr int S = NF;
                o[0 * S] = f[0]; o[1 * S] = f[1]; o[2 * S] = f[2]; o[3 * S] = f[3];
                o[4 * S] = f5; o[5 * S] = f6; o[6 * S] = f7;
            } else {
                // un-permute (hlld.cu:170-194): g1 = f3, g2 = f1, g3 = f2,
                // g4 = f6, g5 = f4 = 0, g6 = f5.
                const double g4 = f[6] + 0.5 * (r0[R_JZ * RF] + r0[R_JZ * RF + rs]);
                const double g6 = f[5] - 0.5 * (r0[R_JX * RF] + r0[R_JX * RF + rs]);
                const double g7 = f[7] + (0.5 * (r0[R_JZBX * RF] + r0[R_JZBX * RF + rs])
                                        - 0.5 * (r0[R_JXBZ * RF] + r0[R_JXBZ * RF + rs]));
                double *o = Gs + (it - NF);
                constexpr int S = NG;
                o[0 * S] = f[0]; o[1 * S] = f[3]; o[2 * S] = f[1]; o[3 * S] = f[2];
                o[4 * S] = g4; o[5 * S] = g6; o[6 * S] = g7;
            }
        }
    }
    __syncthreads();

    constexpr int SF = FI_ * FJ_, SG = GI_ * GJ_;
    const double dtdx = dt / g.dx, dtdy = dt / g.dy;

    if (STAGE == 1) {
        // ---- corner EMF (ct.cu:22-41) on (TI+1) x (TJ+1) corners ----
        for (int c = tid; c < EI_ * EJ_; c += STAGE_THREADS) {
            const int ei = c / EJ_, ej = c - ei * EJ_;
            const double eZG1 = Gs[4 * SG + ei * GJ_ + ej];
            const double eZG2 = Gs[4 * SG + (ei + 1) * GJ_ + ej];
            const double eZF1 = -1.0 * Fs[4 * SF + ei * FJ_ + ej];
            const double eZF2 = -1.0 * Fs[4 * SF + ei * FJ_ + ej + 1];
            Ez[c] = 0.25 * (eZG1 + eZG2 + eZF1 + eZF2);
        }
        __syncthreads();
    }

    // ---- update of the tile's own cells ----
    const int li = tid / TJ, lj = tid - (tid / TJ) * TJ;
    const int i = i0 + li, j = j0 + lj;
    const bool own = (i < g.nx - HALO) && (j < g.ny - HALO);
    const long long k = (long long)i * g.pitch + j;
    const long long PL = g.plane;
    const double *fR = Fs + (li + 1) * FJ_ + (lj + 1);   // F(i)
    const double *fL = fR - FJ_;                          // F(i-1)
    const double *gU = Gs + (li + 1) * GJ_ + (lj + 1);   // G(j)
    const double *gD = gU - 1;                            // G(j-1)
    // field -> flux component slot
    const int fld[6] = {RHO, MX, MY, MZ, BZF, EN};
    const int slot[6] = {0, 1, 2, 3, 5, 6};

    if (STAGE == 1) {
        if (own) {
            // oneStepFirstFunctor (resistiveMHD_2D.cu:53-86)
#pragma unroll
            for (int n = 0; n < 6; ++n) {
                const int s = slot[n];
                const double u = a.src[fld[n] * PL + k];
                a.dst[fld[n] * PL + k] = u - dtdx * (fR[s * SF] - fL[s * SF]) - dtdy * (gU[s * SG] - gD[s * SG]);
            }
            // CT_kernel (ct.cu:44-59) with the EMF of this stage
            const double *ez = Ez + (li + 1) * EJ_ + (lj + 1);
            const double bXOld = a.src[BXF * PL + k], bYOld = a.src[BYF * PL + k];
            a.dst[BXF * PL + k] = bXOld - dtdy * (ez[0] - ez[-1]);
            a.dst[BYF * PL + k] = bYOld + dtdx * (ez[0] - ez[-EJ_]);
            // Symmetric boundaries read the CT'd face bY at j = 2 (the lower
            // wall face) before replacing it (TS boundary.cu:57-88).
            if (a.row2 && j0 == HALO && lj == 0) {
                const double *e2 = Ez + (li + 1) * EJ_;
                const double bY2 = a.src[BYF * PL + k - 1];
                a.row2[i] = bY2 + dtdx * (e2[0] - e2[-EJ_]);
            }
        }
    } else {
        // oneStepSecondFunctor (resistiveMHD_2D.cu:88-130); the face B of
        // the new state equals the stage-1 CT result, which is copied.
        double nv[8];
        if (own) {
#pragma unroll
            for (int n = 0; n < 6; ++n) {
                const int s = slot[n];
                const double u = a.un[fld[n] * PL + k];
                const double ub = a.src[fld[n] * PL + k];
                nv[fld[n]] = 0.5 * (u + ub - dtdx * (fR[s * SF] - fL[s * SF]) - dtdy * (gU[s * SG] - gD[s * SG]));
            }
            nv[BXF] = a.src[BXF * PL + k];
            nv[BYF] = a.src[BYF * PL + k];
#pragma unroll
            for (int n = 0; n < 8; ++n) a.dst[n * PL + k] = nv[n];
        }
        // next step's CFL rate and the crash flag over the interior
        // (ghosts are reduced by the boundary kernel)
        unsigned long long bits = 0ull;
        int nan_e = 0;
        if (own) {
#if RMHD_FAST_MATH
            const double r = cfl_rate_fast(nv[RHO], nv[MX], nv[MY], nv[MZ], nv[BXF], nv[BYF], nv[BZF], nv[EN],
                                           gm, 1.0 / g.dx, 1.0 / g.dy);
#else
            const double r = cfl_rate(nv[RHO], nv[MX], nv[MY], nv[MZ], nv[BXF], nv[BYF], nv[BZF], nv[EN],
                                      gm, g.dx, g.dy);
#endif
            bits = rate_bits(r);
            nan_e = nv[EN] != nv[EN];
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            const unsigned long long o = __shfl_xor_sync(0xffffffffu, bits, off);
            bits = o > bits ? o : bits;
        }
        // Ps is dead after the flux phase: reuse it for the per-warp maxima.
        unsigned long long *wmax = reinterpret_cast<unsigned long long *>(Ps);
        if ((tid & 31) == 0) wmax[tid >> 5] = bits;
        const int any_nan = __syncthreads_or(nan_e);
        if (tid == 0) {
            unsigned long long m = 0ull;
            for (int w = 0; w < STAGE_THREADS / 32; ++w) m = wmax[w] > m ? wmax[w] : m;
            atomicMax(&a.ctl->amax[a.parity ^ 1], m);
            if (any_nan) atomicExch(&a.ctl->crashed, 1);
        }
    }
}

size_t stage_smem_bytes() { return SMEM_BYTES; }

int stage_regs(int stage)
{
    cudaFuncAttributes attr{};
    cudaFuncGetAttributes(&attr, stage == 1 ? (const void *)stage_kernel<1> : (const void *)stage_kernel<2>);
    return attr.numRegs;
}

void launch_stage(int stage, const CUtensorMap *tmap, const StageArgs &args, cudaStream_t stream)
{
    static bool configured = false;
    if (!configured) {
        cudaFuncSetAttribute(stage_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_BYTES);
        cudaFuncSetAttribute(stage_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_BYTES);
        configured = true;
    }
    const dim3 grid((args.g.ny - 2 * HALO + TJ - 1) / TJ, (args.g.nx - 2 * HALO + TI - 1) / TI);
    if (stage == 1)
        stage_kernel<1><<<grid, STAGE_THREADS, SMEM_BYTES, stream>>>(*tmap, args);
    else
        stage_kernel<2><<<grid, STAGE_THREADS, SMEM_BYTES, stream>>>(*tmap, args);
}

}  // namespace RMHD_VARIANT
}  // namespace rmhd2d
