// stage_impl.cuh -- body of the fused stage kernel (see stage.cuh).  Included
// once per variant by stage_exact.cu and stage_fast.cu, which define
// RMHD_VARIANT, RMHD_ALL_CANDIDATES and RMHD_FAST_MATH.
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

// ---- per-stage tile geometry and shared-memory carve-up (doubles) ----
// Ut [8][UI][UJ]        TMA: U at i0-3..i0+TI+2, j0-3..j0+TJ+2 (kept for the whole CTA)
// Et [UI][UJ]           TMA: eta table on the same cells (when a table is set)
// Ps [7][TI+4][TJ+4]    u, v, w, centred bX, centred bY, x- and y-sweep pressures
// Rs [3][TI+2][TJ+2]    eta*Jx, eta*Jy, eta*Jz per cell; reused for the corner EMF
// Fs [NC][TI+1][F_NJ]   x fluxes f0 f1 f2 f3 f6 f7 (+ f5 in stage 1) at i+1/2
// Gs [NC][G_NI][TJ+1]   y fluxes g0 g1 g2 g3 g6 g7 (+ g4 in stage 1) at j+1/2
// Stage 1 needs x fluxes on rows j0-1..j0+TJ and y fluxes on columns
// i0-1..i0+TI for its corner EMF; stage 2 only the tile's own interfaces and
// no EMF components.
template <int STAGE> struct Tile {
    static constexpr int TI = stage_ti(STAGE);
    static constexpr int UI = TI + 2 * HALO;
    static constexpr int PI_ = TI + 4, PJ_ = TJ + 4;
    static constexpr int RI_ = TI + 2, RJ_ = TJ + 2;
    static constexpr int NC = STAGE == 1 ? 7 : 6;            // flux components stored
    static constexpr int F_NI = TI + 1;
    static constexpr int F_J0 = STAGE == 1 ? -1 : 0;         // row of fj = 0, relative to j0
    static constexpr int F_NJ = STAGE == 1 ? TJ + 2 : TJ;
    static constexpr int G_I0 = STAGE == 1 ? -1 : 0;         // column of gi = 0, relative to i0
    static constexpr int G_NI = STAGE == 1 ? TI + 2 : TI;
    static constexpr int G_NJ = TJ + 1;
    static constexpr int EI_ = TI + 1, EJ_ = TJ + 1;
    static constexpr int UF = UI * UJ;                       // doubles per staged field
    static constexpr int PF = PI_ * PJ_;
    static constexpr int RF = RI_ * RJ_;
    static constexpr int SF = F_NI * F_NJ;
    static constexpr int SG = G_NI * G_NJ;
    static constexpr int NF = SF, NG = SG;                   // interfaces per sweep
    static constexpr int U_DOUBLES = NFIELD * UF;
    static constexpr int E_DOUBLES = UF;
    static constexpr int P_DOUBLES = 7 * PF;
    static constexpr int R_DOUBLES = 3 * RF;
    static constexpr int F_DOUBLES = NC * SF;
    static constexpr int G_DOUBLES = NC * SG;
    static constexpr size_t SMEM_BYTES =
        (size_t)(U_DOUBLES + E_DOUBLES + P_DOUBLES + R_DOUBLES + F_DOUBLES + G_DOUBLES) * 8 + 16;
    static constexpr unsigned U_BYTES = (unsigned)(U_DOUBLES * 8);
    static constexpr unsigned E_BYTES = (unsigned)(E_DOUBLES * 8);
    static_assert(STAGE != 1 || EI_ * EJ_ <= R_DOUBLES, "corner EMF must fit in the eta*J region");
    static_assert(STAGE_THREADS / 32 <= P_DOUBLES, "per-warp maxima must fit in the primitive region");
    // Two CTAs per SM (228 KB of shared memory, 1 KB reserved per CTA).
    static_assert(SMEM_BYTES <= 113 * 1024, "shared memory for two CTAs per SM");
};

// primitive planes in Ps (rho and bZ are read from the staged tile)
enum { P_U = 0, P_V, P_W, P_BXC, P_BYC, P_PX, P_PY };
// eta*J planes in Rs
enum { R_JX = 0, R_JY, R_JZ };
// flux component slots: 0..5 the hydro fields rho, rhoU, rhoV, rhoW, bZ, e;
// slot 6 (stage 1) the EMF component F.f5 / G.f4.
constexpr int SLOT_EMF = 6;

__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Waits for phase `phase` of the mbarrier with a bounded number of tries
// (each try suspends for at most 20 us); false when the bound expired.
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
__global__ void __launch_bounds__(STAGE_THREADS, 2)
stage_kernel(const __grid_constant__ CUtensorMap tmap, const __grid_constant__ CUtensorMap emap,
             const StageArgs a)
{
    using T = Tile<STAGE>;
    constexpr int TI = T::TI, UF = T::UF, PF = T::PF, RF = T::RF, SF = T::SF, SG = T::SG;
    constexpr int PJ_ = T::PJ_, RJ_ = T::RJ_, F_NJ = T::F_NJ, G_NJ = T::G_NJ, EJ_ = T::EJ_;
    extern __shared__ __align__(1024) double smem[];
    double *Ut = smem;
    double *Et = Ut + T::U_DOUBLES;
    double *Ps = Et + T::E_DOUBLES;
    double *Rs = Ps + T::P_DOUBLES;
    double *Ez = Rs;
    double *Fs = Rs + T::R_DOUBLES;
    double *Gs = Fs + T::F_DOUBLES;
    uint64_t *bar = reinterpret_cast<uint64_t *>(Gs + T::G_DOUBLES);

    const Grid &g = a.g;
    const int tid = threadIdx.x;
    const int j0 = HALO + blockIdx.x * TJ;
    const int i0 = HALO + blockIdx.y * TI;
    const bool has_eta = a.eta != nullptr;

    // ---- stage the tile + halo: one 3-D TMA load of all 8 field planes
    // (and one 2-D load of the eta table) ----
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    if (tid == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                     ::"r"(smem_addr(bar)), "r"(T::U_BYTES + (has_eta ? T::E_BYTES : 0u)) : "memory");
        // x coordinate (j) = j0 - 3 = blockIdx.x * TJ: a multiple of TJ, so
        // 16-byte aligned in the global tensor as TMA requires.
        asm volatile(
            "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
            " [%0], [%1, {%3, %4, %5}], [%2];"
            ::"r"(smem_addr(Ut)), "l"(reinterpret_cast<uint64_t>(&tmap)), "r"(smem_addr(bar)),
              "r"(j0 - HALO), "r"(i0 - HALO), "r"(0)
            : "memory");
        if (has_eta)
            asm volatile(
                "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
                " [%0], [%1, {%3, %4}], [%2];"
                ::"r"(smem_addr(Et)), "l"(reinterpret_cast<uint64_t>(&emap)), "r"(smem_addr(bar)),
                  "r"(j0 - HALO), "r"(i0 - HALO)
                : "memory");
    }

    // own cell of this thread in the update phase
    const int li = tid / TJ, lj = tid - (tid / TJ) * TJ;
    const int i = i0 + li, j = j0 + lj;
    const bool own = (tid < TI * TJ) && (i < g.nx - HALO) && (j < g.ny - HALO);
    const long long k = (long long)i * g.pitch + j;
    const long long PL = g.plane;
    if (STAGE == 2 && own) {
        // U^n is read only at the end; start pulling it into L2 now.
#pragma unroll
        for (int f = 0; f < NFIELD; ++f)
            if (f != BXF && f != BYF)
                asm volatile("prefetch.global.L2 [%0];" ::"l"(__cvta_generic_to_global(a.un + f * PL + k)));
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
    for (int c = tid; c < PF; c += STAGE_THREADS) {
        const int pi = c / PJ_, pj = c - pi * PJ_;
        const double *u0 = Ut + (pi + 1) * UJ + (pj + 1);
        const double rho = u0[RHO * UF];
#if RMHD_FAST_MATH
        const double irho = rcp_nr(rho);
        const double u = u0[MX * UF] * irho;
        const double v = u0[MY * UF] * irho;
        const double w = u0[MZ * UF] * irho;
#else
        const double u = u0[MX * UF] / rho;
        const double v = u0[MY * UF] / rho;
        const double w = u0[MZ * UF] / rho;
#endif
        const double bXc = 0.5 * (u0[BXF * UF] + u0[BXF * UF - UJ]);
        const double bYc = 0.5 * (u0[BYF * UF] + u0[BYF * UF - 1]);
        const double bZ = u0[BZF * UF];
        const double e = u0[EN * UF];
        const double px = (gm - 1.0) * (e - 0.5 * (rho * (u * u + v * v + w * w))
                        - 0.5 * (bXc * bXc + bYc * bYc + bZ * bZ));
        const double py = (gm - 1.0) * (e - 0.5 * (rho * (v * v + w * w + u * u))
                        - 0.5 * (bYc * bYc + bZ * bZ + bXc * bXc));
        double *p0 = Ps + c;
        p0[P_U * PF] = u;
        p0[P_V * PF] = v;
        p0[P_W * PF] = w;
        p0[P_BXC * PF] = bXc;
        p0[P_BYC * PF] = bYc;
        p0[P_PX * PF] = px;
        p0[P_PY * PF] = py;
    }
    __syncthreads();

    // ---- eta*J on (TI+2) x (TJ+2) cells (driver hook,
    // examples2D/plasmoid/main_plasmoid.cu:175-274) ----
    {
        const double two_dx = 2.0 * g.dx, two_dy = 2.0 * g.dy;
#if RMHD_FAST_MATH
        const double i2dx = 1.0 / two_dx, i2dy = 1.0 / two_dy;
#endif
        for (int c = tid; c < RF; c += STAGE_THREADS) {
            const int ri = c / RJ_, rj = c - ri * RJ_;
            const double *p0 = Ps + (ri + 1) * PJ_ + (rj + 1);
            const double *z0 = Ut + BZF * UF + (ri + 2) * UJ + (rj + 2);
#if RMHD_FAST_MATH
            const double jY = -(z0[UJ] - z0[-UJ]) * i2dx;
            const double jX = (z0[1] - z0[-1]) * i2dy;
            const double jZ = (p0[P_BYC * PF + PJ_] - p0[P_BYC * PF - PJ_]) * i2dx
                            - (p0[P_BXC * PF + 1] - p0[P_BXC * PF - 1]) * i2dy;
#else
            const double jY = -(z0[UJ] - z0[-UJ]) / two_dx;
            const double jX = (z0[1] - z0[-1]) / two_dy;
            const double jZ = (p0[P_BYC * PF + PJ_] - p0[P_BYC * PF - PJ_]) / two_dx
                            - (p0[P_BXC * PF + 1] - p0[P_BXC * PF - 1]) / two_dy;
#endif
            const double eta = has_eta ? Et[(ri + 2) * UJ + (rj + 2)] : g.eta;
            double *r0 = Rs + c;
            r0[R_JX * RF] = eta * jX;
            r0[R_JY * RF] = eta * jY;
            r0[R_JZ * RF] = eta * jZ;
        }
    }
    __syncthreads();

    // ---- HLLD fluxes (hlld.cu:110-233, muscl.cu:6-126, flux_solver.cu:10-33)
    // with the resistive terms ----
    for (int it = tid; it < T::NF + T::NG; it += STAGE_THREADS) {
        const bool isF = it < T::NF;
        int a0, a1;   // (fi, fj) or (gi, gj)
        int ci, cj;   // the cell left of / below the interface, relative to (i0, j0)
        if (isF) {
            a0 = it / F_NJ;
            a1 = it - a0 * F_NJ;
            ci = a0 - 1;
            cj = a1 + T::F_J0;
        } else {
            const int t = it - T::NF;
            a0 = t / G_NJ;
            a1 = t - a0 * G_NJ;
            ci = a0 + T::G_I0;
            cj = a1 - 1;
        }
        const double *uc = Ut + (ci + HALO) * UJ + (cj + HALO);
        const double *pc = Ps + (ci + 2) * PJ_ + (cj + 2);
        const double *r0 = Rs + (ci + 1) * RJ_ + (cj + 1);
        const int us = isF ? UJ : 1, ps = isF ? PJ_ : 1;
        // sweep-frame components (the y sweep runs the x-sweep arithmetic on
        // (rho, v, w, u, bY, bZ, bX, e), hlld.cu:134-152)
        const double *cp[7] = {uc + RHO * UF,
                               pc + (isF ? P_U : P_V) * PF,
                               pc + (isF ? P_V : P_W) * PF,
                               pc + (isF ? P_W : P_U) * PF,
                               isF ? pc + P_BYC * PF : uc + BZF * UF,
                               isF ? uc + BZF * UF : pc + P_BXC * PF,
                               pc + (isF ? P_PX : P_PY) * PF};
        const int cs[7] = {us, ps, ps, ps, isF ? ps : us, isF ? us : ps, ps};
        double qL[7], qR[7];
#pragma unroll
        for (int n = 0; n < 7; ++n) {
            const double *q = cp[n];
            const int st = cs[n];
            const double qm = q[-st], q0 = q[0], qp = q[st], qpp = q[2 * st];
            qL[n] = q0 + 0.5 * minmod(q0 - qm, qp - q0, EPS);
            qR[n] = qp - 0.5 * minmod(qp - q0, qpp - qp, EPS);
        }
        const double *nb = pc + (isF ? P_BXC : P_BYC) * PF;
        const double bn = 0.5 * (nb[0] + nb[ps]);
        const Prim L{qL[0], qL[1], qL[2], qL[3], bn, qL[4], qL[5], qL[6]};
        const Prim R{qR[0], qR[1], qR[2], qR[3], bn, qR[4], qR[5], qR[6]};
        double f[8];
#if RMHD_FAST_MATH
        hlld_flux_fast(L, R, gm, inv_gm1, EPS, f);
#else
        hlld_flux<RMHD_ALL_CANDIDATES>(L, R, gm, EPS, f);
#endif
        // eta*J of the two cells sharing the interface and their B
        const int rs = isF ? RJ_ : 1;
        const double z0 = uc[BZF * UF], z1 = uc[BZF * UF + us];
        if (isF) {
            const double eY0 = r0[R_JY * RF], eY1 = r0[R_JY * RF + rs];
            const double eZ0 = r0[R_JZ * RF], eZ1 = r0[R_JZ * RF + rs];
            const double y0 = pc[P_BYC * PF], y1 = pc[P_BYC * PF + ps];
            const double f6 = f[6] + 0.5 * (eY0 + eY1);
            const double f7 = f[7] + (0.5 * (eY0 * z0 + eY1 * z1) - 0.5 * (eZ0 * y0 + eZ1 * y1));
            double *o = Fs + a0 * F_NJ + a1;
            o[0 * SF] = f[0]; o[1 * SF] = f[1]; o[2 * SF] = f[2]; o[3 * SF] = f[3];
            o[4 * SF] = f6; o[5 * SF] = f7;
            if (STAGE == 1) o[SLOT_EMF * SF] = f[5] - 0.5 * (eZ0 + eZ1);
        } else {
            const double eX0 = r0[R_JX * RF], eX1 = r0[R_JX * RF + rs];
            const double eZ0 = r0[R_JZ * RF], eZ1 = r0[R_JZ * RF + rs];
            const double x0 = pc[P_BXC * PF], x1 = pc[P_BXC * PF + ps];
            // un-permute (hlld.cu:170-194): g1 = f3, g2 = f1, g3 = f2,
            // g4 = f6, g5 = f4 = 0, g6 = f5.
            const double g6 = f[5] - 0.5 * (eX0 + eX1);
            const double g7 = f[7] + (0.5 * (eZ0 * x0 + eZ1 * x1) - 0.5 * (eX0 * z0 + eX1 * z1));
            double *o = Gs + a0 * G_NJ + a1;
            o[0 * SG] = f[0]; o[1 * SG] = f[3]; o[2 * SG] = f[1]; o[3 * SG] = f[2];
            o[4 * SG] = g6; o[5 * SG] = g7;
            if (STAGE == 1) o[SLOT_EMF * SG] = f[6] + 0.5 * (eZ0 + eZ1);
        }
    }
    __syncthreads();

    const double dtdx = dt / g.dx, dtdy = dt / g.dy;

    if (STAGE == 1) {
        // ---- corner EMF (ct.cu:22-41) on (TI+1) x (TJ+1) corners (i, j) =
        // (i0-1+ei, j0-1+ej), i.e. Fs (fi, fj) = (ei, ej) and Gs (gi, gj) = (ei, ej) ----
        for (int c = tid; c < T::EI_ * EJ_; c += STAGE_THREADS) {
            const int ei = c / EJ_, ej = c - ei * EJ_;
            const double eZG1 = Gs[SLOT_EMF * SG + ei * G_NJ + ej];
            const double eZG2 = Gs[SLOT_EMF * SG + (ei + 1) * G_NJ + ej];
            const double eZF1 = -1.0 * Fs[SLOT_EMF * SF + ei * F_NJ + ej];
            const double eZF2 = -1.0 * Fs[SLOT_EMF * SF + ei * F_NJ + ej + 1];
            Ez[c] = 0.25 * (eZG1 + eZG2 + eZF1 + eZF2);
        }
        __syncthreads();
    }

    // ---- update of the tile's own cells ----
    const double *fR = Fs + (li + 1) * F_NJ + (lj - T::F_J0);    // F(i)
    const double *fL = fR - F_NJ;                                  // F(i-1)
    const double *gU = Gs + (li - T::G_I0) * G_NJ + (lj + 1);    // G(j)
    const double *gD = gU - 1;                                     // G(j-1)
    const double *uo = Ut + (li + HALO) * UJ + (lj + HALO);        // own cell in the staged tile
    const int fld[6] = {RHO, MX, MY, MZ, BZF, EN};

    if (STAGE == 1) {
        if (own) {
            // oneStepFirstFunctor (resistiveMHD_2D.cu:53-86)
#pragma unroll
            for (int n = 0; n < 6; ++n)
                a.dst[fld[n] * PL + k] = uo[fld[n] * UF] - dtdx * (fR[n * SF] - fL[n * SF])
                                       - dtdy * (gU[n * SG] - gD[n * SG]);
            // CT_kernel (ct.cu:44-59) with the EMF of this stage
            const double *ez = Ez + (li + 1) * EJ_ + (lj + 1);
            a.dst[BXF * PL + k] = uo[BXF * UF] - dtdy * (ez[0] - ez[-1]);
            a.dst[BYF * PL + k] = uo[BYF * UF] + dtdx * (ez[0] - ez[-EJ_]);
            // Symmetric boundaries read the CT'd face bY at j = 2 (the lower
            // wall face) before replacing it (TS boundary.cu:57-88).
            if (a.row2 && j0 == HALO && lj == 0) {
                const double *e2 = Ez + (li + 1) * EJ_;
                a.row2[i] = uo[BYF * UF - 1] + dtdx * (e2[0] - e2[-EJ_]);
            }
        }
    } else {
        // oneStepSecondFunctor (resistiveMHD_2D.cu:88-130); the face B of
        // the new state equals the stage-1 CT result, which is copied.
        double nv[8];
        if (own) {
#pragma unroll
            for (int n = 0; n < 6; ++n) {
                const double u = a.un[fld[n] * PL + k];
                const double ub = uo[fld[n] * UF];
                nv[fld[n]] = 0.5 * (u + ub - dtdx * (fR[n * SF] - fL[n * SF]) - dtdy * (gU[n * SG] - gD[n * SG]));
            }
            nv[BXF] = uo[BXF * UF];
            nv[BYF] = uo[BYF * UF];
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

size_t stage_smem_bytes(int stage) { return stage == 1 ? Tile<1>::SMEM_BYTES : Tile<2>::SMEM_BYTES; }

int stage_regs(int stage)
{
    cudaFuncAttributes attr{};
    cudaFuncGetAttributes(&attr, stage == 1 ? (const void *)stage_kernel<1> : (const void *)stage_kernel<2>);
    return attr.numRegs;
}

void launch_stage(int stage, const CUtensorMap *tmap, const CUtensorMap *emap, const StageArgs &args,
                  cudaStream_t stream)
{
    if (stage == 1) {
        constexpr size_t sm = Tile<1>::SMEM_BYTES;
        cudaFuncSetAttribute(stage_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        const dim3 grid((args.g.ny - 2 * HALO + TJ - 1) / TJ, (args.g.nx - 2 * HALO + Tile<1>::TI - 1) / Tile<1>::TI);
        stage_kernel<1><<<grid, STAGE_THREADS, sm, stream>>>(*tmap, *emap, args);
    } else {
        constexpr size_t sm = Tile<2>::SMEM_BYTES;
        cudaFuncSetAttribute(stage_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        const dim3 grid((args.g.ny - 2 * HALO + TJ - 1) / TJ, (args.g.nx - 2 * HALO + Tile<2>::TI - 1) / Tile<2>::TI);
        stage_kernel<2><<<grid, STAGE_THREADS, sm, stream>>>(*tmap, *emap, args);
    }
}

}  // namespace RMHD_VARIANT
}  // namespace rmhd2d
