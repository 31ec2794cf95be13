// stage_impl.cuh -- body of the fused stage kernel (see stage.cuh).  Included
// once per variant by stage_exact.cu, stage_fast.cu and stage_bulk32.cu,
// which define RMHD_VARIANT and, as they need them, RMHD_FAST_MATH,
// RMHD_REAL and RMHD_BULK.
#pragma once

#include "stage.cuh"
#include "tma_ptx.cuh"

#ifndef RMHD_FAST_MATH
#define RMHD_FAST_MATH 0
#endif

#ifndef RMHD_BULK
#define RMHD_BULK 0
#endif

#ifndef RMHD_REAL
#define RMHD_REAL double
#endif

// Whether the flux planes overlay the staged tile (and the update reads its
// own cell from global memory).  The FP64 variants spill registers in the
// flux phase and gain from the L1 the smaller block leaves; FP32-bulk does
// not spill, and its persistent batch kernel measured 1.3 % faster reading
// the own cell from the staged tile.  Shapes of 3 CTAs per SM overlay in
// every variant, to fit.
#ifndef RMHD_OVERLAY
#define RMHD_OVERLAY (!RMHD_BULK)
#endif

#ifndef RMHD_VARIANT
#error "define RMHD_VARIANT (exact or fast) before including stage_impl.cuh"
#endif

namespace rmhd2d {
namespace RMHD_VARIANT {

// Threads per CTA of a stage and tile shape in this variant.  Shapes 0 and 1
// run at 384 threads (80 registers, 24 warps per SM) where that measured
// faster than 320 (96 registers, 20 warps): both stages of FP32-bulk, whose
// single-precision flux body spills little at 80 registers (3-7 %), and
// stage 1 of FP64-fast (3 %).  The exact variant and FP64-fast's stage 2
// keep 320: at 80 registers their FP64 bodies spill 550-590 bytes and were
// 2-8 % slower.
constexpr int variant_threads(int stage, int shape)
{
    return shape >= 2 ? shape_threads(shape)
                      : ((RMHD_BULK || (RMHD_FAST_MATH && stage == 1)) ? 384 : shape_threads(shape));
}

// ---- per-stage tile geometry and shared-memory carve-up ----
// Ut [8][UI][UJ] f64     TMA: U at i0-3..i0+TI+2, j0-3..j0+TJ+2
// Et [UI][UJ] f64        TMA: eta table on the same cells (when a table is set)
// Pv [4][TI+4][TJ+4]     u, v, w, rho (flux-side type)
// Pb [5][TI+4][TJ+4] f64 centred bX, centred bY, x- and y-sweep pressures, bZ
// Rs [3][TI+2][TJ+2]     eta*Jx, eta*Jy, eta*Jz (flux-side type)
// Fm [3][TI+1][F_NJ] f64 x fluxes of rhoU, rhoV, rhoW at i+1/2
// Fo [NO][TI+1][F_NJ]    x fluxes of rho, bZ, e (+ bY = EMF part, stage 1), flux-side type
// Gm, Go                 the same for the y fluxes at j+1/2 (Go slot 3: the bX flux)
// Stage 1 needs x fluxes on rows j0-1..j0+TJ and y fluxes on columns
// i0-1..i0+TI for its corner EMF; stage 2 only the tile's own interfaces.
// Ut is read only by the primitive phase (and, without RMHD_OVERLAY, the
// update) and Et by the eta*J phase, which copy into Pv / Pb what the later
// phases need (rho, bZ).  With RMHD_OVERLAY the update reads its own cell
// from global memory, Rs overlays Ut and the flux planes overlay both:
// about 73 KB per CTA instead of 104-113 KB in shape 0, so that two CTAs
// take 164 KB of the SM's unified L1 / shared memory and leave 92 KB
// (instead of 28) to the cache, where the flux phase's register spills go.
template <int STAGE, int SHAPE> struct Tile {
    using Real = RMHD_REAL;                                  // flux-side arithmetic type
    static constexpr int TI = stage_ti(STAGE, SHAPE);
    static constexpr int TJ = shape_tj(SHAPE);
    static constexpr int UJ = shape_uj(SHAPE);
    static constexpr int UI = TI + 2 * HALO;
    static constexpr int PI_ = TI + 4, PJ_ = TJ + 4;
    static constexpr int RI_ = TI + 2, RJ_ = TJ + 2;
    static constexpr int NO = STAGE == 1 ? 4 : 3;            // non-momentum flux components stored
    static constexpr int F_NI = TI + 1;
    static constexpr int F_J0 = STAGE == 1 ? -1 : 0;         // row of fj = 0, relative to j0
    static constexpr int F_NJ = STAGE == 1 ? TJ + 2 : TJ;
    static constexpr int G_I0 = STAGE == 1 ? -1 : 0;         // column of gi = 0, relative to i0
    static constexpr int G_NI = STAGE == 1 ? TI + 2 : TI;
    static constexpr int G_NJ = TJ + 1;
    static constexpr int UF = UI * UJ;                       // doubles per staged field
    static constexpr int PF = PI_ * PJ_;
    static constexpr int RF = RI_ * RJ_;
    static constexpr int SF = F_NI * F_NJ;
    static constexpr int SG = G_NI * G_NJ;
    static constexpr int NF = SF, NG = SG;                   // interfaces per sweep
    static constexpr size_t up16(size_t b) { return (b + 15) / 16 * 16; }
    static constexpr size_t U_BYTES_ = (size_t)NFIELD * UF * 8;
    static constexpr size_t E_BYTES_ = (size_t)UF * 8;
    static constexpr size_t PV_BYTES = up16((size_t)4 * PF * sizeof(Real));
    static constexpr size_t PB_BYTES = up16((size_t)5 * PF * 8);
    static constexpr size_t R_ETA = (size_t)3 * RF * sizeof(Real);
    static constexpr size_t R_BYTES = up16(R_ETA);
    static constexpr size_t FM_BYTES = up16((size_t)3 * SF * 8);
    static constexpr size_t FO_BYTES = up16((size_t)NO * SF * sizeof(Real));
    static constexpr size_t GM_BYTES = up16((size_t)3 * SG * 8);
    static constexpr size_t GO_BYTES = up16((size_t)NO * SG * sizeof(Real));
    static constexpr size_t up128(size_t b) { return (b + 127) / 128 * 128; }
    // With RMHD_OVERLAY the staged tile (Et, then Ut) and the flux planes
    // share the start of the block, and Rs follows the flux planes over the
    // rest of Ut: Ut is dead after the primitive phase, Et after the eta*J
    // phase, and the flux planes are written only after the eta*J barrier.
    // Without it they follow the staged tile.
    static constexpr size_t OFF_E = 0;
    static constexpr size_t OFF_U = up128(E_BYTES_);          // TMA destinations: 128-byte aligned
    static constexpr size_t STAGED_END = OFF_U + U_BYTES_;
    static constexpr bool OVERLAY = RMHD_OVERLAY || shape_max_ctas(SHAPE) >= 3;
    static constexpr size_t OFF_FM = OVERLAY ? 0 : STAGED_END;
    static constexpr size_t OFF_FO = OFF_FM + FM_BYTES;
    static constexpr size_t OFF_GM = OFF_FO + FO_BYTES;
    static constexpr size_t OFF_GO = OFF_GM + GM_BYTES;
    static constexpr size_t OFF_R = OFF_GO + GO_BYTES;
    static constexpr size_t R_END = OFF_R + R_BYTES;
    static constexpr size_t OFF_PV = STAGED_END > R_END ? STAGED_END : R_END;
    static constexpr size_t OFF_PB = OFF_PV + PV_BYTES;
    static constexpr size_t OFF_BAR = OFF_PB + PB_BYTES;
    static constexpr size_t SMEM_BYTES = OFF_BAR + 16;
    static constexpr unsigned U_BYTES = (unsigned)U_BYTES_;
    static constexpr unsigned E_BYTES = (unsigned)E_BYTES_;
    static constexpr int THREADS = variant_threads(STAGE, SHAPE);
    static constexpr int CTAS = shape_max_ctas(SHAPE);
    static_assert(THREADS / 32 * 8 <= PB_BYTES, "per-warp maxima must fit in the primitive region");
    static_assert(OFF_R >= OFF_U, "the eta*J planes must not overlay the staged eta table");
    // CTAS CTAs per SM (228 KB of shared memory, 1 KB reserved per CTA).
    static_assert(SMEM_BYTES <= (228 / CTAS - 1) * 1024, "shared memory for the CTAs per SM");
};

// velocity and density planes (Pv) and B / pressure planes (Pb)
enum { V_U = 0, V_V, V_W, V_RHO };
enum { B_XC = 0, B_YC, B_PX, B_PY, B_Z };
// eta*J planes in Rs
enum { R_JX = 0, R_JY, R_JZ };
// non-momentum flux slots (Fo / Go): rho, bZ, e, and in stage 1 the EMF
// component (F: bY flux f5, G: bX flux g4)
enum { O_RHO = 0, O_BZ = 1, O_EN = 2, O_EMF = 3 };

// FP64 value + single-precision limited slope (MUSCL, muscl.cu:6-126): the
// differences are taken in FP64, the minmod in single precision.
__device__ __forceinline__ void muscl_dev(double qm, double q0, double qp, double qpp, float eps, double &qL,
                                          double &qR)
{
    const double d0 = q0 - qm, d1 = qp - q0, d2 = qpp - qp;
    const float mL = minmod((float)d0, (float)d1, eps);
    const float mR = minmod((float)d1, (float)d2, eps);
    qL = q0 + (double)(0.5f * mL);
    qR = qp - (double)(0.5f * mR);
}

// Tries of the bounded wait for the staged tile.  A separate test build of
// the library (RMHD_TEST_WAIT_EXPIRY, tests/test_gpu_wait_expiry.py) issues
// no tile load and gives up after a few tries, so that the expiry path --
// error flag, RMHD2D_ERR_KERNEL, a usable context afterwards -- is exercised
// without a fault.
#if defined(RMHD_TEST_WAIT_EXPIRY)
constexpr int STAGE_WAIT_TRIES = 4;
#else
constexpr int STAGE_WAIT_TRIES = 50000;
#endif

// Waits for phase `phase` of the mbarrier with a bounded number of tries
// (each try suspends for at most 20 us); false when the bound expired.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t phase)
{
    for (int tries = 0; tries < STAGE_WAIT_TRIES; ++tries)
        if (mbar_try_wait(bar, phase)) return true;
    return false;
}

// A tile's staging: its run's tensor maps, its tile index, and whether the
// run has an eta table.
struct TileLoad {
    const CUtensorMap *tmap, *emap;
    int ti, tj;
    bool eta;
};

// Stages a tile and its halo (thread 0 only): one 3-D TMA load of all 8
// field planes and one 2-D load of the eta table, completing the CTA's
// mbarrier phase.
template <int STAGE, int SHAPE>
__device__ __forceinline__ void issue_tile_load(const TileLoad &n, unsigned char *smem_raw, uint64_t *bar)
{
    using T = Tile<STAGE, SHAPE>;
    // order this CTA's earlier shared-memory accesses before the async copy
    fence_proxy_async();
    mbar_expect_tx(bar, T::U_BYTES + (n.eta ? T::E_BYTES : 0u));
#if !defined(RMHD_TEST_WAIT_EXPIRY)
    // x coordinate (j) = j0 - 3 = tj * TJ: a multiple of TJ (even), so
    // 16-byte aligned in the global tensor as TMA requires.
    const int x = n.tj * T::TJ, y = n.ti * T::TI;
    tma_load_3d(smem_raw + T::OFF_U, n.tmap, bar, x, y, 0);
    if (n.eta) tma_load_2d(smem_raw + T::OFF_E, n.emap, bar, x, y);
#else
    (void)smem_raw;
#endif
}

// One tile of one stage: stage the tile and its halo (`load`), then the
// primitive, eta*J, flux, EMF and update phases.  (ti, tj) is the tile index
// of the run, `phase` the parity of the CTA's mbarrier for this tile's load,
// and ctl_tile marks the tile that updates the run's control block.
// Returns false when the bounded wait for the staged tile expired (the CTA
// must stop).
template <int STAGE, int SHAPE>
__device__ __forceinline__ bool stage_tile(const StageArgs &a, const TileLoad &load, bool ctl_tile,
                                           unsigned char *smem_raw, uint64_t *bar, uint32_t phase)
{
    using T = Tile<STAGE, SHAPE>;
    using Real = typename T::Real;
    constexpr int TI = T::TI, TJ = T::TJ, UJ = T::UJ, UF = T::UF, PF = T::PF, RF = T::RF, SF = T::SF, SG = T::SG;
    constexpr int PJ_ = T::PJ_, RJ_ = T::RJ_, F_NJ = T::F_NJ, G_NJ = T::G_NJ;
    double *Ut = reinterpret_cast<double *>(smem_raw + T::OFF_U);
    double *Et = reinterpret_cast<double *>(smem_raw + T::OFF_E);
    Real *Pv = reinterpret_cast<Real *>(smem_raw + T::OFF_PV);
    double *Pb = reinterpret_cast<double *>(smem_raw + T::OFF_PB);
    Real *Rs = reinterpret_cast<Real *>(smem_raw + T::OFF_R);
    double *Fm = reinterpret_cast<double *>(smem_raw + T::OFF_FM);
    Real *Fo = reinterpret_cast<Real *>(smem_raw + T::OFF_FO);
    double *Gm = reinterpret_cast<double *>(smem_raw + T::OFF_GM);
    Real *Go = reinterpret_cast<Real *>(smem_raw + T::OFF_GO);

    const Grid &g = a.g;
    const int tid = threadIdx.x;
    const int j0 = HALO + load.tj * TJ;
    const int i0 = HALO + load.ti * TI;
    const bool has_eta = a.eta != nullptr;

    if (tid == 0) issue_tile_load<STAGE, SHAPE>(load, smem_raw, bar);

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
                prefetch_l2(a.un + f * PL + k);
    }

    // dt of this step from the CFL reduction of the previous state
    // (resistiveMHD_2D.cu:277-291), identical in every thread, unless the
    // run holds dt fixed (a recorded trajectory being replayed): read from
    // dt_in, or the control block's dt_fixed.
    const double dt = a.dt_in ? *a.dt_in
                    : a.ctl->use_fixed_dt
                          ? a.ctl->dt_fixed
                          : step_dt(a.ctl->amax[a.parity], a.ctl->first_nan[a.parity], g.dx, g.dy, g.eps, g.eta, g.cfl);
    if (STAGE == 1 && ctl_tile && tid == 0) {
        a.ctl->dt = dt;
        if (a.dt_log) *a.dt_log = dt;
        a.ctl->total_time = a.ctl->total_time + dt;
        a.ctl->amax[a.parity ^ 1] = 0ull;
        a.ctl->first_nan[a.parity ^ 1] = 0;
        a.ctl->crashed = 0;
    }

    // Every thread waits (bounded) for the staged tile; the CTA gives up as a
    // whole if any wait expired, after one more bounded wait for the copy in
    // flight, and reports it in the control block.
    const bool staged = mbar_wait_bounded(bar, phase);
    if (__syncthreads_or(!staged)) {
        if (tid == 0) {
            atomicExch(&a.ctl->error, (int)KERR_TMA_TIMEOUT);
            mbar_wait_bounded(bar, phase);
        }
        return false;
    }

    const double gm = g.gamma, EPS = g.eps;
#if RMHD_FAST_MATH
    const Real gmR = (Real)gm, EPSR = (Real)EPS, inv_gm1 = (Real)(1.0 / (gm - 1.0));
#else
    const Real EPSR = EPS;
    // reciprocals of the constant divisors, for the shared-reciprocal
    // division of the exact arithmetic (MdDiv), and whether they qualify
    MdDiv cdiv;
    const double ygm1 = cdiv.recip(gm - 1.0);
    const bool gm1_ok = cdiv.ok;
    const double y2dx = cdiv.recip(2.0 * g.dx), y2dy = cdiv.recip(2.0 * g.dy);
    const bool d2_ok = cdiv.ok;
#endif

    // ---- primitives on (TI+4) x (TJ+4) cells ----
    // calculate_half_Q.cu:4-38 on the centred state (shift kernels,
    // resistiveMHD_2D.cu:313-337), once for the x sweep and once for the
    // permuted y sweep (hlld.cu:134-152), whose pressure sums in another order.
    for (int c = tid; c < PF; c += T::THREADS) {
        const int pi = c / PJ_, pj = c - pi * PJ_;
        const double *u0 = Ut + (pi + 1) * UJ + (pj + 1);
        const double rho = u0[RHO * UF];
#if RMHD_FAST_MATH
        const double irho = rcp_nr(rho);
        const double u = u0[MX * UF] * irho;
        const double v = u0[MY * UF] * irho;
        const double w = u0[MZ * UF] * irho;
#else
        MdDiv md;
        const double yr = md.recip(rho);
        double u = md.div(u0[MX * UF], rho, yr);
        double v = md.div(u0[MY * UF], rho, yr);
        double w = md.div(u0[MZ * UF], rho, yr);
        if (!md.ok) {
            u = u0[MX * UF] / rho;
            v = u0[MY * UF] / rho;
            w = u0[MZ * UF] / rho;
        }
#endif
        const double bXc = 0.5 * (u0[BXF * UF] + u0[BXF * UF - UJ]);
        const double bYc = 0.5 * (u0[BYF * UF] + u0[BYF * UF - 1]);
        const double bZ = u0[BZF * UF];
        const double e = u0[EN * UF];
        const double px = (gm - 1.0) * (e - 0.5 * (rho * (u * u + v * v + w * w))
                        - 0.5 * (bXc * bXc + bYc * bYc + bZ * bZ));
        // The y sweep's pressure sums its squares in the permuted order; the
        // contracted variants, which differ from the reference by rounding
        // anyway, take the x sweep's.
        const double py = RMHD_FAST_MATH ? px
                        : (gm - 1.0) * (e - 0.5 * (rho * (v * v + w * w + u * u))
                          - 0.5 * (bYc * bYc + bZ * bZ + bXc * bXc));
        // primitives are recovered in FP64; the velocities and the density
        // are stored in the flux-side type, B and pressures in FP64
        Real *v0 = Pv + c;
        v0[V_U * PF] = (Real)u;
        v0[V_V * PF] = (Real)v;
        v0[V_W * PF] = (Real)w;
        v0[V_RHO * PF] = (Real)rho;
        double *b0 = Pb + c;
        b0[B_XC * PF] = bXc;
        b0[B_YC * PF] = bYc;
        b0[B_PX * PF] = px;
        b0[B_PY * PF] = py;
        b0[B_Z * PF] = bZ;
    }
    __syncthreads();

    // ---- eta*J on (TI+2) x (TJ+2) cells (driver hook,
    // examples2D/plasmoid/main_plasmoid.cu:175-274) ----
    {
        const double two_dx = 2.0 * g.dx, two_dy = 2.0 * g.dy;
#if RMHD_FAST_MATH
        const Real i2dx = (Real)(1.0 / two_dx), i2dy = (Real)(1.0 / two_dy);
#endif
        for (int c = tid; c < RF; c += T::THREADS) {
            const int ri = c / RJ_, rj = c - ri * RJ_;
            const double *p0 = Pb + (ri + 1) * PJ_ + (rj + 1);
            const double *z0 = p0 + B_Z * PF;
#if RMHD_FAST_MATH
            const Real jY = -(Real)(z0[PJ_] - z0[-PJ_]) * i2dx;
            const Real jX = (Real)(z0[1] - z0[-1]) * i2dy;
            const Real jZ = (Real)(p0[B_YC * PF + PJ_] - p0[B_YC * PF - PJ_]) * i2dx
                          - (Real)(p0[B_XC * PF + 1] - p0[B_XC * PF - 1]) * i2dy;
#else
            const double nY = -(z0[PJ_] - z0[-PJ_]), nX = z0[1] - z0[-1];
            const double nZx = p0[B_YC * PF + PJ_] - p0[B_YC * PF - PJ_];
            const double nZy = p0[B_XC * PF + 1] - p0[B_XC * PF - 1];
            MdDiv md;
            md.ok = d2_ok;
            double jY = md.div(nY, two_dx, y2dx);
            double jX = md.div(nX, two_dy, y2dy);
            double jZ = md.div(nZx, two_dx, y2dx) - md.div(nZy, two_dy, y2dy);
            if (!md.ok) {
                jY = nY / two_dx;
                jX = nX / two_dy;
                jZ = nZx / two_dx - nZy / two_dy;
            }
#endif
            const Real eta = (Real)(has_eta ? Et[(ri + 2) * UJ + (rj + 2)] : g.eta);
            Real *r0 = Rs + c;
            r0[R_JX * RF] = eta * jX;
            r0[R_JY * RF] = eta * jY;
            r0[R_JZ * RF] = eta * jZ;
        }
    }
    __syncthreads();

    // ---- HLLD fluxes (hlld.cu:110-233, muscl.cu:6-126, flux_solver.cu:10-33)
    // with the resistive terms ----
    // One interface per call.  Stage 2 of the contracted variants and both
    // stages of FP32-bulk pass the sweep as a compile-time tag (a copy of the
    // body per sweep, with constant plane strides); FP64-fast's stage 1 and
    // the exact variant, which measured slower with two copies (8 % and
    // 10-25 % at 256-thread tiles), pass it at run time.  Both sweeps share
    // one index space, so the threads stay balanced.
    // `full` (a FullC tag) selects the rare path for an interface whose
    // common-case flux declined (hlld_flux_sel, hlld_flux_fast_sel or
    // hlld_flux_bulk_sel returned false; flux_at then stores nothing and
    // returns false): every case of the fast or FP32-bulk flux, or in the
    // exact variant the reference's arithmetic in full (hlld_flux_ieee).
    auto flux_at = [&](const int it, const auto sweep, const auto full) -> bool {
        (void)full;
        const bool isF = sweep.value;
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
        const Real *vc = Pv + (ci + 2) * PJ_ + (cj + 2);
        const double *bc = Pb + (ci + 2) * PJ_ + (cj + 2);
        const Real *r0 = Rs + (ci + 1) * RJ_ + (cj + 1);
        const int ps = isF ? PJ_ : 1;
        // sweep frame: the y sweep runs the x-sweep arithmetic on
        // (rho, v, w, u, bY, bZ, bX, e) (hlld.cu:134-152)
        const int pu = isF ? V_U : V_V, pv = isF ? V_V : V_W, pw = isF ? V_W : V_U;
        const double *pp = bc + (isF ? B_PX : B_PY) * PF;
        const double *bt1 = bc + (isF ? B_YC : B_Z) * PF;   // tangential B 1
        const double *bt2 = bc + (isF ? B_Z : B_XC) * PF;   // tangential B 2
        const double *nb = bc + (isF ? B_XC : B_YC) * PF;
        const double bn = 0.5 * (nb[0] + nb[ps]);
        double fmv[3];   // momentum fluxes (rhoU, rhoV, rhoW in the sweep frame)
        Real fov[4];     // mass, bZ-frame tangential-2 induction, energy, tangential-1 induction
#if RMHD_BULK
        {
            const float EPSF = (float)EPS;
            BulkStates st;
            {
                // density: MUSCL in single precision from the staged copy
                const Real *q = vc + V_RHO * PF;
                const float qm = q[-ps], q0 = q[0], qp = q[ps], qpp = q[2 * ps];
                st.rhoL = q0 + 0.5f * minmod(q0 - qm, qp - q0, EPSF);
                st.rhoR = qp - 0.5f * minmod(qp - q0, qpp - qp, EPSF);
            }
            {
                const Real *q = vc + pu * PF;
                const float qm = q[-ps], q0 = q[0], qp = q[ps], qpp = q[2 * ps];
                st.uL = q0 + 0.5f * minmod(q0 - qm, qp - q0, EPSF);
                st.uR = qp - 0.5f * minmod(qp - q0, qpp - qp, EPSF);
            }
            {
                const Real *q = vc + pv * PF;
                const float qm = q[-ps], q0 = q[0], qp = q[ps], qpp = q[2 * ps];
                st.vL = q0 + 0.5f * minmod(q0 - qm, qp - q0, EPSF);
                st.vR = qp - 0.5f * minmod(qp - q0, qpp - qp, EPSF);
            }
            {
                const Real *q = vc + pw * PF;
                const float qm = q[-ps], q0 = q[0], qp = q[ps], qpp = q[2 * ps];
                st.wL = q0 + 0.5f * minmod(q0 - qm, qp - q0, EPSF);
                st.wR = qp - 0.5f * minmod(qp - q0, qpp - qp, EPSF);
            }
            muscl_dev(pp[-ps], pp[0], pp[ps], pp[2 * ps], EPSF, st.pL, st.pR);
            muscl_dev(bt1[-ps], bt1[0], bt1[ps], bt1[2 * ps], EPSF, st.bYL, st.bYR);
            muscl_dev(bt2[-ps], bt2[0], bt2[ps], bt2[2 * ps], EPSF, st.bZL, st.bZR);
            st.bn = bn;
            float fo4[4];
            if (full.value)
                hlld_flux_bulk(st, gmR, inv_gm1, EPSF, fmv, fo4);
            else if (!hlld_flux_bulk_sel(st, gmR, inv_gm1, EPSF, fmv, fo4))
                return false;
            // fo4: f0, f5 (tangential-1 induction), f6 (tangential-2), f7
            fov[0] = fo4[0]; fov[1] = fo4[2]; fov[2] = fo4[3]; fov[3] = fo4[1];
        }
#else
        {
            Real qL[7], qR[7];
            auto rec = [&](const Real qm, const Real q0, const Real qp, const Real qpp, Real &l, Real &r) {
                l = q0 + Real(0.5) * minmod(q0 - qm, qp - q0, EPSR);
                r = qp - Real(0.5) * minmod(qp - q0, qpp - qp, EPSR);
            };
            {
                const Real *q = vc + V_RHO * PF;
                rec(q[-ps], q[0], q[ps], q[2 * ps], qL[0], qR[0]);
            }
            {
                const Real *q = vc + pu * PF;
                rec(q[-ps], q[0], q[ps], q[2 * ps], qL[1], qR[1]);
            }
            {
                const Real *q = vc + pv * PF;
                rec(q[-ps], q[0], q[ps], q[2 * ps], qL[2], qR[2]);
            }
            {
                const Real *q = vc + pw * PF;
                rec(q[-ps], q[0], q[ps], q[2 * ps], qL[3], qR[3]);
            }
            rec((Real)bt1[-ps], (Real)bt1[0], (Real)bt1[ps], (Real)bt1[2 * ps], qL[4], qR[4]);
            rec((Real)bt2[-ps], (Real)bt2[0], (Real)bt2[ps], (Real)bt2[2 * ps], qL[5], qR[5]);
            rec((Real)pp[-ps], (Real)pp[0], (Real)pp[ps], (Real)pp[2 * ps], qL[6], qR[6]);
            const PrimT<Real> L{qL[0], qL[1], qL[2], qL[3], (Real)bn, qL[4], qL[5], qL[6]};
            const PrimT<Real> R{qR[0], qR[1], qR[2], qR[3], (Real)bn, qR[4], qR[5], qR[6]};
            Real f[8];
#if RMHD_FAST_MATH
            if (full.value)
                hlld_flux_fast(L, R, gmR, inv_gm1, EPSR, f);
            else if (!hlld_flux_fast_sel(L, R, gmR, inv_gm1, EPSR, f))
                return false;
#else
            if (full.value)
                hlld_flux_ieee(L, R, gm, EPS, f);
            else if (!hlld_flux_sel(L, R, gm, EPS, ygm1, gm1_ok, f))
                return false;
#endif
            fmv[0] = f[1]; fmv[1] = f[2]; fmv[2] = f[3];
            fov[0] = f[0]; fov[1] = f[6]; fov[2] = f[7]; fov[3] = f[5];
        }
#endif
        // eta*J of the two cells sharing the interface and their B
        const int rs = isF ? RJ_ : 1;
        const Real z0 = (Real)bc[B_Z * PF], z1 = (Real)bc[B_Z * PF + ps];
        const Real h = Real(0.5);
        if (isF) {
            const Real eY0 = r0[R_JY * RF], eY1 = r0[R_JY * RF + rs];
            const Real eZ0 = r0[R_JZ * RF], eZ1 = r0[R_JZ * RF + rs];
            const Real y0 = (Real)bc[B_YC * PF], y1 = (Real)bc[B_YC * PF + ps];
            double *om = Fm + a0 * F_NJ + a1;
            Real *oo = Fo + a0 * F_NJ + a1;
            om[0 * SF] = fmv[0]; om[1 * SF] = fmv[1]; om[2 * SF] = fmv[2];
            oo[O_RHO * SF] = fov[0];
            oo[O_BZ * SF] = fov[1] + h * (eY0 + eY1);
            oo[O_EN * SF] = fov[2] + (h * (eY0 * z0 + eY1 * z1) - h * (eZ0 * y0 + eZ1 * y1));
            if (STAGE == 1) oo[O_EMF * SF] = fov[3] - h * (eZ0 + eZ1);
        } else {
            const Real eX0 = r0[R_JX * RF], eX1 = r0[R_JX * RF + rs];
            const Real eZ0 = r0[R_JZ * RF], eZ1 = r0[R_JZ * RF + rs];
            const Real x0 = (Real)bc[B_XC * PF], x1 = (Real)bc[B_XC * PF + ps];
            // un-permute (hlld.cu:170-194): g1 = f3, g2 = f1, g3 = f2,
            // g4 = f6, g5 = f4 = 0, g6 = f5.
            double *om = Gm + a0 * G_NJ + a1;
            Real *oo = Go + a0 * G_NJ + a1;
            om[0 * SG] = fmv[2]; om[1 * SG] = fmv[0]; om[2 * SG] = fmv[1];
            oo[O_RHO * SG] = fov[0];
            oo[O_BZ * SG] = fov[3] - h * (eX0 + eX1);
            oo[O_EN * SG] = fov[2] + (h * (eZ0 * x0 + eZ1 * x1) - h * (eX0 * z0 + eX1 * z1));
            if (STAGE == 1) oo[O_EMF * SG] = fov[1] + h * (eZ0 + eZ1);
        }
        return true;
    };
    // bit r of `redo`: this thread's interface of pass r asked for the full path
    unsigned redo = 0u;
    static_assert((T::NF + T::NG + T::THREADS - 1) / T::THREADS <= 32, "passes of the flux phase");
    for (int it = tid, r = 0; it < T::NF + T::NG; it += T::THREADS, ++r) {
        bool done;
        if ((STAGE == 1 && !RMHD_BULK) || !RMHD_FAST_MATH)
            done = flux_at(it, SweepRT{it < T::NF}, FullC<false>{});
        else if (it < T::NF)
            done = flux_at(it, SweepC<true>{}, FullC<false>{});
        else
            done = flux_at(it, SweepC<false>{}, FullC<false>{});
        redo |= done ? 0u : 1u << r;
    }
    // The rare path, after the loop, so that its registers do not weigh on
    // the loop's.
    if (redo) {
        for (int it = tid, r = 0; it < T::NF + T::NG; it += T::THREADS, ++r)
            if ((redo >> r) & 1u) flux_at(it, SweepRT{it < T::NF}, FullC<true>{});
    }
    // The update's own cell of the stage's source state (from global memory
    // when the flux planes overlay the staged tile), and in stage 2 that of
    // U^n: issue those loads here, so that their latency overlaps the
    // barrier wait of the CTA's slower warps.
    double uo[NFIELD], un_h[6];
    if (own) {
#pragma unroll
        for (int f = 0; f < NFIELD; ++f)
            uo[f] = T::OVERLAY ? a.src[f * PL + k] : Ut[f * UF + (li + HALO) * UJ + (lj + HALO)];
        if (STAGE == 2) {
#pragma unroll
            for (int n = 0; n < 6; ++n) {
                const int f = n == 0 ? RHO : n == 1 ? MX : n == 2 ? MY : n == 3 ? MZ : n == 4 ? BZF : EN;
                un_h[n] = a.un[f * PL + k];
            }
        }
    }
    __syncthreads();

    const double dtdx = dt / g.dx, dtdy = dt / g.dy;

    // ---- corner EMF (ct.cu:22-41) at corner (i, j) = (i0-1+ei, j0-1+ej),
    // i.e. Fs (fi, fj) = (ei, ej) and Gs (gi, gj) = (ei, ej); formed by each
    // update cell for the corners it reads (no phase and barrier of its own) ----
    auto corner_ez = [&](const int ei, const int ej) -> double {
        // accumulated in FP64 whatever the flux-side type
        const double eZG1 = (double)Go[O_EMF * SG + ei * G_NJ + ej];
        const double eZG2 = (double)Go[O_EMF * SG + (ei + 1) * G_NJ + ej];
        const double eZF1 = -1.0 * (double)Fo[O_EMF * SF + ei * F_NJ + ej];
        const double eZF2 = -1.0 * (double)Fo[O_EMF * SF + ei * F_NJ + ej + 1];
        return 0.25 * (eZG1 + eZG2 + eZF1 + eZF2);
    };

    // ---- update of the tile's own cells ----
    const int fo_ = (li + 1) * F_NJ + (lj - T::F_J0);             // F(i); F(i-1) is F_NJ before
    const int go_ = (li - T::G_I0) * G_NJ + (lj + 1);             // G(j); G(j-1) is 1 before
    const int fld[6] = {RHO, MX, MY, MZ, BZF, EN};
    // flux difference of hydro field n (0..5), in FP64
    auto dF = [&](int n) -> double {
        if (n >= 1 && n <= 3) return Fm[(n - 1) * SF + fo_] - Fm[(n - 1) * SF + fo_ - F_NJ];
        const int o = n == 0 ? O_RHO : (n == 4 ? O_BZ : O_EN);
        return (double)Fo[o * SF + fo_] - (double)Fo[o * SF + fo_ - F_NJ];
    };
    auto dG = [&](int n) -> double {
        if (n >= 1 && n <= 3) return Gm[(n - 1) * SG + go_] - Gm[(n - 1) * SG + go_ - 1];
        const int o = n == 0 ? O_RHO : (n == 4 ? O_BZ : O_EN);
        return (double)Go[o * SG + go_] - (double)Go[o * SG + go_ - 1];
    };

    if (STAGE == 1) {
        if (own) {
            // oneStepFirstFunctor (resistiveMHD_2D.cu:53-86)
#pragma unroll
            for (int n = 0; n < 6; ++n)
                a.dst[fld[n] * PL + k] = uo[fld[n]] - dtdx * dF(n) - dtdy * dG(n);
            // CT_kernel (ct.cu:44-59) with the EMF of this stage
            const double ez_c = corner_ez(li + 1, lj + 1), ez_w = corner_ez(li + 1, lj);
            const double ez_s = corner_ez(li, lj + 1);
            a.dst[BXF * PL + k] = uo[BXF] - dtdy * (ez_c - ez_w);
            a.dst[BYF * PL + k] = uo[BYF] + dtdx * (ez_c - ez_s);
            // Symmetric boundaries read the CT'd face bY at j = 2 (the lower
            // wall face) before replacing it (TS boundary.cu:57-88).
            if (a.row2 && j0 == HALO && lj == 0) {
                const double b2 = T::OVERLAY ? a.src[BYF * PL + k - 1]
                                               : Ut[BYF * UF + (li + HALO) * UJ + (lj + HALO) - 1];
                a.row2[i] = b2 + dtdx * (ez_w - corner_ez(li, lj));
            }
        }
    } else {
        // oneStepSecondFunctor (resistiveMHD_2D.cu:88-130); the face B of
        // the new state equals the stage-1 CT result, which is copied.
        double nv[8];
        if (own) {
#pragma unroll
            for (int n = 0; n < 6; ++n) {
                const double u = un_h[n];
                const double ub = uo[fld[n]];
                nv[fld[n]] = 0.5 * (u + ub - dtdx * dF(n) - dtdy * dG(n));
            }
            nv[BXF] = uo[BXF];
            nv[BYF] = uo[BYF];
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
            MdDiv dd;
            const double ydx = dd.recip(g.dx), ydy = dd.recip(g.dy);
            const double r = cfl_rate_md(nv[RHO], nv[MX], nv[MY], nv[MZ], nv[BXF], nv[BYF], nv[BZF], nv[EN],
                                         gm, g.dx, g.dy, ydx, ydy, dd.ok);
#endif
            bits = rate_bits(r);
            nan_e = nv[EN] != nv[EN];
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            const unsigned long long o = __shfl_xor_sync(0xffffffffu, bits, off);
            bits = o > bits ? o : bits;
        }
        // Pb is dead after the flux phase: reuse it for the per-warp maxima.
        unsigned long long *wmax = reinterpret_cast<unsigned long long *>(Pb);
        if ((tid & 31) == 0) wmax[tid >> 5] = bits;
        const int any_nan = __syncthreads_or(nan_e);
        if (tid == 0) {
            unsigned long long m = 0ull;
            for (int w = 0; w < T::THREADS / 32; ++w) m = wmax[w] > m ? wmax[w] : m;
            atomicMax(&a.ctl->amax[a.parity ^ 1], m);
            if (any_nan) atomicExch(&a.ctl->crashed, 1);
        }
    }
    return true;
}

__device__ __forceinline__ void init_tile_barrier(uint64_t *bar)
{
    if (threadIdx.x == 0) mbar_init_tile(bar);
    __syncthreads();
}

// One CTA per tile of one run.
template <int STAGE, int SHAPE>
__global__ void __launch_bounds__(variant_threads(STAGE, SHAPE), shape_max_ctas(SHAPE))
stage_kernel(const __grid_constant__ CUtensorMap tmap, const __grid_constant__ CUtensorMap emap,
             const StageArgs a)
{
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    using T = Tile<STAGE, SHAPE>;
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem_raw + T::OFF_BAR);
    init_tile_barrier(bar);
    const TileLoad load{&tmap, &emap, (int)blockIdx.y, (int)blockIdx.x, a.eta != nullptr};
    stage_tile<STAGE, SHAPE>(a, load, blockIdx.x == 0 && blockIdx.y == 0, smem_raw, bar, 0);
}

// The stage arguments of one run of a batch.
template <int STAGE>
__device__ __forceinline__ StageArgs batch_args(const BatchRun &r, int parity)
{
    StageArgs a{};
    a.g = r.g;
    a.src = STAGE == 1 ? r.A : r.B;
    a.un = r.A;
    a.dst = STAGE == 1 ? r.B : r.A;
    a.eta = r.eta;
    a.row2 = r.g.bc_x == BC_SYMMETRIC ? r.row2 : nullptr;
    a.ctl = r.ctl;
    a.parity = parity;
    return a;
}

// Persistent CTAs over the tile table of a batch of independent runs (each
// with its own grid, eta, state buffers, tensor maps and control block).
template <int STAGE, int SHAPE>
__global__ void __launch_bounds__(variant_threads(STAGE, SHAPE), shape_max_ctas(SHAPE))
stage_batch_kernel(const BatchRun *runs, const CUtensorMap *maps, const TileRef *tiles, int ntiles, int parity)
{
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    using T = Tile<STAGE, SHAPE>;
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem_raw + T::OFF_BAR);
    init_tile_barrier(bar);
    uint32_t phase = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const TileRef tr = tiles[t];
        const BatchRun &r = runs[tr.run];
        const CUtensorMap *m = maps + (size_t)tr.run * MAPS_PER_RUN;
        const TileLoad load{m + (STAGE - 1), m + 2 + (STAGE - 1), tr.ti, tr.tj, r.eta != nullptr};
        if (!stage_tile<STAGE, SHAPE>(batch_args<STAGE>(r, parity), load, tr.ti == 0 && tr.tj == 0, smem_raw, bar,
                                      phase))
            return;
        phase ^= 1;
        // every thread is done with this tile's shared memory, whose flux
        // planes the next tile's staging overwrites through the async proxy
        fence_proxy_async();
        __syncthreads();
    }
}

template <int STAGE, int SHAPE> constexpr size_t smem_of() { return Tile<STAGE, SHAPE>::SMEM_BYTES; }

// Calls f.template operator()<STAGE, SHAPE>() for the run-time stage and shape.
template <class F> static void with_stage_shape(int stage, int shape, const F &f)
{
#define RMHD_SHAPE_CASE(SH)                                                                            \
    case SH:                                                                                           \
        if (stage == 1) f.template operator()<1, SH>();                                                \
        else f.template operator()<2, SH>();                                                           \
        break;
    switch (shape) {
    RMHD_SHAPE_CASE(0)
    RMHD_SHAPE_CASE(1)
    RMHD_SHAPE_CASE(2)
    RMHD_SHAPE_CASE(3)
    RMHD_SHAPE_CASE(4)
    default: RMHD_SHAPE_CASE(5)
    }
#undef RMHD_SHAPE_CASE
}
static_assert(NSHAPE == 6, "one case per tile shape in with_stage_shape");

struct SmemOf {
    size_t &n;
    template <int ST, int SH> void operator()() const { n = smem_of<ST, SH>(); }
};

size_t stage_smem_bytes(int stage, int shape)
{
    size_t n = 0;
    with_stage_shape(stage, shape, SmemOf{n});
    return n;
}

struct RegsOf {
    cudaFuncAttributes &attr;
    template <int ST, int SH> void operator()() const
    {
        cudaFuncGetAttributes(&attr, (const void *)stage_kernel<ST, SH>);
    }
};

int stage_regs(int stage, int shape)
{
    cudaFuncAttributes attr{};
    with_stage_shape(stage, shape, RegsOf{attr});
    return attr.numRegs;
}

// Opts a stage kernel into its dynamic shared memory and asks for the
// smallest shared-memory carve-out that holds `ctas` of its CTAs per SM,
// leaving the rest of the SM's unified L1 to the cache.
template <class K> static void set_smem_attributes(K kernel, size_t smem, int ctas)
{
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const size_t need = (size_t)ctas * (smem + 1024), most = 228 * 1024;
    const int pct = (int)((need * 100 + most - 1) / most);
    cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, pct > 100 ? 100 : pct);
}

// The launchers pass the kernels local copies of their arguments, which a
// launch captures by value.
struct LaunchOne {
    const CUtensorMap *tmap, *emap;
    const StageArgs &args;
    cudaStream_t stream;
    template <int ST, int SH> void operator()() const
    {
        using T = Tile<ST, SH>;
        set_smem_attributes(stage_kernel<ST, SH>, T::SMEM_BYTES, T::CTAS);
        const CUtensorMap tm = *tmap, em = *emap;
        const StageArgs a = args;
        const dim3 grid((a.g.ny - 2 * HALO + T::TJ - 1) / T::TJ, (a.g.nx - 2 * HALO + T::TI - 1) / T::TI);
        stage_kernel<ST, SH><<<grid, T::THREADS, T::SMEM_BYTES, stream>>>(tm, em, a);
    }
};

void launch_stage(int stage, int shape, const CUtensorMap *tmap, const CUtensorMap *emap, const StageArgs &args,
                  cudaStream_t stream)
{
    with_stage_shape(stage, shape, LaunchOne{tmap, emap, args, stream});
}

struct LaunchBatch {
    const BatchRun *runs;
    const CUtensorMap *maps;
    const TileRef *tiles;
    int ntiles, ctas, parity;
    cudaStream_t stream;
    template <int ST, int SH> void operator()() const
    {
        using T = Tile<ST, SH>;
        set_smem_attributes(stage_batch_kernel<ST, SH>, T::SMEM_BYTES, T::CTAS);
        const BatchRun *r = runs;
        const CUtensorMap *m = maps;
        const TileRef *t = tiles;
        const int n = ntiles, c = ctas, par = parity;
        stage_batch_kernel<ST, SH><<<c, T::THREADS, T::SMEM_BYTES, stream>>>(r, m, t, n, par);
    }
};

void launch_stage_batch(int stage, int shape, const BatchRun *runs, const CUtensorMap *maps, const TileRef *tiles,
                        int ntiles, int ctas, int parity, cudaStream_t stream)
{
    with_stage_shape(stage, shape, LaunchBatch{runs, maps, tiles, ntiles, ctas, parity, stream});
}

}  // namespace RMHD_VARIANT
}  // namespace rmhd2d
