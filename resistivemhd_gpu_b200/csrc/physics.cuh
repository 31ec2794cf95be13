// physics.cuh -- per-cell and per-interface arithmetic of the 2D resistive-MHD
// step, written for the fused sm_100a stage kernel.  Every expression keeps
// the operation order of the reference's functors so that, compiled without
// FMA contraction (-fmad=false), results are bit-identical to the reference
// evaluated in IEEE binary64 (reference files under
// ResistiveMHD_singleGPU_thrust/lib_ResistiveMHD_2D_GPU_periodicXY/).
#pragma once

#include <cuda_runtime.h>

#include <cstring>

namespace rmhd2d {

__host__ __device__ __forceinline__ double bits_to_double(unsigned long long b)
{
#ifdef __CUDA_ARCH__
    return __longlong_as_double((long long)b);
#else
    double d;
    memcpy(&d, &b, sizeof(d));
    return d;
#endif
}

// thrust::min / thrust::max semantics ((b < a) ? b : a).
__device__ __forceinline__ double tmin(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double tmax(double a, double b) { return (a < b) ? b : a; }

// hlld.cu:26-32 Sign, (x > 0) - (x < 0), as selects (no int conversion).
__device__ __forceinline__ double sgn(double x) { return x > 0.0 ? 1.0 : (x < 0.0 ? -1.0 : 0.0); }

// minmod.hpp:6-16: sign_x * max(min(|x|, sign_x * y), EPS) with an int
// sign_x.  Written with selects: for x > 0 the reference computes
// 1.0 * max(min(|x|, 1.0 * y), EPS), for x < 0 the negation of
// max(min(|x|, -y), EPS), for x == 0 (or NaN) 0.0 * max(min(|x|, 0.0 * y), EPS);
// multiplying by +-1 is exact, so this is bit-identical for every input.
__device__ __forceinline__ double minmod(double x, double y, double eps)
{
    const double ax = fabs(x);
    if (x > 0.0) return tmax(tmin(ax, y), eps);
    if (x < 0.0) return -tmax(tmin(ax, -y), eps);
    return 0.0 * tmax(tmin(ax, 0.0 * y), eps);
}

// Reciprocal by Newton-Raphson iteration on 1/a (x' = x + x (1 - a x), two
// steps, each squaring the relative error) from the hardware seed
// rcp.approx.ftz.f64; used by the fast variant only.  Accurate to about one
// ulp for normal finite a; a = 0 or +-inf give NaN (the fast variant's
// denominators carry the reference's +EPS and are never 0 in a finite state).
__device__ __forceinline__ double rcp_nr(double a)
{
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(a));
    double e = fma(-a, r, 1.0);
    r = fma(r, e, r);
    e = fma(-a, r, 1.0);
    r = fma(r, e, r);
    return r;
}

// Interface state fed to HLLD: BasicParameter (basic_parameter_struct.hpp:5-27).
struct Prim {
    double rho, u, v, w, bX, bY, bZ, p;
};

// hlld.cu:448-467 getOneFlux, accumulated into f (f4 is identically 0 and
// is not produced).
__device__ __forceinline__ void add_one_flux(double rho, double u, double v, double w, double bX,
                                             double bY, double bZ, double e, double pT, double f[8])
{
    f[0] += rho * u;
    f[1] += rho * u * u + pT - bX * bX;
    f[2] += rho * u * v - bX * bY;
    f[3] += rho * u * w - bX * bZ;
    f[5] += u * bY - v * bX;
    f[6] += u * bZ - w * bX;
    f[7] += (e + pT) * u - bX * (bX * u + bY * v + bZ * w);
}

// Weighted candidate: f += F(state) * ind (all six candidates are formed,
// so non-finite values propagate exactly as in the reference's
// CalculateFluxFunctor, hlld.cu:35-107).
__device__ __forceinline__ void add_weighted_flux(double rho, double u, double v, double w, double bX,
                                                  double bY, double bZ, double e, double pT,
                                                  double ind, double f[8])
{
    f[0] += (rho * u) * ind;
    f[1] += (rho * u * u + pT - bX * bX) * ind;
    f[2] += (rho * u * v - bX * bY) * ind;
    f[3] += (rho * u * w - bX * bZ) * ind;
    f[4] += 0.0 * ind;
    f[5] += (u * bY - v * bX) * ind;
    f[6] += (u * bZ - w * bX) * ind;
    f[7] += ((e + pT) * u - bX * (bX * u + bY * v + bZ * w)) * ind;
}

// HLLD flux through one interface: hlld.cu:256-432
// (calculateHLLDParameterFunctor), hlld.cu:469-549 (setFluxFunctor) and
// hlld.cu:35-107 (CalculateFluxFunctor).
//
// ALL_CANDIDATES = true forms all six candidate fluxes and sums them with the
// reference's 0/1 indicator weights (bit-identical to the reference for every
// input, including non-finite ones).  ALL_CANDIDATES = false forms only the
// candidates whose indicator is 1 and adds them in the reference's order,
// which gives the same bits whenever all six candidates are finite.
template <bool ALL_CANDIDATES>
__device__ __forceinline__ void hlld_flux(const Prim &L, const Prim &R, double gm, double EPS,
                                          double f[8])
{
    const double rhoL = L.rho, uL = L.u, vL = L.v, wL = L.w, bXL = L.bX, bYL = L.bY, bZL = L.bZ, pL = L.p;
    const double rhoR = R.rho, uR = R.u, vR = R.v, wR = R.w, bXR = R.bX, bYR = R.bY, bZR = R.bZ, pR = R.p;

    const double eL = pL / (gm - 1.0)
                    + 0.5 * rhoL * (uL * uL + vL * vL + wL * wL)
                    + 0.5 * (bXL * bXL + bYL * bYL + bZL * bZL);
    const double pTL = pL + 0.5 * (bXL * bXL + bYL * bYL + bZL * bZL);
    const double eR = pR / (gm - 1.0)
                    + 0.5 * rhoR * (uR * uR + vR * vR + wR * wR)
                    + 0.5 * (bXR * bXR + bYR * bYR + bZR * bZR);
    const double pTR = pR + 0.5 * (bXR * bXR + bYR * bYR + bZR * bZR);

    const double csL = sqrt(gm * pL / rhoL);
    const double caL = sqrt((bXL * bXL + bYL * bYL + bZL * bZL) / rhoL);
    const double vaL = sqrt(bXL * bXL / rhoL);
    const double cfL = sqrt(0.5 * (csL * csL + caL * caL
                     + sqrt((csL * csL + caL * caL) * (csL * csL + caL * caL)
                     - 4.0 * csL * csL * vaL * vaL)));
    const double csR = sqrt(gm * pR / rhoR);
    const double caR = sqrt((bXR * bXR + bYR * bYR + bZR * bZR) / rhoR);
    const double vaR = sqrt(bXR * bXR / rhoR);
    const double cfR = sqrt(0.5 * (csR * csR + caR * caR
                     + sqrt((csR * csR + caR * caR) * (csR * csR + caR * caR)
                     - 4.0 * csR * csR * vaR * vaR)));

    double SL = tmin(uL, uR) - tmax(cfL, cfR);
    double SR = tmax(uL, uR) + tmax(cfL, cfR);
    SL = tmin(SL, 0.0);
    SR = tmax(SR, 0.0);

    const double SM = ((SR - uR) * rhoR * uR - (SL - uL) * rhoL * uL - pTR + pTL)
                    / ((SR - uR) * rhoR - (SL - uL) * rhoL + EPS);
    const double pT1 = ((SR - uR) * rhoR * pTL - (SL - uL) * rhoL * pTR
                     + rhoL * rhoR * (SR - uR) * (SL - uL) * (uR - uL))
                     / ((SR - uR) * rhoR - (SL - uL) * rhoL + EPS);

    const double rho1L = rhoL * (SL - uL) / (SL - SM + EPS);
    const double u1L = SM;
    const double v1L = vL - bXL * bYL * (SM - uL) / (rhoL * (SL - uL) * (SL - SM) - bXL * bXL + EPS);
    const double w1L = wL - bXL * bZL * (SM - uL) / (rhoL * (SL - uL) * (SL - SM) - bXL * bXL + EPS);
    const double bX1L = bXL;
    const double bY1L = bYL * (rhoL * (SL - uL) * (SL - uL) - bXL * bXL)
                      / (rhoL * (SL - uL) * (SL - SM) - bXL * bXL + EPS);
    const double bZ1L = bZL * (rhoL * (SL - uL) * (SL - uL) - bXL * bXL)
                      / (rhoL * (SL - uL) * (SL - SM) - bXL * bXL + EPS);
    const double e1L = ((SL - uL) * eL - pTL * uL + pT1 * SM
                     + bXL * ((uL * bXL + vL * bYL + wL * bZL) - (u1L * bX1L + v1L * bY1L + w1L * bZ1L)))
                     / (SL - SM + EPS);

    const double rho1R = rhoR * (SR - uR) / (SR - SM + EPS);
    const double u1R = SM;
    const double v1R = vR - bXR * bYR * (SM - uR) / (rhoR * (SR - uR) * (SR - SM) - bXR * bXR + EPS);
    const double w1R = wR - bXR * bZR * (SM - uR) / (rhoR * (SR - uR) * (SR - SM) - bXR * bXR + EPS);
    const double bX1R = bXR;
    const double bY1R = bYR * (rhoR * (SR - uR) * (SR - uR) - bXR * bXR)
                      / (rhoR * (SR - uR) * (SR - SM) - bXR * bXR + EPS);
    const double bZ1R = bZR * (rhoR * (SR - uR) * (SR - uR) - bXR * bXR)
                      / (rhoR * (SR - uR) * (SR - SM) - bXR * bXR + EPS);
    const double e1R = ((SR - uR) * eR - pTR * uR + pT1 * SM
                     + bXR * ((uR * bXR + vR * bYR + wR * bZR) - (u1R * bX1R + v1R * bY1R + w1R * bZ1R)))
                     / (SR - SM + EPS);

    const double S1L = SM - sqrt(bX1L * bX1L / rho1L);
    const double S1R = SM + sqrt(bX1R * bX1R / rho1R);

    const double sqL = sqrt(rho1L), sqR = sqrt(rho1R), sqLR = sqrt(rho1L * rho1R);
    const double sbX = sgn(bX1L);
    const double u2 = SM;
    const double v2 = (sqL * v1L + sqR * v1R + (bY1R - bY1L) * sbX) / (sqL + sqR + EPS);
    const double w2 = (sqL * w1L + sqR * w1R + (bZ1R - bZ1L) * sbX) / (sqL + sqR + EPS);
    const double bY2 = (sqL * bY1R + sqR * bY1L + sqLR * (v1R - v1L) * sbX) / (sqL + sqR + EPS);
    const double bZ2 = (sqL * bZ1R + sqR * bZ1L + sqLR * (w1R - w1L) * sbX) / (sqL + sqR + EPS);
    const double e2L = e1L - sqL * ((u1L * bX1L + v1L * bY1L + w1L * bZ1L) - (u2 * bXL + v2 * bY2 + w2 * bZ2))
                     * sgn(bXL);
    const double e2R = e1R + sqR * ((u1R * bX1R + v1R * bY1R + w1R * bZ1R) - (u2 * bXR + v2 * bY2 + w2 * bZ2))
                     * sgn(bXR);

    const bool bOL = SL > 0.0;
    const bool bML = (SL <= 0.0) && (0.0 < S1L);
    const bool bIL = (S1L <= 0.0) && (0.0 < SM);
    const bool bOR = SR <= 0.0;
    const bool bMR = (S1R <= 0.0) && (0.0 < SR);
    const bool bIR = (SM <= 0.0) && (0.0 < S1R);

#pragma unroll
    for (int n = 0; n < 8; ++n) f[n] = 0.0;
    if (ALL_CANDIDATES) {
        // rho2L = rho1L, rho2R = rho1R, pT2 = pT1 (hlld.cu:360-378).
        add_weighted_flux(rhoL, uL, vL, wL, bXL, bYL, bZL, eL, pTL, (double)bOL, f);
        add_weighted_flux(rho1L, u1L, v1L, w1L, bXL, bY1L, bZ1L, e1L, pT1, (double)bML, f);
        add_weighted_flux(rho1L, u2, v2, w2, bXL, bY2, bZ2, e2L, pT1, (double)bIL, f);
        add_weighted_flux(rhoR, uR, vR, wR, bXR, bYR, bZR, eR, pTR, (double)bOR, f);
        add_weighted_flux(rho1R, u1R, v1R, w1R, bXR, bY1R, bZ1R, e1R, pT1, (double)bMR, f);
        add_weighted_flux(rho1R, u2, v2, w2, bXR, bY2, bZ2, e2R, pT1, (double)bIR, f);
    } else {
        if (bOL) add_one_flux(rhoL, uL, vL, wL, bXL, bYL, bZL, eL, pTL, f);
        if (bML) add_one_flux(rho1L, u1L, v1L, w1L, bXL, bY1L, bZ1L, e1L, pT1, f);
        if (bIL) add_one_flux(rho1L, u2, v2, w2, bXL, bY2, bZ2, e2L, pT1, f);
        if (bOR) add_one_flux(rhoR, uR, vR, wR, bXR, bYR, bZR, eR, pTR, f);
        if (bMR) add_one_flux(rho1R, u1R, v1R, w1R, bXR, bY1R, bZ1R, e1R, pT1, f);
        if (bIR) add_one_flux(rho1R, u2, v2, w2, bXR, bY2, bZ2, e2R, pT1, f);
    }
}

// HLLD flux of the fast variant: the same wave-speed estimates, star and
// double-star states and candidate selection as hlld_flux (hlld.cu:256-565),
// rearranged for the FP64 pipe.  It differs from the exact form by rounding
// only: one correctly rounded reciprocal per distinct denominator (8 instead
// of 28 divisions), squared sound/Alfven speeds used directly (the reference
// squares their square roots), sqrt(rho*) and |bX|/sqrt(rho*) from one rsqrt,
// and bX taken once (left and right states share the interface-normal B).
__device__ __forceinline__ void hlld_flux_fast(const Prim &L, const Prim &R, double gm, double inv_gm1,
                                               double EPS, double f[8])
{
    const double bX = L.bX;
    const double bx2 = bX * bX;
    const double iRL = rcp_nr(L.rho), iRR = rcp_nr(R.rho);
    const double b2L = bx2 + L.bY * L.bY + L.bZ * L.bZ;
    const double b2R = bx2 + R.bY * R.bY + R.bZ * R.bZ;
    const double eL = L.p * inv_gm1 + 0.5 * L.rho * (L.u * L.u + L.v * L.v + L.w * L.w) + 0.5 * b2L;
    const double eR = R.p * inv_gm1 + 0.5 * R.rho * (R.u * R.u + R.v * R.v + R.w * R.w) + 0.5 * b2R;
    const double pTL = L.p + 0.5 * b2L, pTR = R.p + 0.5 * b2R;

    const double cs2L = gm * L.p * iRL, ca2L = b2L * iRL, va2L = bx2 * iRL;
    const double cs2R = gm * R.p * iRR, ca2R = b2R * iRR, va2R = bx2 * iRR;
    const double sL = cs2L + ca2L, sR = cs2R + ca2R;
    // The reference takes sqrt of each squared speed, so a negative one makes
    // its fast speed NaN; keep that.
    const double qnan = bits_to_double(0x7FF8000000000000ull);
    const bool okL = (cs2L >= 0.0) & (ca2L >= 0.0) & (va2L >= 0.0);
    const bool okR = (cs2R >= 0.0) & (ca2R >= 0.0) & (va2R >= 0.0);
    const double cfL = okL ? sqrt(0.5 * (sL + sqrt(sL * sL - 4.0 * cs2L * va2L))) : qnan;
    const double cfR = okR ? sqrt(0.5 * (sR + sqrt(sR * sR - 4.0 * cs2R * va2R))) : qnan;

    const double uL = L.u, uR = R.u;
    double SL = tmin(uL, uR) - tmax(cfL, cfR);
    double SR = tmax(uL, uR) + tmax(cfL, cfR);
    SL = tmin(SL, 0.0);
    SR = tmax(SR, 0.0);

    const double dSL = SL - uL, dSR = SR - uR;
    const double rdSL = L.rho * dSL, rdSR = R.rho * dSR;
    const double iden = rcp_nr(rdSR - rdSL + EPS);
    const double SM = (rdSR * uR - rdSL * uL - pTR + pTL) * iden;
    const double pT1 = (rdSR * pTL - rdSL * pTR + rdSL * rdSR * (uR - uL)) * iden;

    const double iSLM = rcp_nr(SL - SM + EPS), iSRM = rcp_nr(SR - SM + EPS);
    const double rho1L = rdSL * iSLM, rho1R = rdSR * iSRM;
    const double id1L = rcp_nr(rdSL * (SL - SM) - bx2 + EPS);
    const double id1R = rcp_nr(rdSR * (SR - SM) - bx2 + EPS);
    const double tL = bX * (SM - uL) * id1L, tR = bX * (SM - uR) * id1R;
    const double v1L = L.v - L.bY * tL, w1L = L.w - L.bZ * tL;
    const double v1R = R.v - R.bY * tR, w1R = R.w - R.bZ * tR;
    const double gL = (rdSL * dSL - bx2) * id1L, gR = (rdSR * dSR - bx2) * id1R;
    const double bY1L = L.bY * gL, bZ1L = L.bZ * gL;
    const double bY1R = R.bY * gR, bZ1R = R.bZ * gR;
    const double vbL = uL * bX + L.v * L.bY + L.w * L.bZ, vbR = uR * bX + R.v * R.bY + R.w * R.bZ;
    const double vb1L = SM * bX + v1L * bY1L + w1L * bZ1L, vb1R = SM * bX + v1R * bY1R + w1R * bZ1R;
    const double e1L = (dSL * eL - pTL * uL + pT1 * SM + bX * (vbL - vb1L)) * iSLM;
    const double e1R = (dSR * eR - pTR * uR + pT1 * SM + bX * (vbR - vb1R)) * iSRM;

    const double rsL = rsqrt(rho1L), rsR = rsqrt(rho1R);
    const double sqL = rho1L * rsL, sqR = rho1R * rsR;
    const double abx = fabs(bX);
    const double S1L = SM - abx * rsL, S1R = SM + abx * rsR;
    const double sb = sgn(bX);
    const double id2 = rcp_nr(sqL + sqR + EPS);
    const double sqLR = sqL * sqR;
    const double v2 = (sqL * v1L + sqR * v1R + (bY1R - bY1L) * sb) * id2;
    const double w2 = (sqL * w1L + sqR * w1R + (bZ1R - bZ1L) * sb) * id2;
    const double bY2 = (sqL * bY1R + sqR * bY1L + sqLR * (v1R - v1L) * sb) * id2;
    const double bZ2 = (sqL * bZ1R + sqR * bZ1L + sqLR * (w1R - w1L) * sb) * id2;
    const double vb2 = SM * bX + v2 * bY2 + w2 * bZ2;
    const double e2L = e1L - sqL * (vb1L - vb2) * sb;
    const double e2R = e1R + sqR * (vb1R - vb2) * sb;

    const bool bOL = SL > 0.0;
    const bool bML = (SL <= 0.0) && (0.0 < S1L);
    const bool bIL = (S1L <= 0.0) && (0.0 < SM);
    const bool bOR = SR <= 0.0;
    const bool bMR = (S1R <= 0.0) && (0.0 < SR);
    const bool bIR = (SM <= 0.0) && (0.0 < S1R);
#pragma unroll
    for (int n = 0; n < 8; ++n) f[n] = 0.0;
    const int nsel = (int)bOL + (int)bML + (int)bIL + (int)bOR + (int)bMR + (int)bIR;
    if (nsel == 1) {
        // The usual case: one region is selected; pick its state with
        // selects and form one flux (no per-candidate divergence in a warp).
        const bool lft = bOL | bML | bIL;
        const bool outer = bOL | bOR, inner = bIL | bIR;
        const double rho = bOL ? L.rho : (bOR ? R.rho : (lft ? rho1L : rho1R));
        const double u = bOL ? uL : (bOR ? uR : SM);
        const double v = outer ? (bOL ? L.v : R.v) : (inner ? v2 : (bML ? v1L : v1R));
        const double w = outer ? (bOL ? L.w : R.w) : (inner ? w2 : (bML ? w1L : w1R));
        const double by = outer ? (bOL ? L.bY : R.bY) : (inner ? bY2 : (bML ? bY1L : bY1R));
        const double bz = outer ? (bOL ? L.bZ : R.bZ) : (inner ? bZ2 : (bML ? bZ1L : bZ1R));
        const double e = bOL ? eL : (bOR ? eR : (bML ? e1L : (bIL ? e2L : (bMR ? e1R : e2R))));
        const double pT = bOL ? pTL : (bOR ? pTR : pT1);
        add_one_flux(rho, u, v, w, bX, by, bz, e, pT, f);
    } else {
        if (bOL) add_one_flux(L.rho, uL, L.v, L.w, bX, L.bY, L.bZ, eL, pTL, f);
        if (bML) add_one_flux(rho1L, SM, v1L, w1L, bX, bY1L, bZ1L, e1L, pT1, f);
        if (bIL) add_one_flux(rho1L, SM, v2, w2, bX, bY2, bZ2, e2L, pT1, f);
        if (bOR) add_one_flux(R.rho, uR, R.v, R.w, bX, R.bY, R.bZ, eR, pTR, f);
        if (bMR) add_one_flux(rho1R, SM, v1R, w1R, bX, bY1R, bZ1R, e1R, pT1, f);
        if (bIR) add_one_flux(rho1R, SM, v2, w2, bX, bY2, bZ2, e2R, pT1, f);
    }
    // NaN wave speeds select no candidate here, while the reference's
    // weighted sum turns them into a NaN flux: do the same.
    if ((SL != SL) | (SR != SR) | (SM != SM) | (S1L != S1L) | (S1R != S1R)) {
#pragma unroll
        for (int n = 0; n < 8; ++n) f[n] = qnan;
    }
}

// calculateDtFunctor arithmetic with reciprocals (fast variant); a negative
// squared sound speed gives NaN as the reference's sqrt(gamma p / rho) does.

__device__ __forceinline__ double cfl_rate_fast(double rho, double mx, double my, double mz, double bX,
                                                double bY, double bZ, double e, double gm, double idx,
                                                double idy)
{
    const double ir = rcp_nr(rho);
    const double u = mx * ir, v = my * ir, w = mz * ir;
    const double b2 = bX * bX + bY * bY + bZ * bZ;
    const double p = (gm - 1.0) * (e - 0.5 * rho * (u * u + v * v + w * w) - 0.5 * b2);
    const double cs2 = gm * p * ir, ca2 = b2 * ir;
    const double c = ((cs2 >= 0.0) & (ca2 >= 0.0)) ? sqrt(cs2 + ca2) : bits_to_double(0x7FF8000000000000ull);
    return (fabs(u) + c) * idx + (fabs(v) + c) * idy;
}

// resistiveMHD_2D.cu:247-274 calculateDtFunctor, returning the denominator
// term a = maxSpeedX/dx + maxSpeedY/dy; the cell's dt candidate is
// 1/(a + EPS), so the minimum over cells is 1/(max a + EPS).
__device__ __forceinline__ double cfl_rate(double rho, double mx, double my, double mz, double bX,
                                           double bY, double bZ, double e, double gm, double dx,
                                           double dy)
{
    const double u = mx / rho, v = my / rho, w = mz / rho;
    const double p = (gm - 1.0)
                   * (e - 0.5 * rho * (u * u + v * v + w * w)
                   - 0.5 * (bX * bX + bY * bY + bZ * bZ));
    const double cs = sqrt(gm * p / rho);
    const double ca = sqrt((bX * bX + bY * bY + bZ * bZ) / rho);
    const double sx = fabs(u) + sqrt(cs * cs + ca * ca);
    const double sy = fabs(v) + sqrt(cs * cs + ca * ca);
    return sx / dx + sy / dy;
}

// Order-preserving encoding of a non-negative rate for atomicMax.  A NaN
// rate encodes as 0: the reference's thrust::min_element over the cells'
// dt candidates 1/(a + EPS) (resistiveMHD_2D.cu:286) compares with '<', so
// a NaN candidate never becomes the minimum -- unless it sits in cell k = 0,
// the initial minimum, which the reductions flag separately (first_nan).
__device__ __forceinline__ unsigned long long rate_bits(double a)
{
    if (a != a) return 0ull;
    return (unsigned long long)__double_as_longlong(a);
}


// dt of a step from the reduced rates (resistiveMHD_2D.cu:286-288):
// dtMin = 1/(max a + EPS), or NaN when cell 0's candidate is NaN;
// dt = CFL * min(dtMin, dx^2/eta, dy^2/eta) with the host min() (fmin).
__host__ __device__ __forceinline__ double step_dt(unsigned long long amax_bits, int first_nan, double dx,
                                                  double dy, double eps, double eta, double cfl)
{
    const double dtMin = first_nan ? bits_to_double(0x7FF8000000000000ull) : 1.0 / (bits_to_double(amax_bits) + eps);
    return fmin(dtMin, fmin(dx * dx / eta, dy * dy / eta)) * cfl;
}

}  // namespace rmhd2d
