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
template <typename T> __device__ __forceinline__ T tmin(T a, T b) { return (b < a) ? b : a; }
template <typename T> __device__ __forceinline__ T tmax(T a, T b) { return (a < b) ? b : a; }

// hlld.cu:26-32 Sign, (x > 0) - (x < 0), as selects (no int conversion).
template <typename T> __device__ __forceinline__ T sgn(T x) { return x > T(0) ? T(1) : (x < T(0) ? T(-1) : T(0)); }

// minmod.hpp:6-16: sign_x * max(min(|x|, sign_x * y), EPS) with an int
// sign_x.  Written with selects: for x > 0 the reference computes
// 1.0 * max(min(|x|, 1.0 * y), EPS), for x < 0 the negation of
// max(min(|x|, -y), EPS), for x == 0 (or NaN) 0.0 * max(min(|x|, 0.0 * y), EPS);
// multiplying by +-1 is exact, so this is bit-identical for every input.
//
// Evaluated without branches: m = max(min(|x|, x < 0 ? -y : y), EPS), then
// m, -m or 0 * m by the sign of x.  For x == 0 the reference's inner min
// sees 0 * y where this sees y; min(0, y) and min(0, 0 * y) differ only for
// y < 0 (y versus -0 or 0), and max(., EPS) turns both into EPS, so 0 * m is
// +0 in both; a NaN x or y reaches m the same way in both forms.
template <typename T> __device__ __forceinline__ T minmod(T x, T y, T eps)
{
    const T ax = fabs(x);
    const T m = tmax(tmin(ax, x < T(0) ? -y : y), eps);
    return x > T(0) ? m : (x < T(0) ? -m : T(0) * m);
}

// Single-precision reciprocal and square roots of the FP32-bulk variant
// (hardware approximations, ~1 ulp of float).  A host build of the kernels
// (CPU tests, RMHD_HOST_EMULATION) takes the correctly rounded values.
__device__ __forceinline__ float rcp_nr(float a)
{
#if defined(RMHD_HOST_EMULATION)
    return 1.0f / a;
#else
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a));
    return r;
#endif
}
__device__ __forceinline__ float rsqrt_t(float a)
{
#if defined(RMHD_HOST_EMULATION)
    return 1.0f / sqrtf(a);
#else
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a));
    return r;
#endif
}
__device__ __forceinline__ float sqrt_t(float a)
{
#if defined(RMHD_HOST_EMULATION)
    return sqrtf(a);
#else
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a));
    return r;
#endif
}
__device__ __forceinline__ double rsqrt_t(double a) { return rsqrt(a); }
__device__ __forceinline__ double sqrt_t(double a) { return sqrt(a); }

// Reciprocal by Newton-Raphson iteration on 1/a (x' = x + x (1 - a x), two
// steps, each squaring the relative error) from the hardware seed
// rcp.approx.ftz.f64 (a host build: the correctly rounded 1/a); used by the
// fast variant only.  Accurate to about one ulp for normal finite a; a = 0
// or +-inf give NaN (the fast variant's denominators carry the reference's
// +EPS and are never 0 in a finite state).
__device__ __forceinline__ double rcp_nr(double a)
{
    double r;
#if defined(RMHD_HOST_EMULATION)
    r = 1.0 / a;
#else
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(a));
#endif
    double e = fma(-a, r, 1.0);
    r = fma(r, e, r);
    e = fma(-a, r, 1.0);
    r = fma(r, e, r);
    return r;
}

// ---- correctly rounded division through a shared reciprocal ----
//
// An IEEE division costs about as much FP64 issue as 14 fused multiply-adds
// on sm_100.  The exact variant divides by the same denominator several
// times per interface, so it divides through the correctly rounded
// reciprocal y = RN(1/b) instead, with Markstein's correction (P. Markstein,
// "Computation of elementary functions on the IBM RISC System/6000
// processor", IBM J. Res. Dev. 34(1), 1990; Theorem 4.10 of Muller et al.,
// Handbook of Floating-Point Arithmetic): with q = RN(a y) within one ulp of
// a/b, the remainder r = a - b q is exact in one fma and RN(q + r y) =
// RN(a/b), as long as nothing overflows or underflows.
//
// y comes from the hardware seed by two Newton steps (each squares the
// relative error, leaving y within an ulp of 1/b) and Markstein's last
// step y + y (1 - b y), which rounds correctly except for significands of b
// that are all ones.  The guard of MdDiv records every operand outside the
// range where all of this holds -- a divisor outside [2^-400, 2^400) or with
// an all-ones significand, a quotient outside [2^-500, 2^500) unless the
// dividend is zero -- and the caller then repeats the computation with IEEE
// division.  A zero dividend returns q itself, which carries the sign
// IEEE division gives (q + r y would turn -0 into +0).
//
// tests/test_division.py checks the quotients against IEEE division on
// random and special operands (on the CPU for the algorithm, on the GPU for
// the hardware seed).
__device__ __forceinline__ double rcp_rn_md(double b)
{
    double y;
#if defined(RMHD_HOST_EMULATION)
    // a seed with the precision of the hardware's (its low 28 significand
    // bits cleared), so that a host build exercises the refinement
    {
        unsigned long long u;
        const double r = 1.0 / b;
        memcpy(&u, &r, sizeof(u));
        u &= ~((1ull << 28) - 1);
        memcpy(&y, &u, sizeof(y));
    }
#else
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(b));
#endif
    double e = fma(-b, y, 1.0);
    y = fma(y, e, y);
    e = fma(-b, y, 1.0);
    y = fma(y, e, y);
    e = fma(-b, y, 1.0);
    return fma(y, e, y);
}

__host__ __device__ __forceinline__ unsigned int hi_word(double x)
{
#ifdef __CUDA_ARCH__
    return (unsigned int)__double2hiint(x);
#else
    unsigned long long u;
    memcpy(&u, &x, sizeof(u));
    return (unsigned int)(u >> 32);
#endif
}
__host__ __device__ __forceinline__ unsigned int lo_word(double x)
{
#ifdef __CUDA_ARCH__
    return (unsigned int)__double2loint(x);
#else
    unsigned long long u;
    memcpy(&u, &x, sizeof(u));
    return (unsigned int)u;
#endif
}

// Division policy of the exact arithmetic: shared reciprocals with the
// guard above.  recip(b) returns y; div(a, b, y) returns RN(a/b) whenever ok
// stays true.
struct MdDiv {
    bool ok = true;
    __device__ __forceinline__ double recip(double b)
    {
        const unsigned int h = hi_word(b);
        // |b| in [2^-400, 2^400): biased exponent in [623, 1423)
        ok &= ((h & 0x7FFFFFFFu) - 0x26F00000u) < 0x32000000u;
        ok &= ((h & 0x000FFFFFu) != 0x000FFFFFu) | (lo_word(b) != 0xFFFFFFFFu);
        return rcp_rn_md(b);
    }
    __device__ __forceinline__ double div(double a, double b, double y)
    {
        const double q = a * y;
        const double r = fma(-q, b, a);
        const double q1 = fma(r, y, q);
        const bool z = a == 0.0;
        // |q| in [2^-500, 2^500): biased exponent in [523, 1523)
        ok &= z | (((hi_word(q) & 0x7FFFFFFFu) - 0x20B00000u) < 0x3E800000u);
        return z ? q : q1;
    }
};

// Division policy with plain IEEE division (the fallback of MdDiv).
struct IeeeDiv {
    static constexpr bool ok = true;
    __device__ __forceinline__ double recip(double b) { return b; }
    __device__ __forceinline__ double div(double a, double b, double) { return a / b; }
};

// Interface state fed to HLLD: BasicParameter (basic_parameter_struct.hpp:5-27).
template <typename T> struct PrimT {
    T rho, u, v, w, bX, bY, bZ, p;
};
using Prim = PrimT<double>;

// hlld.cu:448-467 getOneFlux, accumulated into f (f4 is identically 0 and
// is not produced).
template <typename T>
__device__ __forceinline__ void add_one_flux(T rho, T u, T v, T w, T bX, T bY, T bZ, T e, T pT, T f[8])
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
// hlld.cu:35-107 (CalculateFluxFunctor), with the divisions of the policy
// Div (MdDiv: shared correctly rounded reciprocals; IeeeDiv: plain division);
// both give the reference's quotients bit for bit while Div::ok holds.
// ygm1 is Div's reciprocal handle of gm - 1.
//
// ALL_CANDIDATES = true gives the bits of the reference's sum of all six
// candidate fluxes with 0/1 indicator weights for every input, including
// non-finite ones: it forms that sum unless exactly one candidate is selected
// and all candidate values are bounded, where the selected flux alone has the
// same bits.  ALL_CANDIDATES = false forms only the candidates whose
// indicator is 1 and adds them in the reference's order, which gives the same
// bits whenever all six candidates are finite.
template <bool ALL_CANDIDATES, class Div>
__device__ __forceinline__ void hlld_body(const Prim &L, const Prim &R, double gm, double EPS, double ygm1, Div &dv,
                                          double f[8])
{
    const double rhoL = L.rho, uL = L.u, vL = L.v, wL = L.w, bXL = L.bX, bYL = L.bY, bZL = L.bZ, pL = L.p;
    const double rhoR = R.rho, uR = R.u, vR = R.v, wR = R.w, bXR = R.bX, bYR = R.bY, bZR = R.bZ, pR = R.p;
    const double gm1 = gm - 1.0;

    const double eL = dv.div(pL, gm1, ygm1)
                    + 0.5 * rhoL * (uL * uL + vL * vL + wL * wL)
                    + 0.5 * (bXL * bXL + bYL * bYL + bZL * bZL);
    const double pTL = pL + 0.5 * (bXL * bXL + bYL * bYL + bZL * bZL);
    const double eR = dv.div(pR, gm1, ygm1)
                    + 0.5 * rhoR * (uR * uR + vR * vR + wR * wR)
                    + 0.5 * (bXR * bXR + bYR * bYR + bZR * bZR);
    const double pTR = pR + 0.5 * (bXR * bXR + bYR * bYR + bZR * bZR);

    const double yrL = dv.recip(rhoL), yrR = dv.recip(rhoR);
    const double csL = sqrt(dv.div(gm * pL, rhoL, yrL));
    const double caL = sqrt(dv.div(bXL * bXL + bYL * bYL + bZL * bZL, rhoL, yrL));
    const double vaL = sqrt(dv.div(bXL * bXL, rhoL, yrL));
    const double cfL = sqrt(0.5 * (csL * csL + caL * caL
                     + sqrt((csL * csL + caL * caL) * (csL * csL + caL * caL)
                     - 4.0 * csL * csL * vaL * vaL)));
    const double csR = sqrt(dv.div(gm * pR, rhoR, yrR));
    const double caR = sqrt(dv.div(bXR * bXR + bYR * bYR + bZR * bZR, rhoR, yrR));
    const double vaR = sqrt(dv.div(bXR * bXR, rhoR, yrR));
    const double cfR = sqrt(0.5 * (csR * csR + caR * caR
                     + sqrt((csR * csR + caR * caR) * (csR * csR + caR * caR)
                     - 4.0 * csR * csR * vaR * vaR)));

    double SL = tmin(uL, uR) - tmax(cfL, cfR);
    double SR = tmax(uL, uR) + tmax(cfL, cfR);
    SL = tmin(SL, 0.0);
    SR = tmax(SR, 0.0);

    const double den = (SR - uR) * rhoR - (SL - uL) * rhoL + EPS;
    const double yden = dv.recip(den);
    const double SM = dv.div((SR - uR) * rhoR * uR - (SL - uL) * rhoL * uL - pTR + pTL, den, yden);
    const double pT1 = dv.div((SR - uR) * rhoR * pTL - (SL - uL) * rhoL * pTR
                              + rhoL * rhoR * (SR - uR) * (SL - uL) * (uR - uL), den, yden);

    const double dLM = SL - SM + EPS, dRM = SR - SM + EPS;
    const double yLM = dv.recip(dLM), yRM = dv.recip(dRM);
    const double DL = rhoL * (SL - uL) * (SL - SM) - bXL * bXL + EPS;
    const double DR = rhoR * (SR - uR) * (SR - SM) - bXR * bXR + EPS;
    const double yDL = dv.recip(DL), yDR = dv.recip(DR);
    const double NL = rhoL * (SL - uL) * (SL - uL) - bXL * bXL;
    const double NR = rhoR * (SR - uR) * (SR - uR) - bXR * bXR;

    const double rho1L = dv.div(rhoL * (SL - uL), dLM, yLM);
    const double u1L = SM;
    const double v1L = vL - dv.div(bXL * bYL * (SM - uL), DL, yDL);
    const double w1L = wL - dv.div(bXL * bZL * (SM - uL), DL, yDL);
    const double bX1L = bXL;
    const double bY1L = dv.div(bYL * NL, DL, yDL);
    const double bZ1L = dv.div(bZL * NL, DL, yDL);
    const double e1L = dv.div((SL - uL) * eL - pTL * uL + pT1 * SM
                              + bXL * ((uL * bXL + vL * bYL + wL * bZL) - (u1L * bX1L + v1L * bY1L + w1L * bZ1L)),
                              dLM, yLM);

    const double rho1R = dv.div(rhoR * (SR - uR), dRM, yRM);
    const double u1R = SM;
    const double v1R = vR - dv.div(bXR * bYR * (SM - uR), DR, yDR);
    const double w1R = wR - dv.div(bXR * bZR * (SM - uR), DR, yDR);
    const double bX1R = bXR;
    const double bY1R = dv.div(bYR * NR, DR, yDR);
    const double bZ1R = dv.div(bZR * NR, DR, yDR);
    const double e1R = dv.div((SR - uR) * eR - pTR * uR + pT1 * SM
                              + bXR * ((uR * bXR + vR * bYR + wR * bZR) - (u1R * bX1R + v1R * bY1R + w1R * bZ1R)),
                              dRM, yRM);

    const double S1L = SM - sqrt(bX1L * bX1L / rho1L);
    const double S1R = SM + sqrt(bX1R * bX1R / rho1R);

    const double sqL = sqrt(rho1L), sqR = sqrt(rho1R), sqLR = sqrt(rho1L * rho1R);
    const double sbX = sgn(bX1L);
    const double u2 = SM;
    const double dsq = sqL + sqR + EPS;
    const double ysq = dv.recip(dsq);
    const double v2 = dv.div(sqL * v1L + sqR * v1R + (bY1R - bY1L) * sbX, dsq, ysq);
    const double w2 = dv.div(sqL * w1L + sqR * w1R + (bZ1R - bZ1L) * sbX, dsq, ysq);
    const double bY2 = dv.div(sqL * bY1R + sqR * bY1L + sqLR * (v1R - v1L) * sbX, dsq, ysq);
    const double bZ2 = dv.div(sqL * bZ1R + sqR * bZ1L + sqLR * (w1R - w1L) * sbX, dsq, ysq);
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
        // The weighted sum adds F * 0 = +-0 for every unselected candidate
        // whose flux is finite, which leaves the selected candidate's flux
        // bit for bit.  A flux component is a product of at most three of
        // the candidate's values plus a few such products, so it is finite
        // whenever every value is below 1e75 in magnitude; the sum of
        // magnitudes below is NaN or infinite, and fails the test, as soon
        // as one value is.  Then, with exactly one region selected, only
        // that candidate is formed; otherwise all six are.
        const int nsel = (int)bOL + (int)bML + (int)bIL + (int)bOR + (int)bMR + (int)bIR;
        const double mag = fabs(rhoL) + fabs(uL) + fabs(vL) + fabs(wL) + fabs(bXL) + fabs(bYL) + fabs(bZL)
                         + fabs(eL) + fabs(pTL) + fabs(rhoR) + fabs(uR) + fabs(vR) + fabs(wR) + fabs(bXR)
                         + fabs(bYR) + fabs(bZR) + fabs(eR) + fabs(pTR) + fabs(rho1L) + fabs(rho1R) + fabs(SM)
                         + fabs(pT1) + fabs(v1L) + fabs(w1L) + fabs(bY1L) + fabs(bZ1L) + fabs(e1L) + fabs(v1R)
                         + fabs(w1R) + fabs(bY1R) + fabs(bZ1R) + fabs(e1R) + fabs(v2) + fabs(w2) + fabs(bY2)
                         + fabs(bZ2) + fabs(e2L) + fabs(e2R);
        if (nsel == 1 && mag < 1e75) {
            const bool lft = bOL | bML | bIL;
            const bool outer = bOL | bOR, inner = bIL | bIR;
            const double rho = bOL ? rhoL : (bOR ? rhoR : (lft ? rho1L : rho1R));
            const double u = bOL ? uL : (bOR ? uR : SM);
            const double v = outer ? (bOL ? vL : vR) : (inner ? v2 : (bML ? v1L : v1R));
            const double w = outer ? (bOL ? wL : wR) : (inner ? w2 : (bML ? w1L : w1R));
            const double bx = lft ? bXL : bXR;
            const double by = outer ? (bOL ? bYL : bYR) : (inner ? bY2 : (bML ? bY1L : bY1R));
            const double bz = outer ? (bOL ? bZL : bZR) : (inner ? bZ2 : (bML ? bZ1L : bZ1R));
            const double e = bOL ? eL : (bOR ? eR : (bML ? e1L : (bIL ? e2L : (bMR ? e1R : e2R))));
            const double pT = bOL ? pTL : (bOR ? pTR : pT1);
            add_one_flux(rho, u, v, w, bx, by, bz, e, pT, f);
            return;
        }
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

// The exact HLLD flux: shared correctly rounded reciprocals, repeated with
// IEEE division where the guard of MdDiv fails (non-finite, huge or tiny
// operands).  ygm1 = rcp_rn_md(gm - 1), gm1_ok = MdDiv's guard on it.
template <bool ALL_CANDIDATES>
__device__ __forceinline__ void hlld_flux(const Prim &L, const Prim &R, double gm, double EPS, double ygm1,
                                          bool gm1_ok, double f[8])
{
    MdDiv md;
    md.ok = gm1_ok;
    hlld_body<ALL_CANDIDATES>(L, R, gm, EPS, ygm1, md, f);
    if (!md.ok) {
        IeeeDiv id;
        hlld_body<ALL_CANDIDATES>(L, R, gm, EPS, gm - 1.0, id, f);
    }
}

// The same, forming the reciprocal of gm - 1 itself.
template <bool ALL_CANDIDATES>
__device__ __forceinline__ void hlld_flux(const Prim &L, const Prim &R, double gm, double EPS, double f[8])
{
    MdDiv g1;
    const double ygm1 = g1.recip(gm - 1.0);
    hlld_flux<ALL_CANDIDATES>(L, R, gm, EPS, ygm1, g1.ok, f);
}

// The reference's arithmetic in full: IEEE division and all six candidates
// weighted, for every input.  The rare path of hlld_flux_sel.
__device__ __forceinline__ void hlld_flux_ieee(const Prim &L, const Prim &R, double gm, double EPS, double f[8])
{
    IeeeDiv id;
    hlld_body<true>(L, R, gm, EPS, gm - 1.0, id, f);
}

// The exact HLLD flux with the candidate picked as the fan is built.  Every
// value is the same expression as in hlld_body, so the bits are those of
// hlld_flux<true>; only what stays live differs.  hlld_body keeps all six
// candidate states (38 values) live until the region flags are known and
// then selects; here each candidate is taken into the nine `c*` values as
// soon as its own flag is known, so the left and right input states die
// after the star states, and the magnitude guard is summed as the values
// appear.  Where the shortcut's conditions fail -- a guard of the shared
// reciprocals, more or fewer than one region selected, a value of 1e75 or
// more (or non-finite) -- it returns false with f unwritten, and the caller
// forms the interface with hlld_flux_ieee, away from its common path (the
// stage kernel's flux phase does that after its loop, for the interfaces
// that asked, so the rare path does not shape the common path's registers).
__device__ __forceinline__ bool hlld_flux_sel(const Prim &L, const Prim &R, double gm, double EPS, double ygm1,
                                              bool gm1_ok, double f[8])
{
    MdDiv dv;
    dv.ok = gm1_ok;
    const double rhoL = L.rho, uL = L.u, vL = L.v, wL = L.w, bXL = L.bX, bYL = L.bY, bZL = L.bZ, pL = L.p;
    const double rhoR = R.rho, uR = R.u, vR = R.v, wR = R.w, bXR = R.bX, bYR = R.bY, bZR = R.bZ, pR = R.p;
    const double gm1 = gm - 1.0;

    const double eL = dv.div(pL, gm1, ygm1)
                    + 0.5 * rhoL * (uL * uL + vL * vL + wL * wL)
                    + 0.5 * (bXL * bXL + bYL * bYL + bZL * bZL);
    const double pTL = pL + 0.5 * (bXL * bXL + bYL * bYL + bZL * bZL);
    const double eR = dv.div(pR, gm1, ygm1)
                    + 0.5 * rhoR * (uR * uR + vR * vR + wR * wR)
                    + 0.5 * (bXR * bXR + bYR * bYR + bZR * bZR);
    const double pTR = pR + 0.5 * (bXR * bXR + bYR * bYR + bZR * bZR);
    // magnitude guard of the shortcut (any order of summation will do: the
    // guard only chooses between two evaluations with the same bits)
    double mag = fabs(rhoL) + fabs(uL) + fabs(vL) + fabs(wL) + fabs(bXL) + fabs(bYL) + fabs(bZL) + fabs(eL)
               + fabs(pTL) + fabs(rhoR) + fabs(uR) + fabs(vR) + fabs(wR) + fabs(bXR) + fabs(bYR) + fabs(bZR)
               + fabs(eR) + fabs(pTR);

    const double yrL = dv.recip(rhoL), yrR = dv.recip(rhoR);
    const double csL = sqrt(dv.div(gm * pL, rhoL, yrL));
    const double caL = sqrt(dv.div(bXL * bXL + bYL * bYL + bZL * bZL, rhoL, yrL));
    const double vaL = sqrt(dv.div(bXL * bXL, rhoL, yrL));
    const double cfL = sqrt(0.5 * (csL * csL + caL * caL
                     + sqrt((csL * csL + caL * caL) * (csL * csL + caL * caL)
                     - 4.0 * csL * csL * vaL * vaL)));
    const double csR = sqrt(dv.div(gm * pR, rhoR, yrR));
    const double caR = sqrt(dv.div(bXR * bXR + bYR * bYR + bZR * bZR, rhoR, yrR));
    const double vaR = sqrt(dv.div(bXR * bXR, rhoR, yrR));
    const double cfR = sqrt(0.5 * (csR * csR + caR * caR
                     + sqrt((csR * csR + caR * caR) * (csR * csR + caR * caR)
                     - 4.0 * csR * csR * vaR * vaR)));

    double SL = tmin(uL, uR) - tmax(cfL, cfR);
    double SR = tmax(uL, uR) + tmax(cfL, cfR);
    SL = tmin(SL, 0.0);
    SR = tmax(SR, 0.0);

    // the outer states: candidates of their own
    const bool bOL = SL > 0.0;
    const bool bOR = SR <= 0.0;
    double cr = bOL ? rhoL : rhoR, cu = bOL ? uL : uR, cv = bOL ? vL : vR, cw = bOL ? wL : wR;
    double cbx = bOL ? bXL : bXR, cby = bOL ? bYL : bYR, cbz = bOL ? bZL : bZR;
    double ce = bOL ? eL : eR, cpt = bOL ? pTL : pTR;
    int nsel = (int)bOL + (int)bOR;

    const double den = (SR - uR) * rhoR - (SL - uL) * rhoL + EPS;
    const double yden = dv.recip(den);
    const double SM = dv.div((SR - uR) * rhoR * uR - (SL - uL) * rhoL * uL - pTR + pTL, den, yden);
    const double pT1 = dv.div((SR - uR) * rhoR * pTL - (SL - uL) * rhoL * pTR
                              + rhoL * rhoR * (SR - uR) * (SL - uL) * (uR - uL), den, yden);
    mag += fabs(SM) + fabs(pT1);

    // left star state (u1L = SM, bX1L = bXL)
    const double dLM = SL - SM + EPS;
    const double yLM = dv.recip(dLM);
    const double DL = rhoL * (SL - uL) * (SL - SM) - bXL * bXL + EPS;
    const double yDL = dv.recip(DL);
    const double NL = rhoL * (SL - uL) * (SL - uL) - bXL * bXL;
    const double rho1L = dv.div(rhoL * (SL - uL), dLM, yLM);
    const double v1L = vL - dv.div(bXL * bYL * (SM - uL), DL, yDL);
    const double w1L = wL - dv.div(bXL * bZL * (SM - uL), DL, yDL);
    const double bY1L = dv.div(bYL * NL, DL, yDL);
    const double bZ1L = dv.div(bZL * NL, DL, yDL);
    const double vb1L = SM * bXL + v1L * bY1L + w1L * bZ1L;
    const double e1L = dv.div((SL - uL) * eL - pTL * uL + pT1 * SM
                              + bXL * ((uL * bXL + vL * bYL + wL * bZL) - vb1L),
                              dLM, yLM);
    mag += fabs(rho1L) + fabs(v1L) + fabs(w1L) + fabs(bY1L) + fabs(bZ1L) + fabs(e1L);
    const double yr1L = dv.recip(rho1L);
    const double S1L = SM - sqrt(dv.div(bXL * bXL, rho1L, yr1L));
    const bool bML = (SL <= 0.0) && (0.0 < S1L);
    const bool bIL = (S1L <= 0.0) && (0.0 < SM);
    if (bML) {
        cr = rho1L; cu = SM; cv = v1L; cw = w1L; cbx = bXL; cby = bY1L; cbz = bZ1L; ce = e1L; cpt = pT1;
    }

    // right star state
    const double dRM = SR - SM + EPS;
    const double yRM = dv.recip(dRM);
    const double DR = rhoR * (SR - uR) * (SR - SM) - bXR * bXR + EPS;
    const double yDR = dv.recip(DR);
    const double NR = rhoR * (SR - uR) * (SR - uR) - bXR * bXR;
    const double rho1R = dv.div(rhoR * (SR - uR), dRM, yRM);
    const double v1R = vR - dv.div(bXR * bYR * (SM - uR), DR, yDR);
    const double w1R = wR - dv.div(bXR * bZR * (SM - uR), DR, yDR);
    const double bY1R = dv.div(bYR * NR, DR, yDR);
    const double bZ1R = dv.div(bZR * NR, DR, yDR);
    const double vb1R = SM * bXR + v1R * bY1R + w1R * bZ1R;
    const double e1R = dv.div((SR - uR) * eR - pTR * uR + pT1 * SM
                              + bXR * ((uR * bXR + vR * bYR + wR * bZR) - vb1R),
                              dRM, yRM);
    mag += fabs(rho1R) + fabs(v1R) + fabs(w1R) + fabs(bY1R) + fabs(bZ1R) + fabs(e1R);
    const double yr1R = dv.recip(rho1R);
    const double S1R = SM + sqrt(dv.div(bXR * bXR, rho1R, yr1R));
    const bool bMR = (S1R <= 0.0) && (0.0 < SR);
    const bool bIR = (SM <= 0.0) && (0.0 < S1R);
    if (bMR) {
        cr = rho1R; cu = SM; cv = v1R; cw = w1R; cbx = bXR; cby = bY1R; cbz = bZ1R; ce = e1R; cpt = pT1;
    }
    nsel += (int)bML + (int)bIL + (int)bMR + (int)bIR;

    // double-star states (u2 = SM)
    const double sqL = sqrt(rho1L), sqR = sqrt(rho1R), sqLR = sqrt(rho1L * rho1R);
    const double sbX = sgn(bXL);
    const double dsq = sqL + sqR + EPS;
    const double ysq = dv.recip(dsq);
    const double v2 = dv.div(sqL * v1L + sqR * v1R + (bY1R - bY1L) * sbX, dsq, ysq);
    const double w2 = dv.div(sqL * w1L + sqR * w1R + (bZ1R - bZ1L) * sbX, dsq, ysq);
    const double bY2 = dv.div(sqL * bY1R + sqR * bY1L + sqLR * (v1R - v1L) * sbX, dsq, ysq);
    const double bZ2 = dv.div(sqL * bZ1R + sqR * bZ1L + sqLR * (w1R - w1L) * sbX, dsq, ysq);
    const double e2L = e1L - sqL * (vb1L - (SM * bXL + v2 * bY2 + w2 * bZ2)) * sgn(bXL);
    const double e2R = e1R + sqR * (vb1R - (SM * bXR + v2 * bY2 + w2 * bZ2)) * sgn(bXR);
    mag += fabs(v2) + fabs(w2) + fabs(bY2) + fabs(bZ2) + fabs(e2L) + fabs(e2R);
    if (bIL | bIR) {
        cr = bIL ? rho1L : rho1R; cu = SM; cv = v2; cw = w2; cbx = bIL ? bXL : bXR;
        cby = bY2; cbz = bZ2; ce = bIL ? e2L : e2R; cpt = pT1;
    }

    if (!dv.ok || nsel != 1 || !(mag < 1e75)) return false;
#pragma unroll
    for (int n = 0; n < 8; ++n) f[n] = 0.0;
    add_one_flux(cr, cu, cv, cw, cbx, cby, cbz, ce, cpt, f);
    return true;
}

// HLLD flux of the fast variant: the same wave-speed estimates, star and
// double-star states and candidate selection as hlld_flux (hlld.cu:256-565),
// rearranged for the FP64 pipe.  It differs from the exact form by rounding
// only: one correctly rounded reciprocal per distinct denominator (8 instead
// of 28 divisions), squared sound/Alfven speeds used directly (the reference
// squares their square roots), sqrt(rho*) and |bX|/sqrt(rho*) from one rsqrt,
// and bX taken once (left and right states share the interface-normal B).
//
// ONE = true forms the common case only: exactly one region selected and
// finite wave speeds.  That region's state is taken into the `c*` values as
// soon as its flag is known, so the input states need not stay live until
// the end; it returns false (f unwritten) when the case does not apply.
// ONE = false forms every case.
template <bool ONE, typename T>
__device__ __forceinline__ bool hlld_fast_body(const PrimT<T> &L, const PrimT<T> &R, T gm, T inv_gm1, T EPS, T f[8])
{
    const T bX = L.bX;
    const T bx2 = bX * bX;
    const T iRL = rcp_nr(L.rho), iRR = rcp_nr(R.rho);
    const T b2L = bx2 + L.bY * L.bY + L.bZ * L.bZ;
    const T b2R = bx2 + R.bY * R.bY + R.bZ * R.bZ;
    const T eL = L.p * inv_gm1 + T(0.5) * L.rho * (L.u * L.u + L.v * L.v + L.w * L.w) + T(0.5) * b2L;
    const T eR = R.p * inv_gm1 + T(0.5) * R.rho * (R.u * R.u + R.v * R.v + R.w * R.w) + T(0.5) * b2R;
    const T pTL = L.p + T(0.5) * b2L, pTR = R.p + T(0.5) * b2R;

    const T cs2L = gm * L.p * iRL, ca2L = b2L * iRL, va2L = bx2 * iRL;
    const T cs2R = gm * R.p * iRR, ca2R = b2R * iRR, va2R = bx2 * iRR;
    const T sL = cs2L + ca2L, sR = cs2R + ca2R;
    // The reference takes sqrt of each squared speed, so a negative one makes
    // its fast speed NaN; keep that.  The discriminant
    // (cs2 + ca2)^2 - 4 cs2 va2 is formed as (cs2 - ca2)^2 + 4 cs2 bt2 / rho
    // (bt2 the tangential |B|^2, ca2 - va2 = bt2 / rho): the same number
    // without the cancellation that rounds it below zero where the
    // tangential field vanishes and cs ~ ca.
    const T qnan = T(bits_to_double(0x7FF8000000000000ull));
    const bool okL = (cs2L >= T(0)) & (ca2L >= T(0)) & (va2L >= T(0));
    const bool okR = (cs2R >= T(0)) & (ca2R >= T(0)) & (va2R >= T(0));
    const T dcL = cs2L - ca2L, dcR = cs2R - ca2R;
    const T discL = dcL * dcL + T(4.0) * cs2L * (L.bY * L.bY + L.bZ * L.bZ) * iRL;
    const T discR = dcR * dcR + T(4.0) * cs2R * (R.bY * R.bY + R.bZ * R.bZ) * iRR;
    const T cfL = okL ? sqrt_t(T(0.5) * (sL + sqrt_t(discL))) : qnan;
    const T cfR = okR ? sqrt_t(T(0.5) * (sR + sqrt_t(discR))) : qnan;

    const T uL = L.u, uR = R.u;
    T SL = tmin(uL, uR) - tmax(cfL, cfR);
    T SR = tmax(uL, uR) + tmax(cfL, cfR);
    SL = tmin(SL, T(0));
    SR = tmax(SR, T(0));

    const bool bOL = SL > T(0);
    const bool bOR = SR <= T(0);
    T cr, cu, cv, cw, cby, cbz, ce, cpt;   // the selected candidate (ONE)
    if (ONE) {
        cr = bOL ? L.rho : R.rho; cu = bOL ? L.u : R.u; cv = bOL ? L.v : R.v; cw = bOL ? L.w : R.w;
        cby = bOL ? L.bY : R.bY; cbz = bOL ? L.bZ : R.bZ; ce = bOL ? eL : eR; cpt = bOL ? pTL : pTR;
    }

    const T dSL = SL - uL, dSR = SR - uR;
    const T rdSL = L.rho * dSL, rdSR = R.rho * dSR;
    const T iden = rcp_nr(rdSR - rdSL + EPS);
    const T SM = (rdSR * uR - rdSL * uL - pTR + pTL) * iden;
    const T pT1 = (rdSR * pTL - rdSL * pTR + rdSL * rdSR * (uR - uL)) * iden;

    const T iSLM = rcp_nr(SL - SM + EPS), iSRM = rcp_nr(SR - SM + EPS);
    const T rho1L = rdSL * iSLM, rho1R = rdSR * iSRM;
    const T id1L = rcp_nr(rdSL * (SL - SM) - bx2 + EPS);
    const T id1R = rcp_nr(rdSR * (SR - SM) - bx2 + EPS);
    const T tL = bX * (SM - uL) * id1L, tR = bX * (SM - uR) * id1R;
    const T v1L = L.v - L.bY * tL, w1L = L.w - L.bZ * tL;
    const T v1R = R.v - R.bY * tR, w1R = R.w - R.bZ * tR;
    const T gL = (rdSL * dSL - bx2) * id1L, gR = (rdSR * dSR - bx2) * id1R;
    const T bY1L = L.bY * gL, bZ1L = L.bZ * gL;
    const T bY1R = R.bY * gR, bZ1R = R.bZ * gR;
    const T vbL = uL * bX + L.v * L.bY + L.w * L.bZ, vbR = uR * bX + R.v * R.bY + R.w * R.bZ;
    const T vb1L = SM * bX + v1L * bY1L + w1L * bZ1L, vb1R = SM * bX + v1R * bY1R + w1R * bZ1R;
    const T e1L = (dSL * eL - pTL * uL + pT1 * SM + bX * (vbL - vb1L)) * iSLM;
    const T e1R = (dSR * eR - pTR * uR + pT1 * SM + bX * (vbR - vb1R)) * iSRM;

    const T rsL = rsqrt_t(rho1L), rsR = rsqrt_t(rho1R);
    const T sqL = rho1L * rsL, sqR = rho1R * rsR;
    const T abx = fabs(bX);
    const T S1L = SM - abx * rsL, S1R = SM + abx * rsR;
    const bool bML = (SL <= T(0)) && (T(0) < S1L);
    const bool bIL = (S1L <= T(0)) && (T(0) < SM);
    const bool bMR = (S1R <= T(0)) && (T(0) < SR);
    const bool bIR = (SM <= T(0)) && (T(0) < S1R);
    if (ONE && (bML | bMR)) {
        cr = bML ? rho1L : rho1R; cu = SM; cv = bML ? v1L : v1R; cw = bML ? w1L : w1R;
        cby = bML ? bY1L : bY1R; cbz = bML ? bZ1L : bZ1R; ce = bML ? e1L : e1R; cpt = pT1;
    }
    const T sb = sgn(bX);
    const T id2 = rcp_nr(sqL + sqR + EPS);
    const T sqLR = sqL * sqR;
    const T v2 = (sqL * v1L + sqR * v1R + (bY1R - bY1L) * sb) * id2;
    const T w2 = (sqL * w1L + sqR * w1R + (bZ1R - bZ1L) * sb) * id2;
    const T bY2 = (sqL * bY1R + sqR * bY1L + sqLR * (v1R - v1L) * sb) * id2;
    const T bZ2 = (sqL * bZ1R + sqR * bZ1L + sqLR * (w1R - w1L) * sb) * id2;
    const T vb2 = SM * bX + v2 * bY2 + w2 * bZ2;
    const T e2L = e1L - sqL * (vb1L - vb2) * sb;
    const T e2R = e1R + sqR * (vb1R - vb2) * sb;

    const int nsel = (int)bOL + (int)bML + (int)bIL + (int)bOR + (int)bMR + (int)bIR;
    const bool nan_speed = (SL != SL) | (SR != SR) | (SM != SM) | (S1L != S1L) | (S1R != S1R);
    if (ONE) {
        if (nsel != 1 || nan_speed) return false;
        if (bIL | bIR) {
            cr = bIL ? rho1L : rho1R; cu = SM; cv = v2; cw = w2; cby = bY2; cbz = bZ2; ce = bIL ? e2L : e2R;
            cpt = pT1;
        }
#pragma unroll
        for (int n = 0; n < 8; ++n) f[n] = T(0);
        add_one_flux(cr, cu, cv, cw, bX, cby, cbz, ce, cpt, f);
        return true;
    }
#pragma unroll
    for (int n = 0; n < 8; ++n) f[n] = T(0);
    if (nsel == 1) {
        // The usual case: one region is selected; pick its state with
        // selects and form one flux (no per-candidate divergence in a warp).
        const bool lft = bOL | bML | bIL;
        const bool outer = bOL | bOR, inner = bIL | bIR;
        const T rho = bOL ? L.rho : (bOR ? R.rho : (lft ? rho1L : rho1R));
        const T u = bOL ? uL : (bOR ? uR : SM);
        const T v = outer ? (bOL ? L.v : R.v) : (inner ? v2 : (bML ? v1L : v1R));
        const T w = outer ? (bOL ? L.w : R.w) : (inner ? w2 : (bML ? w1L : w1R));
        const T by = outer ? (bOL ? L.bY : R.bY) : (inner ? bY2 : (bML ? bY1L : bY1R));
        const T bz = outer ? (bOL ? L.bZ : R.bZ) : (inner ? bZ2 : (bML ? bZ1L : bZ1R));
        const T e = bOL ? eL : (bOR ? eR : (bML ? e1L : (bIL ? e2L : (bMR ? e1R : e2R))));
        const T pT = bOL ? pTL : (bOR ? pTR : pT1);
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
    if (nan_speed) {
#pragma unroll
        for (int n = 0; n < 8; ++n) f[n] = qnan;
    }
    return true;
}

// Every case of the fast HLLD flux.
template <typename T>
__device__ __forceinline__ void hlld_flux_fast(const PrimT<T> &L, const PrimT<T> &R, T gm, T inv_gm1, T EPS, T f[8])
{
    hlld_fast_body<false>(L, R, gm, inv_gm1, EPS, f);
}

// The common case of the fast HLLD flux (one region, finite wave speeds);
// false, with f unwritten, where it does not apply: the caller then forms
// the interface with hlld_flux_fast away from its common path.
template <typename T>
__device__ __forceinline__ bool hlld_flux_fast_sel(const PrimT<T> &L, const PrimT<T> &R, T gm, T inv_gm1, T EPS,
                                                   T f[8])
{
    return hlld_fast_body<true>(L, R, gm, inv_gm1, EPS, f);
}

// Inputs of the FP32-bulk HLLD flux at one interface: the reconstructed
// left/right states in single precision for the wave speeds and star states,
// plus FP64 copies of the components that carry the large, balanced stresses
// (pressure, tangential B, normal B).
struct BulkStates {
    float rhoL, uL, vL, wL, rhoR, uR, vR, wR;
    double pL, pR, bYL, bYR, bZL, bZR, bn;
};

// HLLD flux of the FP32-bulk variant: the wave-speed estimates, star and
// double-star states and candidate selection of hlld.cu:256-565 in single
// precision, with the total pressure and the tangential B of every candidate
// state carried as an FP64 value plus a single-precision correction:
//   pT*  = pT_L + rdSL (pT_L - pT_R + rdSR (uR - uL)) / (rdSR - rdSL)
//   bY*L = bY_L + bY_L rdSL (SM - uL) / den*L        (and bZ, and R)
//   bY** = bY*L + (sqL (bY*R - bY*L) + sqLR (v*R - v*L) sgn bX) / (sqL + sqR)
// (algebraically the reference's formulas), so the momentum flux
// rho u^2 + pT - bX^2, rho u v - bX bY, rho u w - bX bZ is assembled in FP64
// and pressure- or tension-balanced states keep their FP64 balance.  The
// other flux components (mass, induction, energy) stay single precision.
// fm[0..2]: the three momentum components (f1, f2, f3) in FP64;
// fo[0]: f0, fo[1]: f5, fo[2]: f6, fo[3]: f7 in FP32.
//
// ONE = true forms the common case only (exactly one region, finite wave
// speeds), taking that region's state as soon as its flag is known; it
// returns false (fm, fo unwritten) where the case does not apply.  ONE =
// false forms every case.
template <bool ONE>
__device__ __forceinline__ bool hlld_bulk_body(const BulkStates &s, float gm, float inv_gm1, float EPS,
                                               double fm[3], float fo[4])
{
    const double bn64 = s.bn;
    const float bX = (float)bn64, bx2 = bX * bX;
    const double b2L64 = bn64 * bn64 + s.bYL * s.bYL + s.bZL * s.bZL;
    const double b2R64 = bn64 * bn64 + s.bYR * s.bYR + s.bZR * s.bZR;
    const double pTL64 = s.pL + 0.5 * b2L64, pTR64 = s.pR + 0.5 * b2R64;
    const float dpT = (float)(pTL64 - pTR64);
    const float pL = (float)s.pL, pR = (float)s.pR;
    const float bYL = (float)s.bYL, bYR = (float)s.bYR, bZL = (float)s.bZL, bZR = (float)s.bZR;
    // the fan's own magnetic and total pressures in single precision (the
    // FP64 ones above carry the stresses and the pressure difference)
    const float bt2L = bYL * bYL + bZL * bZL, bt2R = bYR * bYR + bZR * bZR;
    const float b2L = bx2 + bt2L, b2R = bx2 + bt2R;
    const float pTL = pL + 0.5f * b2L, pTR = pR + 0.5f * b2R;
    const float rhoL = s.rhoL, rhoR = s.rhoR, uL = s.uL, uR = s.uR, vL = s.vL, vR = s.vR, wL = s.wL, wR = s.wR;

    const float iRL = rcp_nr(rhoL), iRR = rcp_nr(rhoR);
    const float eL = pL * inv_gm1 + 0.5f * rhoL * (uL * uL + vL * vL + wL * wL) + 0.5f * b2L;
    const float eR = pR * inv_gm1 + 0.5f * rhoR * (uR * uR + vR * vR + wR * wR) + 0.5f * b2R;
    const float cs2L = gm * pL * iRL, ca2L = b2L * iRL, va2L = bx2 * iRL;
    const float cs2R = gm * pR * iRR, ca2R = b2R * iRR, va2R = bx2 * iRR;
    const float sL = cs2L + ca2L, sR = cs2R + ca2R;
    const float qnan = __int_as_float(0x7fc00000);
    const bool okL = (cs2L >= 0.f) & (ca2L >= 0.f) & (va2L >= 0.f);
    const bool okR = (cs2R >= 0.f) & (ca2R >= 0.f) & (va2R >= 0.f);
    // discriminant without cancellation, as in hlld_flux_fast
    const float dcL = cs2L - ca2L, dcR = cs2R - ca2R;
    const float discL = dcL * dcL + 4.f * cs2L * bt2L * iRL, discR = dcR * dcR + 4.f * cs2R * bt2R * iRR;
    const float cfL = okL ? sqrt_t(0.5f * (sL + sqrt_t(discL))) : qnan;
    const float cfR = okR ? sqrt_t(0.5f * (sR + sqrt_t(discR))) : qnan;

    float SL = tmin(uL, uR) - tmax(cfL, cfR);
    float SR = tmax(uL, uR) + tmax(cfL, cfR);
    SL = tmin(SL, 0.f);
    SR = tmax(SR, 0.f);

    // the selected candidate (ONE): single-precision state, FP64 total
    // pressure and tangential B
    const bool bOL = SL > 0.f, bOR = SR <= 0.f;
    float cr, cu, cv, cw, ce;
    double cpt, cby, cbz;
    if (ONE) {
        cr = bOL ? rhoL : rhoR; cu = bOL ? uL : uR; cv = bOL ? vL : vR; cw = bOL ? wL : wR; ce = 0.f;
        cpt = bOL ? pTL64 : pTR64; cby = bOL ? s.bYL : s.bYR; cbz = bOL ? s.bZL : s.bZR;
    }

    const float dSL = SL - uL, dSR = SR - uR;
    const float rdSL = rhoL * dSL, rdSR = rhoR * dSR;
    const float iden = rcp_nr(rdSR - rdSL + EPS);
    const float SM = (rdSR * uR - rdSL * uL + dpT) * iden;
    const float cpT1 = rdSL * (dpT + rdSR * (uR - uL)) * iden;      // pT* - pT_L
    const double pT1_64 = pTL64 + (double)cpT1;
    const float pT1 = pTL + cpT1;

    const float iSLM = rcp_nr(SL - SM + EPS), iSRM = rcp_nr(SR - SM + EPS);
    const float rho1L = rdSL * iSLM, rho1R = rdSR * iSRM;
    // D = rho (S - u)(S - SM) - bX^2 is a difference of two terms of order
    // bX^2.  Single precision resolves it only to about 1e-7 bX^2, so below
    // 1e-5 bX^2 the star state keeps v, w and B_t (the degenerate case of the
    // HLLD solver, Miyoshi & Kusano 2005 sec. 4.4) instead of dividing by a
    // rounding residue.
    const float DL = rdSL * (SL - SM) - bx2 + EPS, DR = rdSR * (SR - SM) - bx2 + EPS;
    const float id1L = fabsf(DL) > 1e-5f * bx2 ? rcp_nr(DL) : 0.f;
    const float id1R = fabsf(DR) > 1e-5f * bx2 ? rcp_nr(DR) : 0.f;
    const float tL = bX * (SM - uL) * id1L, tR = bX * (SM - uR) * id1R;
    const float v1L = vL - bYL * tL, w1L = wL - bZL * tL;
    const float v1R = vR - bYR * tR, w1R = wR - bZR * tR;
    const float gcL = rdSL * (SM - uL) * id1L, gcR = rdSR * (SM - uR) * id1R;   // bY*/bY - 1
    const float cYL = bYL * gcL, cZL = bZL * gcL, cYR = bYR * gcR, cZR = bZR * gcR;
    const float bY1L = bYL + cYL, bZ1L = bZL + cZL, bY1R = bYR + cYR, bZ1R = bZR + cZR;
    const float vbL = uL * bX + vL * bYL + wL * bZL, vbR = uR * bX + vR * bYR + wR * bZR;
    const float vb1L = SM * bX + v1L * bY1L + w1L * bZ1L, vb1R = SM * bX + v1R * bY1R + w1R * bZ1R;
    const float e1L = (dSL * eL - pTL * uL + pT1 * SM + bX * (vbL - vb1L)) * iSLM;
    const float e1R = (dSR * eR - pTR * uR + pT1 * SM + bX * (vbR - vb1R)) * iSRM;

    const float rsL = rsqrt_t(rho1L), rsR = rsqrt_t(rho1R);
    const float sqL = rho1L * rsL, sqR = rho1R * rsR;
    const float abx = fabsf(bX);
    const float S1L = SM - abx * rsL, S1R = SM + abx * rsR;
    const bool bML = (SL <= 0.f) && (0.f < S1L), bIL = (S1L <= 0.f) && (0.f < SM);
    const bool bMR = (S1R <= 0.f) && (0.f < SR), bIR = (SM <= 0.f) && (0.f < S1R);
    if (ONE) {
        ce = bOL ? eL : eR;
        if (bML | bMR) {
            cr = bML ? rho1L : rho1R; cu = SM; cv = bML ? v1L : v1R; cw = bML ? w1L : w1R; ce = bML ? e1L : e1R;
            cpt = pT1_64;
            cby = bML ? s.bYL + (double)cYL : s.bYR + (double)cYR;
            cbz = bML ? s.bZL + (double)cZL : s.bZR + (double)cZR;
        }
    }
    const float sb = sgn(bX);
    const float id2 = rcp_nr(sqL + sqR + EPS);
    const float sqLR = sqL * sqR;
    const float dBY = (float)(s.bYR - s.bYL) + (cYR - cYL);             // bY*R - bY*L
    const float dBZ = (float)(s.bZR - s.bZL) + (cZR - cZL);
    const float c2Y = (sqL * dBY + sqLR * (v1R - v1L) * sb) * id2;      // bY** - bY*L
    const float c2Z = (sqL * dBZ + sqLR * (w1R - w1L) * sb) * id2;
    const float v2 = (sqL * v1L + sqR * v1R + (bY1R - bY1L) * sb) * id2;
    const float w2 = (sqL * w1L + sqR * w1R + (bZ1R - bZ1L) * sb) * id2;
    const float bY2 = bY1L + c2Y, bZ2 = bZ1L + c2Z;
    const float vb2 = SM * bX + v2 * bY2 + w2 * bZ2;
    const float e2L = e1L - sqL * (vb1L - vb2) * sb;
    const float e2R = e1R + sqR * (vb1R - vb2) * sb;

    const bool ind[6] = {bOL, bML, bIL, bOR, bMR, bIR};
    const int nsel = (int)bOL + (int)bML + (int)bIL + (int)bOR + (int)bMR + (int)bIR;
    const bool nan_speed = (SL != SL) | (SR != SR) | (SM != SM) | (S1L != S1L) | (S1R != S1R);
    fm[0] = fm[1] = fm[2] = 0.0;
    fo[0] = fo[1] = fo[2] = fo[3] = 0.f;
    // FP64 momentum stresses and single-precision mass, induction and energy
    // fluxes of one candidate state
    auto add_state = [&](float rho, float u, float v, float w, float e, double pT, double by, double bz) {
        const float by32 = (float)by, bz32 = (float)bz, pT32 = (float)pT;
        const float ru = rho * u;
        fm[0] += (double)(ru * u) + pT - bn64 * bn64;
        fm[1] += (double)(ru * v) - bn64 * by;
        fm[2] += (double)(ru * w) - bn64 * bz;
        fo[0] += ru;
        fo[1] += u * by32 - v * bX;
        fo[2] += u * bz32 - w * bX;
        fo[3] += (e + pT32) * u - bX * (bX * u + by32 * v + bz32 * w);
    };
    if (ONE) {
        if (nsel != 1 || nan_speed) return false;
        if (bIL | bIR) {
            cr = bIL ? rho1L : rho1R; cu = SM; cv = v2; cw = w2; ce = bIL ? e2L : e2R; cpt = pT1_64;
            cby = s.bYL + (double)(cYL + c2Y);   // the double-star B is shared by both sides
            cbz = s.bZL + (double)(cZL + c2Z);
        }
        add_state(cr, cu, cv, cw, ce, cpt, cby, cbz);
        return true;
    }
    // candidate r: 0 outer L, 1 middle L, 2 inner L, 3 outer R, 4 middle R, 5 inner R
    auto add = [&](int r) {
        const bool lft = r < 3;
        const float rho = r == 0 ? rhoL : (r == 3 ? rhoR : (lft ? rho1L : rho1R));
        const float u = r == 0 ? uL : (r == 3 ? uR : SM);
        const float v = r == 0 ? vL : r == 3 ? vR : r == 1 ? v1L : r == 4 ? v1R : v2;
        const float w = r == 0 ? wL : r == 3 ? wR : r == 1 ? w1L : r == 4 ? w1R : w2;
        const float e = r == 0 ? eL : r == 3 ? eR : r == 1 ? e1L : r == 4 ? e1R : (r == 2 ? e2L : e2R);
        // FP64 total pressure and tangential B of the candidate
        const double pT = r == 0 ? pTL64 : (r == 3 ? pTR64 : pT1_64);
        const double by = r == 0 ? s.bYL : r == 3 ? s.bYR : r == 1 ? s.bYL + (double)cYL
                        : r == 4 ? s.bYR + (double)cYR : s.bYL + (double)(cYL + c2Y);
        const double bz = r == 0 ? s.bZL : r == 3 ? s.bZR : r == 1 ? s.bZL + (double)cZL
                        : r == 4 ? s.bZR + (double)cZR : s.bZL + (double)(cZL + c2Z);
        add_state(rho, u, v, w, e, pT, by, bz);
    };
    if (nsel == 1) {
        const int r = ind[0] ? 0 : ind[1] ? 1 : ind[2] ? 2 : ind[3] ? 3 : ind[4] ? 4 : 5;
        add(r);
    } else {
        for (int r = 0; r < 6; ++r)
            if (ind[r]) add(r);
    }
    if (nan_speed) {
        const double dn = bits_to_double(0x7FF8000000000000ull);
        fm[0] = fm[1] = fm[2] = dn;
        fo[0] = fo[1] = fo[2] = fo[3] = qnan;
    }
    return true;
}

// Every case of the FP32-bulk HLLD flux.
__device__ __forceinline__ void hlld_flux_bulk(const BulkStates &s, float gm, float inv_gm1, float EPS, double fm[3],
                                               float fo[4])
{
    hlld_bulk_body<false>(s, gm, inv_gm1, EPS, fm, fo);
}

// Its common case; false, with fm and fo unwritten, where that does not
// apply (the caller then forms the interface with hlld_flux_bulk).
__device__ __forceinline__ bool hlld_flux_bulk_sel(const BulkStates &s, float gm, float inv_gm1, float EPS,
                                                   double fm[3], float fo[4])
{
    return hlld_bulk_body<true>(s, gm, inv_gm1, EPS, fm, fo);
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

// cfl_rate with the divisions of a policy (MdDiv / IeeeDiv); ydx, ydy are
// the policy's reciprocal handles of dx and dy.
template <class Div>
__device__ __forceinline__ double cfl_rate_body(double rho, double mx, double my, double mz, double bX, double bY,
                                                double bZ, double e, double gm, double dx, double dy, double ydx,
                                                double ydy, Div &dv)
{
    const double yr = dv.recip(rho);
    const double u = dv.div(mx, rho, yr), v = dv.div(my, rho, yr), w = dv.div(mz, rho, yr);
    const double p = (gm - 1.0)
                   * (e - 0.5 * rho * (u * u + v * v + w * w)
                   - 0.5 * (bX * bX + bY * bY + bZ * bZ));
    const double cs = sqrt(dv.div(gm * p, rho, yr));
    const double ca = sqrt(dv.div(bX * bX + bY * bY + bZ * bZ, rho, yr));
    const double sx = fabs(u) + sqrt(cs * cs + ca * ca);
    const double sy = fabs(v) + sqrt(cs * cs + ca * ca);
    return dv.div(sx, dx, ydx) + dv.div(sy, dy, ydy);
}

// cfl_rate through shared reciprocals, repeated with IEEE division where the
// guard fails; ydx = rcp_rn_md(dx), ydy = rcp_rn_md(dy), d_ok their guard.
__device__ __forceinline__ double cfl_rate_md(double rho, double mx, double my, double mz, double bX, double bY,
                                              double bZ, double e, double gm, double dx, double dy, double ydx,
                                              double ydy, bool d_ok)
{
    MdDiv md;
    md.ok = d_ok;
    const double r = cfl_rate_body(rho, mx, my, mz, bX, bY, bZ, e, gm, dx, dy, ydx, ydy, md);
    if (md.ok) return r;
    IeeeDiv id;
    return cfl_rate_body(rho, mx, my, mz, bX, bY, bZ, e, gm, dx, dy, dx, dy, id);
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
