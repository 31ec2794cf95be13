/*
 * rmhd2d_tangent.cpp -- the CPU restatement of rmhd2d_oracle.c written once
 * more as a C++ template over the scalar type, so that the same step runs on
 * plain doubles and on forward-mode dual numbers (value + one directional
 * derivative).  TEST INFRASTRUCTURE ONLY: the checker for the discrete
 * adjoint of the CUDA path (rmhd2d_adjoint_backward); the product never
 * links or calls it.
 *
 * Instantiated on double it is the same arithmetic, in the same order, as
 * rmhd2d_oracle.c (which follows the reference files it names line by
 * line), and the tests hold the two bit-identical.  Instantiated on Dual it
 * gives the exact derivative of the frozen-dt step map along a direction:
 * dt of every step is given (the dts of a recorded run) instead of reduced
 * from the state, since the adjoint differentiates the step with its dt
 * held fixed.  Branches (minmod's choice, thrust::min/max, the HLLD region
 * indicators) follow the value, so the derivative is the one-sided one of
 * the branch taken, which is the subgradient the adjoint uses.  Instantiated
 * on an operation-counting scalar it gives the step's floating-point
 * operation count (the algorithm's flops per cell-update).
 *
 * Build: g++ -O2 -ffp-contract=off -fno-fast-math -fopenmp -shared -fPIC.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <omp.h>

#include <vector>

#include "rmhd2d_oracle.h"

namespace {

struct Dual {
    double v, d;
    Dual() : v(0.0), d(0.0) {}
    Dual(double x) : v(x), d(0.0) {}
    Dual(double x, double dx) : v(x), d(dx) {}
};

inline Dual operator+(Dual a, Dual b) { return Dual(a.v + b.v, a.d + b.d); }
inline Dual operator-(Dual a, Dual b) { return Dual(a.v - b.v, a.d - b.d); }
inline Dual operator-(Dual a) { return Dual(-a.v, -a.d); }
inline Dual operator*(Dual a, Dual b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
inline Dual operator/(Dual a, Dual b)
{
    const double q = a.v / b.v;
    return Dual(q, (a.d - q * b.d) / b.v);
}
inline Dual &operator+=(Dual &a, Dual b) { a = a + b; return a; }
inline Dual &operator-=(Dual &a, Dual b) { a = a - b; return a; }
inline bool operator<(Dual a, Dual b) { return a.v < b.v; }
inline bool operator>(Dual a, Dual b) { return a.v > b.v; }
inline bool operator<=(Dual a, Dual b) { return a.v <= b.v; }
inline double sqrt(double a) { return ::sqrt(a); }
inline double fabs(double a) { return ::fabs(a); }
inline Dual sqrt(Dual a)
{
    const double s = ::sqrt(a.v);
    /* sqrt'(0) * 0 is taken as 0: a zero argument with a zero tangent
       (e.g. bX = 0 in bX*bX/rho) has a zero derivative. */
    return Dual(s, a.d == 0.0 ? 0.0 : a.d / (2.0 * s));
}
inline Dual fabs(Dual a) { return a.v < 0.0 ? -a : (a.v > 0.0 ? a : Dual(0.0, 0.0)); }

/* Operation-counting scalar: a double that counts the floating-point
   operations applied to it (into g_ops; run single-threaded).  Instantiated
   on it, the step is the oracle's arithmetic with its operation count. */
struct OpCounts {
    unsigned long long add, mul, div, sqrt, abs, cmp;
};
OpCounts g_ops;

struct Counted {
    double v;
    Counted() : v(0.0) {}
    Counted(double x) : v(x) {}
};
inline Counted operator+(Counted a, Counted b) { ++g_ops.add; return Counted(a.v + b.v); }
inline Counted operator-(Counted a, Counted b) { ++g_ops.add; return Counted(a.v - b.v); }
inline Counted operator-(Counted a) { return Counted(-a.v); }
inline Counted operator*(Counted a, Counted b) { ++g_ops.mul; return Counted(a.v * b.v); }
inline Counted operator/(Counted a, Counted b) { ++g_ops.div; return Counted(a.v / b.v); }
inline Counted &operator+=(Counted &a, Counted b) { a = a + b; return a; }
inline Counted &operator-=(Counted &a, Counted b) { a = a - b; return a; }
inline bool operator<(Counted a, Counted b) { ++g_ops.cmp; return a.v < b.v; }
inline bool operator>(Counted a, Counted b) { ++g_ops.cmp; return a.v > b.v; }
inline bool operator<=(Counted a, Counted b) { ++g_ops.cmp; return a.v <= b.v; }
inline Counted sqrt(Counted a) { ++g_ops.sqrt; return Counted(::sqrt(a.v)); }
inline Counted fabs(Counted a) { ++g_ops.abs; return Counted(::fabs(a.v)); }

inline double val(double x) { return x; }
inline double val(Dual x) { return x.v; }
inline double val(Counted x) { return x.v; }

/* F * I for an HLLD indicator I in {0, 1}: the value is the reference's
   product; a candidate that is not selected contributes no derivative even
   where its own derivative is not finite. */
inline double weigh(double f, double i) { return f * i; }
inline Dual weigh(Dual f, double i) { return Dual(f.v * i, i != 0.0 ? f.d * i : 0.0); }
inline Counted weigh(Counted f, double i) { return f * Counted(i); }

enum { RHO = 0, MX = 1, MY = 2, MZ = 3, BXF = 4, BYF = 5, BZF = 6, EN = 7, NV = 8 };
enum { QR = 0, QU = 1, QV = 2, QW = 3, QBX = 4, QBY = 5, QBZ = 6, QP = 7 };

template <class T> inline T tmin(T a, T b) { return (b < a) ? b : a; }
template <class T> inline T tmax(T a, T b) { return (a < b) ? b : a; }
template <class T> inline double sgn(T x) { return (double)((val(x) > 0.0) - (val(x) < 0.0)); }

/* rmhd2d_oracle.c minmod (minmod.hpp:6-16). */
template <class T> inline T minmod(T x, T y, double eps)
{
    int s = (val(x) > 0) - (val(x) < 0);
    T ax = fabs(x);
    return T((double)s) * tmax(tmin(ax, T((double)s) * y), T(eps));
}

template <class T> void basic_param(const T *c, const T *cp, double gm, T *q)
{
    T rho = c[0];
    T u = c[1] / rho;
    T v = c[2] / rho;
    T w = c[3] / rho;
    T bX = c[4], bY = c[5], bZ = c[6], e = c[7];
    T p = T(gm - 1.0)
        * (e - T(0.5) * (rho * (u * u + v * v + w * w))
        - T(0.5) * (bX * bX + bY * bY + bZ * bZ));
    T bXPlus1 = cp[4];
    q[QR] = rho; q[QU] = u; q[QV] = v; q[QW] = w;
    q[QBX] = T(0.5) * (bX + bXPlus1);
    q[QBY] = bY; q[QBZ] = bZ; q[QP] = p;
}

static const int kComps[7] = {QR, QU, QV, QW, QBY, QBZ, QP};

template <class T> void muscl_left(const T *qm, const T *q, const T *qp, double eps, T *out)
{
    for (int n = 0; n < 7; ++n) {
        int c = kComps[n];
        out[c] = q[c] + T(0.5) * minmod(q[c] - qm[c], qp[c] - q[c], eps);
    }
    out[QBX] = q[QBX];
}

template <class T> void muscl_right(const T *q, const T *qp, const T *qpp, double eps, T *out)
{
    for (int n = 0; n < 7; ++n) {
        int c = kComps[n];
        out[c] = qp[c] - T(0.5) * minmod(qp[c] - q[c], qpp[c] - qp[c], eps);
    }
    out[QBX] = q[QBX];
}

template <class T> void one_flux(T rho, T u, T v, T w, T bX, T bY, T bZ, T e, T pT, T *f)
{
    f[0] = rho * u;
    f[1] = rho * u * u + pT - bX * bX;
    f[2] = rho * u * v - bX * bY;
    f[3] = rho * u * w - bX * bZ;
    f[4] = T(0.0);
    f[5] = u * bY - v * bX;
    f[6] = u * bZ - w * bX;
    f[7] = (e + pT) * u - bX * (bX * u + bY * v + bZ * w);
}

template <class T> void hlld_flux(const T *L, const T *R, double gmd, double EPSd, T *flux)
{
    const T gm(gmd), EPS(EPSd), half(0.5), zero(0.0), four(4.0), one(1.0);
    T rhoL = L[QR], uL = L[QU], vL = L[QV], wL = L[QW];
    T bXL = L[QBX], bYL = L[QBY], bZL = L[QBZ], pL = L[QP];
    T eL = pL / (gm - one)
         + half * rhoL * (uL * uL + vL * vL + wL * wL)
         + half * (bXL * bXL + bYL * bYL + bZL * bZL);
    T pTL = pL + half * (bXL * bXL + bYL * bYL + bZL * bZL);

    T rhoR = R[QR], uR = R[QU], vR = R[QV], wR = R[QW];
    T bXR = R[QBX], bYR = R[QBY], bZR = R[QBZ], pR = R[QP];
    T eR = pR / (gm - one)
         + half * rhoR * (uR * uR + vR * vR + wR * wR)
         + half * (bXR * bXR + bYR * bYR + bZR * bZR);
    T pTR = pR + half * (bXR * bXR + bYR * bYR + bZR * bZR);

    T csL = sqrt(gm * pL / rhoL);
    T caL = sqrt((bXL * bXL + bYL * bYL + bZL * bZL) / rhoL);
    T vaL = sqrt(bXL * bXL / rhoL);
    T cfL = sqrt(half * (csL * csL + caL * caL
          + sqrt((csL * csL + caL * caL) * (csL * csL + caL * caL)
          - four * csL * csL * vaL * vaL)));

    T csR = sqrt(gm * pR / rhoR);
    T caR = sqrt((bXR * bXR + bYR * bYR + bZR * bZR) / rhoR);
    T vaR = sqrt(bXR * bXR / rhoR);
    T cfR = sqrt(half * (csR * csR + caR * caR
          + sqrt((csR * csR + caR * caR) * (csR * csR + caR * caR)
          - four * csR * csR * vaR * vaR)));

    T SL = tmin(uL, uR) - tmax(cfL, cfR);
    T SR = tmax(uL, uR) + tmax(cfL, cfR);
    SL = tmin(SL, zero);
    SR = tmax(SR, zero);

    T SM = ((SR - uR) * rhoR * uR - (SL - uL) * rhoL * uL - pTR + pTL)
         / ((SR - uR) * rhoR - (SL - uL) * rhoL + EPS);
    T pT1 = ((SR - uR) * rhoR * pTL - (SL - uL) * rhoL * pTR
          + rhoL * rhoR * (SR - uR) * (SL - uL) * (uR - uL))
          / ((SR - uR) * rhoR - (SL - uL) * rhoL + EPS);
    T pT1L = pT1, pT1R = pT1;

    T rho1L = rhoL * (SL - uL) / (SL - SM + EPS);
    T u1L = SM;
    T v1L = vL - bXL * bYL * (SM - uL) / (rhoL * (SL - uL) * (SL - SM) - bXL * bXL + EPS);
    T w1L = wL - bXL * bZL * (SM - uL) / (rhoL * (SL - uL) * (SL - SM) - bXL * bXL + EPS);
    T bX1L = bXL;
    T bY1L = bYL * (rhoL * (SL - uL) * (SL - uL) - bXL * bXL)
           / (rhoL * (SL - uL) * (SL - SM) - bXL * bXL + EPS);
    T bZ1L = bZL * (rhoL * (SL - uL) * (SL - uL) - bXL * bXL)
           / (rhoL * (SL - uL) * (SL - SM) - bXL * bXL + EPS);
    T e1L = ((SL - uL) * eL - pTL * uL + pT1 * SM
          + bXL * ((uL * bXL + vL * bYL + wL * bZL) - (u1L * bX1L + v1L * bY1L + w1L * bZ1L)))
          / (SL - SM + EPS);

    T rho1R = rhoR * (SR - uR) / (SR - SM + EPS);
    T u1R = SM;
    T v1R = vR - bXR * bYR * (SM - uR) / (rhoR * (SR - uR) * (SR - SM) - bXR * bXR + EPS);
    T w1R = wR - bXR * bZR * (SM - uR) / (rhoR * (SR - uR) * (SR - SM) - bXR * bXR + EPS);
    T bX1R = bXR;
    T bY1R = bYR * (rhoR * (SR - uR) * (SR - uR) - bXR * bXR)
           / (rhoR * (SR - uR) * (SR - SM) - bXR * bXR + EPS);
    T bZ1R = bZR * (rhoR * (SR - uR) * (SR - uR) - bXR * bXR)
           / (rhoR * (SR - uR) * (SR - SM) - bXR * bXR + EPS);
    T e1R = ((SR - uR) * eR - pTR * uR + pT1 * SM
          + bXR * ((uR * bXR + vR * bYR + wR * bZR) - (u1R * bX1R + v1R * bY1R + w1R * bZ1R)))
          / (SR - SM + EPS);

    T S1L = SM - sqrt(bX1L * bX1L / rho1L);
    T S1R = SM + sqrt(bX1R * bX1R / rho1R);

    T rho2L = rho1L, rho2R = rho1R, u2 = SM;
    const T sb(sgn(bX1L));
    T v2 = (sqrt(rho1L) * v1L + sqrt(rho1R) * v1R + (bY1R - bY1L) * sb)
         / (sqrt(rho1L) + sqrt(rho1R) + EPS);
    T w2 = (sqrt(rho1L) * w1L + sqrt(rho1R) * w1R + (bZ1R - bZ1L) * sb)
         / (sqrt(rho1L) + sqrt(rho1R) + EPS);
    T bY2 = (sqrt(rho1L) * bY1R + sqrt(rho1R) * bY1L + sqrt(rho1L * rho1R) * (v1R - v1L) * sb)
          / (sqrt(rho1L) + sqrt(rho1R) + EPS);
    T bZ2 = (sqrt(rho1L) * bZ1R + sqrt(rho1R) * bZ1L + sqrt(rho1L * rho1R) * (w1R - w1L) * sb)
          / (sqrt(rho1L) + sqrt(rho1R) + EPS);
    T e2L = e1L - sqrt(rho1L)
          * ((u1L * bX1L + v1L * bY1L + w1L * bZ1L) - (u2 * bXL + v2 * bY2 + w2 * bZ2))
          * T(sgn(bXL));
    T e2R = e1R + sqrt(rho1R)
          * ((u1R * bX1R + v1R * bY1R + w1R * bZ1R) - (u2 * bXR + v2 * bY2 + w2 * bZ2))
          * T(sgn(bXR));
    T pT2L = pT1L, pT2R = pT1R;

    T fOL[8], fML[8], fIL[8], fOR[8], fMR[8], fIR[8];
    one_flux(rhoL, uL, vL, wL, bXL, bYL, bZL, eL, pTL, fOL);
    one_flux(rho1L, u1L, v1L, w1L, bXL, bY1L, bZ1L, e1L, pT1L, fML);
    one_flux(rho2L, u2, v2, w2, bXL, bY2, bZ2, e2L, pT2L, fIL);
    one_flux(rhoR, uR, vR, wR, bXR, bYR, bZR, eR, pTR, fOR);
    one_flux(rho1R, u1R, v1R, w1R, bXR, bY1R, bZ1R, e1R, pT1R, fMR);
    one_flux(rho2R, u2, v2, w2, bXR, bY2, bZ2, e2R, pT2R, fIR);

    double iOL = (double)(val(SL) > 0.0);
    double iML = (double)((val(SL) <= 0.0) && (0.0 < val(S1L)));
    double iIL = (double)((val(S1L) <= 0.0) && (0.0 < val(SM)));
    double iOR = (double)(val(SR) <= 0.0);
    double iMR = (double)((val(S1R) <= 0.0) && (0.0 < val(SR)));
    double iIR = (double)((val(SM) <= 0.0) && (0.0 < val(S1R)));
    for (int n = 0; n < 8; ++n) {
        flux[n] = weigh(fOL[n], iOL) + weigh(fML[n], iML) + weigh(fIL[n], iIL)
                + weigh(fOR[n], iOR) + weigh(fMR[n], iMR) + weigh(fIR[n], iIR);
    }
}

template <class T> struct Step {
    const orc_params *p;
    const T *eta;              /* nx*ny cell-centred eta (table or uniform) */
    std::vector<T> UBar, Tm, F, G, dQ, dQL, dQR, bXOld, bYOld, tmp, Ez;

    explicit Step(const orc_params *pp, const T *eta_) : p(pp), eta(eta_)
    {
        const size_t N = (size_t)p->nx * p->ny;
        UBar.resize(N * NV); Tm.resize(N * NV); F.resize(N * 8); G.resize(N * 8);
        dQ.resize(N * 8); dQL.resize(N * 8); dQR.resize(N * 8);
        bXOld.resize(N); bYOld.resize(N); tmp.resize(N); Ez.resize(N);
    }

    void flux_x(const T *Uc)
    {
        const int nx = p->nx, ny = p->ny, N = nx * ny;
        const double gm = p->gamma, EPS = p->eps;
        const T qnan(NAN);
        for (int k = 0; k < N; ++k) {
            if (k < N - ny) basic_param(&Uc[k * NV], &Uc[(k + ny) * NV], gm, &dQ[k * 8]);
            else for (int c = 0; c < 8; ++c) dQ[k * 8 + c] = qnan;
        }
#pragma omp parallel for schedule(static)
        for (int k = 0; k < N; ++k) {
            if (k >= ny && k < N - ny)
                muscl_left(&dQ[(k - ny) * 8], &dQ[k * 8], &dQ[(k + ny) * 8], EPS, &dQL[k * 8]);
            else for (int c = 0; c < 8; ++c) dQL[k * 8 + c] = qnan;
            if (k < N - 2 * ny)
                muscl_right(&dQ[k * 8], &dQ[(k + ny) * 8], &dQ[(k + 2 * ny) * 8], EPS, &dQR[k * 8]);
            else for (int c = 0; c < 8; ++c) dQR[k * 8 + c] = qnan;
        }
#pragma omp parallel for schedule(static)
        for (int k = 0; k < N; ++k) hlld_flux(&dQL[k * 8], &dQR[k * 8], gm, EPS, &F[k * 8]);

        const T two_dx(2.0 * p->dx), two_dy(2.0 * p->dy), half(0.5);
        /* written as (a - b) / (2.0 * dx) exactly as rmhd2d_oracle.c */
#pragma omp parallel for schedule(static)
        for (int i = 1; i < nx - 2; ++i) {
            for (int j = 1; j < ny - 2; ++j) {
                const T *U = Uc;
                T jY, jZ, e;
                T etaJY, etaJYPlus1, etaJZ, etaJZPlus1;
                T etaJYBZ, etaJYBZPlus1, etaJZBY, etaJZBYPlus1;
                jY = -(U[(j + (i + 1) * ny) * NV + BZF] - U[(j + (i - 1) * ny) * NV + BZF]) / two_dx;
                jZ = (U[(j + (i + 1) * ny) * NV + BYF] - U[(j + (i - 1) * ny) * NV + BYF]) / two_dx
                   - (U[(j + 1 + i * ny) * NV + BXF] - U[(j - 1 + i * ny) * NV + BXF]) / two_dy;
                e = eta[j + i * ny];
                etaJY = e * jY;
                etaJZ = e * jZ;
                etaJYBZ = etaJY * U[(j + i * ny) * NV + BZF];
                etaJZBY = etaJZ * U[(j + i * ny) * NV + BYF];

                jY = -(U[(j + (i + 2) * ny) * NV + BZF] - U[(j + i * ny) * NV + BZF]) / two_dx;
                jZ = (U[(j + (i + 2) * ny) * NV + BYF] - U[(j + i * ny) * NV + BYF]) / two_dx
                   - (U[(j + 1 + (i + 1) * ny) * NV + BXF] - U[(j - 1 + (i + 1) * ny) * NV + BXF]) / two_dy;
                e = eta[j + (i + 1) * ny];
                etaJYPlus1 = e * jY;
                etaJZPlus1 = e * jZ;
                etaJYBZPlus1 = etaJYPlus1 * U[(j + (i + 1) * ny) * NV + BZF];
                etaJZBYPlus1 = etaJZPlus1 * U[(j + (i + 1) * ny) * NV + BYF];

                T *f = &F[(j + i * ny) * 8];
                f[5] -= half * (etaJZ + etaJZPlus1);
                f[6] += half * (etaJY + etaJYPlus1);
                f[7] += half * (etaJYBZ + etaJYBZPlus1) - half * (etaJZBY + etaJZBYPlus1);
            }
        }
    }

    void flux_y(const T *Uc)
    {
        const int nx = p->nx, ny = p->ny, N = nx * ny;
        const double gm = p->gamma, EPS = p->eps;
        const T qnan(NAN);
        for (int k = 0; k < N; ++k) {
            const T *u = &Uc[k * NV];
            T *t = &Tm[k * NV];
            t[0] = u[RHO]; t[1] = u[MY]; t[2] = u[MZ]; t[3] = u[MX];
            t[4] = u[BYF]; t[5] = u[BZF]; t[6] = u[BXF]; t[7] = u[EN];
        }
        for (int k = 0; k < N; ++k) {
            if (k < N - 1) basic_param(&Tm[k * NV], &Tm[(k + 1) * NV], gm, &dQ[k * 8]);
            else for (int c = 0; c < 8; ++c) dQ[k * 8 + c] = qnan;
        }
#pragma omp parallel for schedule(static)
        for (int k = 0; k < N; ++k) {
            int j = k % ny;
            if (k >= 1 && k < N - 1 && j >= 1 && j <= ny - 2)
                muscl_left(&dQ[(k - 1) * 8], &dQ[k * 8], &dQ[(k + 1) * 8], EPS, &dQL[k * 8]);
            else for (int c = 0; c < 8; ++c) dQL[k * 8 + c] = qnan;
            if (k < N - 2 && j <= ny - 3)
                muscl_right(&dQ[k * 8], &dQ[(k + 1) * 8], &dQ[(k + 2) * 8], EPS, &dQR[k * 8]);
            else for (int c = 0; c < 8; ++c) dQR[k * 8 + c] = qnan;
        }
#pragma omp parallel for schedule(static)
        for (int k = 0; k < N; ++k) {
            T f[8];
            hlld_flux(&dQL[k * 8], &dQR[k * 8], gm, EPS, f);
            T *g = &G[k * 8];
            g[0] = f[0]; g[1] = f[3]; g[2] = f[1]; g[3] = f[2];
            g[4] = f[6]; g[5] = f[4]; g[6] = f[5]; g[7] = f[7];
        }

        const T two_dx(2.0 * p->dx), two_dy(2.0 * p->dy), half(0.5);
#pragma omp parallel for schedule(static)
        for (int i = 1; i < nx - 2; ++i) {
            for (int j = 1; j < ny - 2; ++j) {
                const T *U = Uc;
                T jX, jZ, e;
                T etaJX, etaJXPlus1, etaJZ, etaJZPlus1;
                T etaJZBX, etaJZBXPlus1, etaJXBZ, etaJXBZPlus1;
                jX = (U[(j + 1 + i * ny) * NV + BZF] - U[(j - 1 + i * ny) * NV + BZF]) / two_dy;
                jZ = (U[(j + (i + 1) * ny) * NV + BYF] - U[(j + (i - 1) * ny) * NV + BYF]) / two_dx
                   - (U[(j + 1 + i * ny) * NV + BXF] - U[(j - 1 + i * ny) * NV + BXF]) / two_dy;
                e = eta[j + i * ny];
                etaJX = e * jX;
                etaJZ = e * jZ;
                etaJXBZ = etaJX * U[(j + i * ny) * NV + BZF];
                etaJZBX = etaJZ * U[(j + i * ny) * NV + BXF];

                jX = (U[(j + 2 + i * ny) * NV + BZF] - U[(j + i * ny) * NV + BZF]) / two_dy;
                jZ = (U[(j + 1 + (i + 1) * ny) * NV + BYF] - U[(j + 1 + (i - 1) * ny) * NV + BYF]) / two_dx
                   - (U[(j + 2 + i * ny) * NV + BXF] - U[(j + i * ny) * NV + BXF]) / two_dy;
                e = eta[j + 1 + i * ny];
                etaJXPlus1 = e * jX;
                etaJZPlus1 = e * jZ;
                etaJXBZPlus1 = etaJXPlus1 * U[(j + 1 + i * ny) * NV + BZF];
                etaJZBXPlus1 = etaJZPlus1 * U[(j + 1 + i * ny) * NV + BXF];

                T *g = &G[(j + i * ny) * 8];
                g[4] += half * (etaJZ + etaJZPlus1);
                g[6] -= half * (etaJX + etaJXPlus1);
                g[7] += half * (etaJZBX + etaJZBXPlus1) - half * (etaJXBZ + etaJXBZPlus1);
            }
        }
    }

    void shift_to_center(T *U)
    {
        const int nx = p->nx, ny = p->ny, N = nx * ny;
        const T half(0.5);
        for (int k = 0; k < N; ++k) tmp[k] = U[k * NV + BXF];
        for (int i = 1; i < nx; ++i)
            for (int j = 0; j < ny; ++j)
                U[(j + i * ny) * NV + BXF] = half * (tmp[j + i * ny] + tmp[j + (i - 1) * ny]);
        for (int k = 0; k < N; ++k) tmp[k] = U[k * NV + BYF];
        for (int i = 0; i < nx; ++i)
            for (int j = 1; j < ny; ++j)
                U[(j + i * ny) * NV + BYF] = half * (tmp[j + i * ny] + tmp[j - 1 + i * ny]);
    }

    void back_to_face(T *U)
    {
        const int nx = p->nx, ny = p->ny, N = nx * ny;
        const T half(0.5);
        for (int k = 0; k < N; ++k) tmp[k] = U[k * NV + BXF];
        for (int i = 0; i < nx - 1; ++i)
            for (int j = 0; j < ny; ++j)
                U[(j + i * ny) * NV + BXF] = half * (tmp[j + i * ny] + tmp[j + (i + 1) * ny]);
        for (int k = 0; k < N; ++k) tmp[k] = U[k * NV + BYF];
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny - 1; ++j)
                U[(j + i * ny) * NV + BYF] = half * (tmp[j + i * ny] + tmp[j + 1 + i * ny]);
    }

    void corner_ez()
    {
        const int nx = p->nx, ny = p->ny;
        const T q(0.25), m1(-1.0);
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) {
                if (i < nx - 1 && j < ny - 1) {
                    T eZG1 = G[(j + i * ny) * 8 + 4];
                    T eZG2 = G[(j + (i + 1) * ny) * 8 + 4];
                    T eZF1 = m1 * F[(j + i * ny) * 8 + 5];
                    T eZF2 = m1 * F[(j + 1 + i * ny) * 8 + 5];
                    Ez[j + i * ny] = q * (eZG1 + eZG2 + eZF1 + eZF2);
                } else {
                    Ez[j + i * ny] = T(NAN);
                }
            }
    }

    void ct_update(double dt, T *U)
    {
        const int nx = p->nx, ny = p->ny;
        const T rdy(dt / p->dy), rdx(dt / p->dx);
        for (int i = 1; i < nx; ++i)
            for (int j = 1; j < ny; ++j) {
                U[(j + i * ny) * NV + BXF] = bXOld[j + i * ny] - rdy * (Ez[j + i * ny] - Ez[j - 1 + i * ny]);
                U[(j + i * ny) * NV + BYF] = bYOld[j + i * ny] + rdx * (Ez[j + i * ny] - Ez[j + (i - 1) * ny]);
            }
    }

    void periodic_x(T *U)
    {
        const int nx = p->nx, ny = p->ny;
        for (int j = 0; j < ny; ++j)
            for (int g = 0; g < 3; ++g)
                for (int f = 0; f < NV; ++f) {
                    U[(j + g * ny) * NV + f] = U[(j + (nx - 6 + g) * ny) * NV + f];
                    U[(j + (nx - 3 + g) * ny) * NV + f] = U[(j + (3 + g) * ny) * NV + f];
                }
    }

    void periodic_y(T *U)
    {
        const int nx = p->nx, ny = p->ny;
        for (int i = 0; i < nx; ++i)
            for (int g = 0; g < 3; ++g)
                for (int f = 0; f < NV; ++f) {
                    U[(g + i * ny) * NV + f] = U[(ny - 6 + g + i * ny) * NV + f];
                    U[(ny - 3 + g + i * ny) * NV + f] = U[(3 + g + i * ny) * NV + f];
                }
    }

#define C(i, j) (&U[((j) + (i) * ny) * NV])
    static void copy_except(T *dst, const T *src, int skip)
    {
        for (int f = 0; f < NV; ++f) if (f != skip) dst[f] = src[f];
    }

    void symmetric_x(T *U)
    {
        const int nx = p->nx, ny = p->ny;
        const T dx(p->dx), dy(p->dy);
        for (int j = 0; j < ny; ++j) {
            copy_except(C(0, j), C(5, j), BXF);
            copy_except(C(1, j), C(4, j), BXF);
            copy_except(C(2, j), C(3, j), BXF);
            copy_except(C(nx - 1, j), C(nx - 6, j), BXF);
            copy_except(C(nx - 2, j), C(nx - 5, j), BXF);
            copy_except(C(nx - 3, j), C(nx - 4, j), BXF);
        }
        for (int j = 0; j < ny; ++j) {
            if (0 < j) {
                C(2, j)[BXF] = C(3, j)[BXF] + (C(3, j)[BYF] - C(3, j - 1)[BYF]) / dy * dx;
                C(1, j)[BXF] = C(2, j)[BXF] + (C(2, j)[BYF] - C(2, j - 1)[BYF]) / dy * dx;
                C(0, j)[BXF] = C(1, j)[BXF] + (C(1, j)[BYF] - C(1, j - 1)[BYF]) / dy * dx;
                C(nx - 3, j)[BXF] = C(nx - 4, j)[BXF] - (C(nx - 3, j)[BYF] - C(nx - 3, j - 1)[BYF]) / dy * dx;
                C(nx - 2, j)[BXF] = C(nx - 3, j)[BXF] - (C(nx - 2, j)[BYF] - C(nx - 2, j - 1)[BYF]) / dy * dx;
                C(nx - 1, j)[BXF] = C(nx - 2, j)[BXF] - (C(nx - 1, j)[BYF] - C(nx - 1, j - 1)[BYF]) / dy * dx;
            }
            if (j == 0) {
                C(2, j)[BXF] = C(3, j)[BXF];
                C(1, j)[BXF] = C(2, j)[BXF];
                C(0, j)[BXF] = C(1, j)[BXF];
                C(nx - 3, j)[BXF] = C(nx - 4, j)[BXF];
                C(nx - 2, j)[BXF] = C(nx - 3, j)[BXF];
                C(nx - 1, j)[BXF] = C(nx - 2, j)[BXF];
            }
        }
    }

    void symmetric_y(T *U)
    {
        const int nx = p->nx, ny = p->ny;
        const T dx(p->dx), dy(p->dy);
        for (int i = 0; i < nx; ++i) {
            copy_except(C(i, 0), C(i, 5), BYF);
            copy_except(C(i, 1), C(i, 4), BYF);
            copy_except(C(i, 2), C(i, 3), BYF);
            copy_except(C(i, ny - 1), C(i, ny - 6), BYF);
            copy_except(C(i, ny - 2), C(i, ny - 5), BYF);
            copy_except(C(i, ny - 3), C(i, ny - 4), BYF);
        }
        for (int i = 0; i < nx; ++i) {
            if (0 < i) {
                C(i, 2)[BYF] = C(i, 3)[BYF] + (C(i, 3)[BXF] - C(i - 1, 3)[BXF]) / dx * dy;
                C(i, 1)[BYF] = C(i, 2)[BYF] + (C(i, 2)[BXF] - C(i - 1, 2)[BXF]) / dx * dy;
                C(i, 0)[BYF] = C(i, 1)[BYF] + (C(i, 1)[BXF] - C(i - 1, 1)[BXF]) / dx * dy;
                C(i, ny - 3)[BYF] = C(i, ny - 4)[BYF] - (C(i, ny - 3)[BXF] - C(i - 1, ny - 3)[BXF]) / dx * dy;
                C(i, ny - 2)[BYF] = C(i, ny - 3)[BYF] - (C(i, ny - 2)[BXF] - C(i - 1, ny - 2)[BXF]) / dx * dy;
                C(i, ny - 1)[BYF] = C(i, ny - 2)[BYF] - (C(i, ny - 1)[BXF] - C(i - 1, ny - 1)[BXF]) / dx * dy;
            }
            if (i == 0) {
                C(i, 2)[BYF] = C(i, 3)[BYF];
                C(i, 1)[BYF] = C(i, 2)[BYF];
                C(i, 0)[BYF] = C(i, 1)[BYF];
                C(i, ny - 3)[BYF] = C(i, ny - 4)[BYF];
                C(i, ny - 2)[BYF] = C(i, ny - 3)[BYF];
                C(i, ny - 1)[BYF] = C(i, ny - 2)[BYF];
            }
        }
    }
#undef C

    void boundary(T *U)
    {
        const int bcy = p->bc_y < 0 ? p->bc : p->bc_y;
        if (p->bc == ORC_BC_SYMMETRIC) symmetric_x(U);
        else periodic_x(U);
        if (bcy == ORC_BC_SYMMETRIC) symmetric_y(U);
        else periodic_y(U);
    }

    /* rmhd2d_oracle.c orc_step with the step's dt given. */
    void step(T *U, double dt)
    {
        const int nx = p->nx, ny = p->ny, N = nx * ny;
        for (int k = 0; k < N; ++k) { bXOld[k] = U[k * NV + BXF]; bYOld[k] = U[k * NV + BYF]; }
        for (size_t k = 0; k < (size_t)N * NV; ++k) UBar[k] = U[k];
        const T rdx(dt / p->dx), rdy(dt / p->dy), half(0.5);

        shift_to_center(U);
        flux_x(U);
        flux_y(U);
        back_to_face(U);
#pragma omp parallel for schedule(static)
        for (int k = ny; k < N; ++k) {
            const T *u = &U[k * NV];
            const T *f = &F[k * 8], *fm = &F[(k - ny) * 8];
            const T *g = &G[k * 8], *gmm = &G[(k - 1) * 8];
            T *ub = &UBar[k * NV];
            for (int c = 0; c < 8; ++c)
                ub[c] = u[c] - rdx * (f[c] - fm[c]) - rdy * (g[c] - gmm[c]);
        }
        corner_ez();
        ct_update(dt, UBar.data());
        boundary(UBar.data());

        shift_to_center(UBar.data());
        flux_x(UBar.data());
        flux_y(UBar.data());
        back_to_face(UBar.data());
#pragma omp parallel for schedule(static)
        for (int k = ny; k < N; ++k) {
            T *u = &U[k * NV];
            const T *ub = &UBar[k * NV];
            const T *f = &F[k * 8], *fm = &F[(k - ny) * 8];
            const T *g = &G[k * 8], *gmm = &G[(k - 1) * 8];
            for (int c = 0; c < 8; ++c)
                u[c] = half * (u[c] + ub[c]
                     - rdx * (f[c] - fm[c])
                     - rdy * (g[c] - gmm[c]));
        }
        ct_update(dt, U);
        boundary(U);
    }
};

}  // namespace

extern "C" {

/* nsteps steps with the given dts from U (boundary applied first when
   apply_boundary != 0), in doubles.  Returns 0. */
int orc_run_fixed_dt(const orc_params *p, double *U, int nsteps, const double *dts, int apply_boundary)
{
    const size_t N = (size_t)p->nx * p->ny;
    std::vector<double> eta(N);
    for (size_t k = 0; k < N; ++k) eta[k] = p->eta_table ? p->eta_table[k] : p->eta;
    Step<double> st(p, eta.data());
    if (apply_boundary) st.boundary(U);
    for (int s = 0; s < nsteps; ++s) st.step(U, dts[s]);
    return 0;
}

/* Tangent of the frozen-dt map U0 -> U_N along (dU0, deta): U0 and dU0
   (nx*ny*8, reference layout) are taken before the boundary, which is
   applied first as the reference drivers' initializeU does; deta (nx*ny,
   may be NULL) perturbs the cell-centred eta field (the table when one is
   set, else the uniform eta).  Writes U_N into U and dU_N into dU. */
int orc_tangent_run(const orc_params *p, double *U, double *dU, const double *deta, int nsteps,
                    const double *dts)
{
    const size_t N = (size_t)p->nx * p->ny;
    std::vector<Dual> eta(N), S(N * NV);
    for (size_t k = 0; k < N; ++k) eta[k] = Dual(p->eta_table ? p->eta_table[k] : p->eta, deta ? deta[k] : 0.0);
    for (size_t k = 0; k < N * NV; ++k) S[k] = Dual(U[k], dU[k]);
    Step<Dual> st(p, eta.data());
    st.boundary(S.data());
    for (int s = 0; s < nsteps; ++s) st.step(S.data(), dts[s]);
    for (size_t k = 0; k < N * NV; ++k) { U[k] = S[k].v; dU[k] = S[k].d; }
    return 0;
}

/* nsteps steps with the given dts from U (boundary applied first when
   apply_boundary != 0), on the operation-counting scalar, single-threaded:
   U_N is written back into U and the operation counts into counts[6] =
   {add/sub, mul, div, sqrt, abs, compare}, summed over the whole array
   (ghost cells included) and all steps. */
int orc_count_ops(const orc_params *p, double *U, int nsteps, const double *dts, int apply_boundary,
                  unsigned long long *counts)
{
    const size_t N = (size_t)p->nx * p->ny;
    const int threads = omp_get_max_threads();
    omp_set_num_threads(1);
    std::vector<Counted> eta(N), S(N * NV);
    for (size_t k = 0; k < N; ++k) eta[k] = Counted(p->eta_table ? p->eta_table[k] : p->eta);
    for (size_t k = 0; k < N * NV; ++k) S[k] = Counted(U[k]);
    g_ops = OpCounts{0, 0, 0, 0, 0, 0};
    {
        Step<Counted> st(p, eta.data());
        if (apply_boundary) st.boundary(S.data());
        for (int s = 0; s < nsteps; ++s) st.step(S.data(), dts[s]);
    }
    for (size_t k = 0; k < N * NV; ++k) U[k] = S[k].v;
    counts[0] = g_ops.add; counts[1] = g_ops.mul; counts[2] = g_ops.div;
    counts[3] = g_ops.sqrt; counts[4] = g_ops.abs; counts[5] = g_ops.cmp;
    omp_set_num_threads(threads);
    return 0;
}

/* One interface of the HLLD solver on dual numbers: the flux f and its
   derivative df along (dL, dR) for primitive states L, R (rho, u, v, w, bX,
   bY, bZ, p).  Used to check the adjoint of a single interface. */
void orc_hlld_jvp(const double *L, const double *R, const double *dL, const double *dR, double gamma, double eps,
                  double *f, double *df)
{
    Dual l[8], r[8], o[8];
    for (int c = 0; c < 8; ++c) { l[c] = Dual(L[c], dL[c]); r[c] = Dual(R[c], dR[c]); }
    hlld_flux(l, r, gamma, eps, o);
    for (int c = 0; c < 8; ++c) { f[c] = o[c].v; df[c] = o[c].d; }
}

}  // extern "C"
