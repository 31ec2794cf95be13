/*
 * rmhd2d_oracle.c -- CPU restatement of one RK2 step of the 2D resistive-MHD
 * solver in keita-akutagawa/ResistiveMHD_GPU (single-GPU Thrust library).
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the CUDA
 * path in resistivemhd_gpu_b200/.  Only tests/, __graft_entry__.smoke() and
 * the cpu_baseline / reference legs of bench.py may load it.  The product
 * never links or calls it.
 *
 * It restates, operation by operation and in the same evaluation order, the
 * arithmetic of these reference files (paths inside the reference project):
 *
 *   ResistiveMHD_singleGPU_thrust/lib_ResistiveMHD_2D_GPU_periodicXY/
 *     resistiveMHD_2D.cu:133-195   oneStepRK2 (stage order, CT reuse)
 *     resistiveMHD_2D.cu:53-130    oneStepFirst/SecondFunctor (update)
 *     resistiveMHD_2D.cu:247-291   calculateDtFunctor / calculateDt
 *     resistiveMHD_2D.cu:294-309   IsNan / checkCalculationIsCrashed
 *     resistiveMHD_2D.cu:313-426   shift/back B to centre for CT
 *     calculate_half_Q.cu:4-67     GetBasicParamterFunctor (primitives)
 *     muscl.cu:6-126, minmod.hpp   MUSCL-minmod interface states
 *     hlld.cu:26-131, 134-233      Sign, CalculateFluxFunctor, y-sweep shuffles
 *     hlld.cu:256-444              calculateHLLDParameterFunctor
 *     hlld.cu:448-565              getOneFlux / setFluxFunctor
 *     ct.cu:22-85                  getEZVector_kernel, CT_kernel
 *     boundary.cu:4-141            periodicBoundaryX2nd / Y2nd
 *   .../lib_ResistiveMHD_2D_GPU_symmetricXY/boundary.cu:4-206
 *                                  symmetricBoundaryX2nd(+BX) / Y2nd(+BY)
 *   ResistiveMHD_singleGPU_thrust/examples2D/plasmoid/main_plasmoid.cu:175-290
 *                                  addResistiveTermToFluxF/G (driver hook)
 *
 * State layout is the reference's: an array of nx*ny cells, cell k = j + i*ny
 * (y fastest), each cell 8 doubles {rho, rhoU, rhoV, rhoW, bX, bY, bZ, e}.
 * nx, ny include 3 ghost layers per side.  bX of cell (i,j) is the x-face
 * value at x_{i+1/2}; bY is the y-face value at y_{j+1/2}.
 *
 * Build with -ffp-contract=off (no fused multiply-add) so every operation is
 * one IEEE-754 binary64 operation, exactly as the reference's host build on
 * x86-64 (SSE2) evaluates it.
 *
 * Where the reference reads buffer entries that the current call did not
 * write (e.g. dQCenter at i = nx-1 in the x sweep, flat-index wrap in the y
 * sweep), this restatement writes NaN instead.  Those entries only feed
 * ghost cells that the boundary pass overwrites, so a finite final state
 * is a check that no such value reaches the result.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "rmhd2d_oracle.h"

enum { RHO = 0, MX = 1, MY = 2, MZ = 3, BXF = 4, BYF = 5, BZF = 6, EN = 7, NV = 8 };

/* BasicParameter field order: rho, u, v, w, bX, bY, bZ, p
   (basic_parameter_struct.hpp:5-27). */
enum { QR = 0, QU = 1, QV = 2, QW = 3, QBX = 4, QBY = 5, QBZ = 6, QP = 7 };

/* thrust::min / thrust::max semantics: min(a,b) = (b < a) ? b : a. */
static inline double tmin(double a, double b) { return (b < a) ? b : a; }
static inline double tmax(double a, double b) { return (a < b) ? b : a; }

/* hlld.cu:26-32 Sign: (x > 0) - (x < 0) as double. */
static inline double sgn(double x) { return (double)((x > 0.0) - (x < 0.0)); }

/* minmod.hpp:6-16: sign_x * max(min(|x|, sign_x*y), EPS), sign_x an int. */
static inline double minmod(double x, double y, double eps)
{
    int s = (x > 0) - (x < 0);
    double ax = fabs(x);
    return (double)s * tmax(tmin(ax, (double)s * y), eps);
}

/* calculate_half_Q.cu:4-38 GetBasicParamterFunctor on a cell c and its
   neighbour cp along the sweep.  c points at 8 doubles in sweep order
   (rho, rhoU, rhoV, rhoW, bX, bY, bZ, e). */
static void basic_param(const double *c, const double *cp, double gm, double *q)
{
    double rho = c[0];
    double u = c[1] / rho;
    double v = c[2] / rho;
    double w = c[3] / rho;
    double bX = c[4], bY = c[5], bZ = c[6], e = c[7];
    double p = (gm - 1.0)
             * (e - 0.5 * (rho * (u * u + v * v + w * w))
             - 0.5 * (bX * bX + bY * bY + bZ * bZ));
    double bXPlus1 = cp[4];
    q[QR] = rho; q[QU] = u; q[QV] = v; q[QW] = w;
    q[QBX] = 0.5 * (bX + bXPlus1);
    q[QBY] = bY; q[QBZ] = bZ; q[QP] = p;
}

/* muscl.cu:6-30 LeftParameterFunctor. */
static void muscl_left(const double *qm, const double *q, const double *qp, double eps, double *out)
{
    static const int comps[7] = {QR, QU, QV, QW, QBY, QBZ, QP};
    for (int n = 0; n < 7; ++n) {
        int c = comps[n];
        out[c] = q[c] + 0.5 * minmod(q[c] - qm[c], qp[c] - q[c], eps);
    }
    out[QBX] = q[QBX];
}

/* muscl.cu:66-90 RightParameterFunctor (q at k, qp at k+off, qpp at k+2off). */
static void muscl_right(const double *q, const double *qp, const double *qpp, double eps, double *out)
{
    static const int comps[7] = {QR, QU, QV, QW, QBY, QBZ, QP};
    for (int n = 0; n < 7; ++n) {
        int c = comps[n];
        out[c] = qp[c] - 0.5 * minmod(qp[c] - q[c], qpp[c] - qp[c], eps);
    }
    out[QBX] = q[QBX];
}

/* hlld.cu:448-467 getOneFlux. */
static void one_flux(double rho, double u, double v, double w, double bX, double bY,
                     double bZ, double e, double pT, double *f)
{
    f[0] = rho * u;
    f[1] = rho * u * u + pT - bX * bX;
    f[2] = rho * u * v - bX * bY;
    f[3] = rho * u * w - bX * bZ;
    f[4] = 0.0;
    f[5] = u * bY - v * bX;
    f[6] = u * bZ - w * bX;
    f[7] = (e + pT) * u - bX * (bX * u + bY * v + bZ * w);
}

/* hlld.cu:256-432 calculateHLLDParameterFunctor, hlld.cu:469-549
   setFluxFunctor and hlld.cu:35-107 CalculateFluxFunctor, fused: all six
   candidate fluxes are formed and summed with the reference's indicator
   weights, so non-finite candidates propagate as they do there. */
static void hlld_flux(const double *L, const double *R, double gm, double EPS, double *flux)
{
    double rhoL = L[QR], uL = L[QU], vL = L[QV], wL = L[QW];
    double bXL = L[QBX], bYL = L[QBY], bZL = L[QBZ], pL = L[QP];
    double eL = pL / (gm - 1.0)
              + 0.5 * rhoL * (uL * uL + vL * vL + wL * wL)
              + 0.5 * (bXL * bXL + bYL * bYL + bZL * bZL);
    double pTL = pL + 0.5 * (bXL * bXL + bYL * bYL + bZL * bZL);

    double rhoR = R[QR], uR = R[QU], vR = R[QV], wR = R[QW];
    double bXR = R[QBX], bYR = R[QBY], bZR = R[QBZ], pR = R[QP];
    double eR = pR / (gm - 1.0)
              + 0.5 * rhoR * (uR * uR + vR * vR + wR * wR)
              + 0.5 * (bXR * bXR + bYR * bYR + bZR * bZR);
    double pTR = pR + 0.5 * (bXR * bXR + bYR * bYR + bZR * bZR);

    double csL = sqrt(gm * pL / rhoL);
    double caL = sqrt((bXL * bXL + bYL * bYL + bZL * bZL) / rhoL);
    double vaL = sqrt(bXL * bXL / rhoL);
    double cfL = sqrt(0.5 * (csL * csL + caL * caL
               + sqrt((csL * csL + caL * caL) * (csL * csL + caL * caL)
               - 4.0 * csL * csL * vaL * vaL)));

    double csR = sqrt(gm * pR / rhoR);
    double caR = sqrt((bXR * bXR + bYR * bYR + bZR * bZR) / rhoR);
    double vaR = sqrt(bXR * bXR / rhoR);
    double cfR = sqrt(0.5 * (csR * csR + caR * caR
               + sqrt((csR * csR + caR * caR) * (csR * csR + caR * caR)
               - 4.0 * csR * csR * vaR * vaR)));

    double SL = tmin(uL, uR) - tmax(cfL, cfR);
    double SR = tmax(uL, uR) + tmax(cfL, cfR);
    SL = tmin(SL, 0.0);
    SR = tmax(SR, 0.0);

    double SM = ((SR - uR) * rhoR * uR - (SL - uL) * rhoL * uL - pTR + pTL)
              / ((SR - uR) * rhoR - (SL - uL) * rhoL + EPS);
    double pT1 = ((SR - uR) * rhoR * pTL - (SL - uL) * rhoL * pTR
               + rhoL * rhoR * (SR - uR) * (SL - uL) * (uR - uL))
               / ((SR - uR) * rhoR - (SL - uL) * rhoL + EPS);
    double pT1L = pT1, pT1R = pT1;

    double rho1L = rhoL * (SL - uL) / (SL - SM + EPS);
    double u1L = SM;
    double v1L = vL - bXL * bYL * (SM - uL) / (rhoL * (SL - uL) * (SL - SM) - bXL * bXL + EPS);
    double w1L = wL - bXL * bZL * (SM - uL) / (rhoL * (SL - uL) * (SL - SM) - bXL * bXL + EPS);
    double bX1L = bXL;
    double bY1L = bYL * (rhoL * (SL - uL) * (SL - uL) - bXL * bXL)
                / (rhoL * (SL - uL) * (SL - SM) - bXL * bXL + EPS);
    double bZ1L = bZL * (rhoL * (SL - uL) * (SL - uL) - bXL * bXL)
                / (rhoL * (SL - uL) * (SL - SM) - bXL * bXL + EPS);
    double e1L = ((SL - uL) * eL - pTL * uL + pT1 * SM
               + bXL * ((uL * bXL + vL * bYL + wL * bZL) - (u1L * bX1L + v1L * bY1L + w1L * bZ1L)))
               / (SL - SM + EPS);

    double rho1R = rhoR * (SR - uR) / (SR - SM + EPS);
    double u1R = SM;
    double v1R = vR - bXR * bYR * (SM - uR) / (rhoR * (SR - uR) * (SR - SM) - bXR * bXR + EPS);
    double w1R = wR - bXR * bZR * (SM - uR) / (rhoR * (SR - uR) * (SR - SM) - bXR * bXR + EPS);
    double bX1R = bXR;
    double bY1R = bYR * (rhoR * (SR - uR) * (SR - uR) - bXR * bXR)
                / (rhoR * (SR - uR) * (SR - SM) - bXR * bXR + EPS);
    double bZ1R = bZR * (rhoR * (SR - uR) * (SR - uR) - bXR * bXR)
                / (rhoR * (SR - uR) * (SR - SM) - bXR * bXR + EPS);
    double e1R = ((SR - uR) * eR - pTR * uR + pT1 * SM
               + bXR * ((uR * bXR + vR * bYR + wR * bZR) - (u1R * bX1R + v1R * bY1R + w1R * bZ1R)))
               / (SR - SM + EPS);

    double S1L = SM - sqrt(bX1L * bX1L / rho1L);
    double S1R = SM + sqrt(bX1R * bX1R / rho1R);

    double rho2L = rho1L, rho2R = rho1R, u2 = SM;
    double v2 = (sqrt(rho1L) * v1L + sqrt(rho1R) * v1R + (bY1R - bY1L) * sgn(bX1L))
              / (sqrt(rho1L) + sqrt(rho1R) + EPS);
    double w2 = (sqrt(rho1L) * w1L + sqrt(rho1R) * w1R + (bZ1R - bZ1L) * sgn(bX1L))
              / (sqrt(rho1L) + sqrt(rho1R) + EPS);
    double bY2 = (sqrt(rho1L) * bY1R + sqrt(rho1R) * bY1L + sqrt(rho1L * rho1R) * (v1R - v1L) * sgn(bX1L))
               / (sqrt(rho1L) + sqrt(rho1R) + EPS);
    double bZ2 = (sqrt(rho1L) * bZ1R + sqrt(rho1R) * bZ1L + sqrt(rho1L * rho1R) * (w1R - w1L) * sgn(bX1L))
               / (sqrt(rho1L) + sqrt(rho1R) + EPS);
    double e2L = e1L - sqrt(rho1L)
               * ((u1L * bX1L + v1L * bY1L + w1L * bZ1L) - (u2 * bXL + v2 * bY2 + w2 * bZ2))
               * sgn(bXL);
    double e2R = e1R + sqrt(rho1R)
               * ((u1R * bX1R + v1R * bY1R + w1R * bZ1R) - (u2 * bXR + v2 * bY2 + w2 * bZ2))
               * sgn(bXR);
    double pT2L = pT1L, pT2R = pT1R;

    double fOL[8], fML[8], fIL[8], fOR[8], fMR[8], fIR[8];
    one_flux(rhoL, uL, vL, wL, bXL, bYL, bZL, eL, pTL, fOL);
    one_flux(rho1L, u1L, v1L, w1L, bXL, bY1L, bZ1L, e1L, pT1L, fML);
    one_flux(rho2L, u2, v2, w2, bXL, bY2, bZ2, e2L, pT2L, fIL);
    one_flux(rhoR, uR, vR, wR, bXR, bYR, bZR, eR, pTR, fOR);
    one_flux(rho1R, u1R, v1R, w1R, bXR, bY1R, bZ1R, e1R, pT1R, fMR);
    one_flux(rho2R, u2, v2, w2, bXR, bY2, bZ2, e2R, pT2R, fIR);

    double iOL = (double)(SL > 0.0);
    double iML = (double)((SL <= 0.0) && (0.0 < S1L));
    double iIL = (double)((S1L <= 0.0) && (0.0 < SM));
    double iOR = (double)(SR <= 0.0);
    double iMR = (double)((S1R <= 0.0) && (0.0 < SR));
    double iIR = (double)((SM <= 0.0) && (0.0 < S1R));
    for (int n = 0; n < 8; ++n) {
        flux[n] = fOL[n] * iOL + fML[n] * iML + fIL[n] * iIL
                + fOR[n] * iOR + fMR[n] * iMR + fIR[n] * iIR;
    }
}

/* eta at cell (i,j): the driver's getEta.  A table (cell-centred, k = j +
   i*ny) when given, else the uniform value. */
static inline double eta_at(const orc_params *p, int i, int j)
{
    return p->eta_table ? p->eta_table[j + i * p->ny] : p->eta;
}

/* x-direction flux F at interface i+1/2 of every cell (HLLD::calculateFluxF,
   hlld.cu:110-131, + resistive hook main_plasmoid.cu:175-215).  Uc is the
   state with cell-centred B. */
static void flux_x(const orc_params *p, const double *Uc, double *F, double *dQ,
                   double *dQL, double *dQR)
{
    const int nx = p->nx, ny = p->ny, N = nx * ny;
    const double gm = p->gamma, EPS = p->eps;
    const double qnan = NAN;

    /* setPhysicalParameterX: k in [0, N - ny); entries at i = nx-1 stale. */
    for (int k = 0; k < N; ++k) {
        if (k < N - ny) basic_param(&Uc[k * NV], &Uc[(k + ny) * NV], gm, &dQ[k * 8]);
        else for (int c = 0; c < 8; ++c) dQ[k * 8 + c] = qnan;
    }
    /* getLeftQX: k in [ny, N - ny). getRightQX: k in [0, N - 2ny). */
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

    /* addResistiveTermToFluxF: 0 < i < nx-2, 0 < j < ny-2, U = Uc. */
    const double dx = p->dx, dy = p->dy;
    #pragma omp parallel for schedule(static)
    for (int i = 1; i < nx - 2; ++i) {
        for (int j = 1; j < ny - 2; ++j) {
            const double *U = Uc;
            double jY, jZ, eta;
            double etaJY, etaJYPlus1, etaJZ, etaJZPlus1;
            double etaJYBZ, etaJYBZPlus1, etaJZBY, etaJZBYPlus1;
            jY = -(U[(j + (i + 1) * ny) * NV + BZF] - U[(j + (i - 1) * ny) * NV + BZF]) / (2.0 * dx);
            jZ = (U[(j + (i + 1) * ny) * NV + BYF] - U[(j + (i - 1) * ny) * NV + BYF]) / (2.0 * dx)
               - (U[(j + 1 + i * ny) * NV + BXF] - U[(j - 1 + i * ny) * NV + BXF]) / (2.0 * dy);
            eta = eta_at(p, i, j);
            etaJY = eta * jY;
            etaJZ = eta * jZ;
            etaJYBZ = etaJY * U[(j + i * ny) * NV + BZF];
            etaJZBY = etaJZ * U[(j + i * ny) * NV + BYF];

            jY = -(U[(j + (i + 2) * ny) * NV + BZF] - U[(j + i * ny) * NV + BZF]) / (2.0 * dx);
            jZ = (U[(j + (i + 2) * ny) * NV + BYF] - U[(j + i * ny) * NV + BYF]) / (2.0 * dx)
               - (U[(j + 1 + (i + 1) * ny) * NV + BXF] - U[(j - 1 + (i + 1) * ny) * NV + BXF]) / (2.0 * dy);
            eta = eta_at(p, i + 1, j);
            etaJYPlus1 = eta * jY;
            etaJZPlus1 = eta * jZ;
            etaJYBZPlus1 = etaJYPlus1 * U[(j + (i + 1) * ny) * NV + BZF];
            etaJZBYPlus1 = etaJZPlus1 * U[(j + (i + 1) * ny) * NV + BYF];

            double *f = &F[(j + i * ny) * 8];
            f[5] -= 0.5 * (etaJZ + etaJZPlus1);
            f[6] += 0.5 * (etaJY + etaJYPlus1);
            f[7] += 0.5 * (etaJYBZ + etaJYBZPlus1) - 0.5 * (etaJZBY + etaJZBYPlus1);
        }
    }
}

/* y-direction flux G at interface j+1/2 (HLLD::calculateFluxG,
   hlld.cu:134-233, + resistive hook main_plasmoid.cu:234-274).  The y sweep
   runs the x-sweep arithmetic on the permuted cell
   (rho, rhoV, rhoW, rhoU, bY, bZ, bX, e) and un-permutes the flux. */
static void flux_y(const orc_params *p, const double *Uc, double *G, double *T,
                   double *dQ, double *dQL, double *dQR)
{
    const int nx = p->nx, ny = p->ny, N = nx * ny;
    const double gm = p->gamma, EPS = p->eps;
    const double qnan = NAN;

    /* shuffleForTmpUForFluxG_kernel */
    for (int k = 0; k < N; ++k) {
        const double *u = &Uc[k * NV];
        double *t = &T[k * NV];
        t[0] = u[RHO]; t[1] = u[MY]; t[2] = u[MZ]; t[3] = u[MX];
        t[4] = u[BYF]; t[5] = u[BZF]; t[6] = u[BXF]; t[7] = u[EN];
    }
    /* setPhysicalParameterY: k in [0, N-1). */
    for (int k = 0; k < N; ++k) {
        if (k < N - 1) basic_param(&T[k * NV], &T[(k + 1) * NV], gm, &dQ[k * 8]);
        else for (int c = 0; c < 8; ++c) dQ[k * 8 + c] = qnan;
    }
    /* getLeftQY: k in [1, N-1).  getRightQY: k in [0, N-2).  Entries that
       wrap across a column (j = 0 or j >= ny-2) mix neighbouring columns in
       the reference; they are poisoned here. */
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
        double f[8];
        hlld_flux(&dQL[k * 8], &dQR[k * 8], gm, EPS, f);
        /* shuffleForFluxG_kernel: f1<-f3, f2<-f1, f3<-f2, f4<-f6, f5<-f4, f6<-f5 */
        double *g = &G[k * 8];
        g[0] = f[0]; g[1] = f[3]; g[2] = f[1]; g[3] = f[2];
        g[4] = f[6]; g[5] = f[4]; g[6] = f[5]; g[7] = f[7];
    }

    const double dx = p->dx, dy = p->dy;
    #pragma omp parallel for schedule(static)
    for (int i = 1; i < nx - 2; ++i) {
        for (int j = 1; j < ny - 2; ++j) {
            const double *U = Uc;
            double jX, jZ, eta;
            double etaJX, etaJXPlus1, etaJZ, etaJZPlus1;
            double etaJZBX, etaJZBXPlus1, etaJXBZ, etaJXBZPlus1;
            jX = (U[(j + 1 + i * ny) * NV + BZF] - U[(j - 1 + i * ny) * NV + BZF]) / (2.0 * dy);
            jZ = (U[(j + (i + 1) * ny) * NV + BYF] - U[(j + (i - 1) * ny) * NV + BYF]) / (2.0 * dx)
               - (U[(j + 1 + i * ny) * NV + BXF] - U[(j - 1 + i * ny) * NV + BXF]) / (2.0 * dy);
            eta = eta_at(p, i, j);
            etaJX = eta * jX;
            etaJZ = eta * jZ;
            etaJXBZ = etaJX * U[(j + i * ny) * NV + BZF];
            etaJZBX = etaJZ * U[(j + i * ny) * NV + BXF];

            jX = (U[(j + 2 + i * ny) * NV + BZF] - U[(j + i * ny) * NV + BZF]) / (2.0 * dy);
            jZ = (U[(j + 1 + (i + 1) * ny) * NV + BYF] - U[(j + 1 + (i - 1) * ny) * NV + BYF]) / (2.0 * dx)
               - (U[(j + 2 + i * ny) * NV + BXF] - U[(j + i * ny) * NV + BXF]) / (2.0 * dy);
            eta = eta_at(p, i, j + 1);
            etaJXPlus1 = eta * jX;
            etaJZPlus1 = eta * jZ;
            etaJXBZPlus1 = etaJXPlus1 * U[(j + 1 + i * ny) * NV + BZF];
            etaJZBXPlus1 = etaJZPlus1 * U[(j + 1 + i * ny) * NV + BXF];

            double *g = &G[(j + i * ny) * 8];
            g[4] += 0.5 * (etaJZ + etaJZPlus1);
            g[6] -= 0.5 * (etaJX + etaJXPlus1);
            g[7] += 0.5 * (etaJZBX + etaJZBXPlus1) - 0.5 * (etaJXBZ + etaJXBZPlus1);
        }
    }
}

/* resistiveMHD_2D.cu:313-368 shiftUToCenterForCT, in place. */
static void shift_to_center(const orc_params *p, double *U, double *tmp)
{
    const int nx = p->nx, ny = p->ny, N = nx * ny;
    for (int k = 0; k < N; ++k) tmp[k] = U[k * NV + BXF];
    for (int i = 1; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            U[(j + i * ny) * NV + BXF] = 0.5 * (tmp[j + i * ny] + tmp[j + (i - 1) * ny]);
    for (int k = 0; k < N; ++k) tmp[k] = U[k * NV + BYF];
    for (int i = 0; i < nx; ++i)
        for (int j = 1; j < ny; ++j)
            U[(j + i * ny) * NV + BYF] = 0.5 * (tmp[j + i * ny] + tmp[j - 1 + i * ny]);
}

/* resistiveMHD_2D.cu:371-426 backUToCenterHalfForCT, in place. */
static void back_to_face(const orc_params *p, double *U, double *tmp)
{
    const int nx = p->nx, ny = p->ny, N = nx * ny;
    for (int k = 0; k < N; ++k) tmp[k] = U[k * NV + BXF];
    for (int i = 0; i < nx - 1; ++i)
        for (int j = 0; j < ny; ++j)
            U[(j + i * ny) * NV + BXF] = 0.5 * (tmp[j + i * ny] + tmp[j + (i + 1) * ny]);
    for (int k = 0; k < N; ++k) tmp[k] = U[k * NV + BYF];
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny - 1; ++j)
            U[(j + i * ny) * NV + BYF] = 0.5 * (tmp[j + i * ny] + tmp[j + 1 + i * ny]);
}

/* ct.cu:22-41 getEZVector_kernel: corner Ez for i < nx-1, j < ny-1; the
   reference never writes the last row/column of eZVector (zero-initialised
   there), which only reaches ghost faces. */
static void corner_ez(const orc_params *p, const double *F, const double *G, double *Ez)
{
    const int nx = p->nx, ny = p->ny;
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) {
            if (i < nx - 1 && j < ny - 1) {
                double eZG1 = G[(j + i * ny) * 8 + 4];
                double eZG2 = G[(j + (i + 1) * ny) * 8 + 4];
                double eZF1 = -1.0 * F[(j + i * ny) * 8 + 5];
                double eZF2 = -1.0 * F[(j + 1 + i * ny) * 8 + 5];
                Ez[j + i * ny] = 0.25 * (eZG1 + eZG2 + eZF1 + eZF2);
            } else {
                Ez[j + i * ny] = NAN;
            }
        }
}

/* ct.cu:44-59 CT_kernel. */
static void ct_update(const orc_params *p, const double *bXOld, const double *bYOld,
                      const double *Ez, double dt, double *U)
{
    const int nx = p->nx, ny = p->ny;
    for (int i = 1; i < nx; ++i)
        for (int j = 1; j < ny; ++j) {
            U[(j + i * ny) * NV + BXF] = bXOld[j + i * ny]
                - dt / p->dy * (Ez[j + i * ny] - Ez[j - 1 + i * ny]);
            U[(j + i * ny) * NV + BYF] = bYOld[j + i * ny]
                + dt / p->dx * (Ez[j + i * ny] - Ez[j + (i - 1) * ny]);
        }
}

/* resistiveMHD_2D.cu:247-291: CFL dt over every cell (ghosts included),
   using the stored face B as if it were cell-centred, then the diffusive
   limit with the scalar eta. */
double orc_calc_dt(const orc_params *p, const double *U)
{
    const int N = p->nx * p->ny;
    const double gm = p->gamma;
    double dtMin = 0.0;
    for (int k = 0; k < N; ++k) {
        const double *c = &U[k * NV];
        double rho = c[RHO];
        double u = c[MX] / rho, v = c[MY] / rho, w = c[MZ] / rho;
        double bX = c[BXF], bY = c[BYF], bZ = c[BZF], e = c[EN];
        double pr = (gm - 1.0)
                  * (e - 0.5 * rho * (u * u + v * v + w * w)
                  - 0.5 * (bX * bX + bY * bY + bZ * bZ));
        double cs = sqrt(gm * pr / rho);
        double ca = sqrt((bX * bX + bY * bY + bZ * bZ) / rho);
        double sx = fabs(u) + sqrt(cs * cs + ca * ca);
        double sy = fabs(v) + sqrt(cs * cs + ca * ca);
        double r = 1.0 / (sx / p->dx + sy / p->dy + p->eps);
        /* thrust::min_element keeps the first minimum: replace only on '<'. */
        if (k == 0 || r < dtMin) dtMin = r;
    }
    double a = p->dx * p->dx / p->eta, b = p->dy * p->dy / p->eta;
    return fmin(dtMin, fmin(a, b)) * p->cfl;
}

/* resistiveMHD_2D.cu:294-309. */
int orc_is_crashed(const orc_params *p, const double *U)
{
    const int N = p->nx * p->ny;
    for (int k = 0; k < N; ++k) if (isnan(U[k * NV + EN])) return 1;
    return 0;
}

/* boundary.cu:4-57 periodicBoundaryX2nd_kernel. */
static void periodic_x(const orc_params *p, double *U)
{
    const int nx = p->nx, ny = p->ny;
    for (int j = 0; j < ny; ++j)
        for (int g = 0; g < 3; ++g) {
            memcpy(&U[(j + g * ny) * NV], &U[(j + (nx - 6 + g) * ny) * NV], NV * sizeof(double));
            memcpy(&U[(j + (nx - 3 + g) * ny) * NV], &U[(j + (3 + g) * ny) * NV], NV * sizeof(double));
        }
}

/* boundary.cu:73-141 periodicBoundaryY2nd_kernel. */
static void periodic_y(const orc_params *p, double *U)
{
    const int nx = p->nx, ny = p->ny;
    for (int i = 0; i < nx; ++i)
        for (int g = 0; g < 3; ++g) {
            memcpy(&U[(g + i * ny) * NV], &U[(ny - 6 + g + i * ny) * NV], NV * sizeof(double));
            memcpy(&U[(ny - 3 + g + i * ny) * NV], &U[(3 + g + i * ny) * NV], NV * sizeof(double));
        }
}

static void copy_except(double *dst, const double *src, int skip)
{
    for (int f = 0; f < NV; ++f) if (f != skip) dst[f] = src[f];
}

#define C(i, j) (&U[((j) + (i) * ny) * NV])

/* symmetricXY/boundary.cu:4-104 symmetricBoundaryX2nd (+BX): mirror copies
   of every field except bX, whose ghosts are integrated from the discrete
   div B = 0. */
static void symmetric_x(const orc_params *p, double *U)
{
    const int nx = p->nx, ny = p->ny;
    const double dx = p->dx, dy = p->dy;
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

/* symmetricXY/boundary.cu:107-205 symmetricBoundaryY2nd (+BY). */
static void symmetric_y(const orc_params *p, double *U)
{
    const int nx = p->nx, ny = p->ny;
    const double dx = p->dx, dy = p->dy;
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

/* The multi-GPU library's walls (ResistiveMHD_multiGPU_cuda/
   ResistiveMHD2D_GPU/boundary.cu:48-355), with its 3 ghost layers. */

/* The resting wall state built from cell c (boundary.cu:63-84): density,
   normal B and bZ kept, velocity and tangential bY set to 0, energy rebuilt
   from the cell's pressure. */
static void mc_wall_state(const double *c, double gm, double *out)
{
    double rho = c[RHO];
    double u = c[MX] / rho, v = c[MY] / rho, w = c[MZ] / rho;
    double bX = c[BXF], bY = c[BYF], bZ = c[BZF], e = c[EN];
    double p = (gm - 1.0) * (e - 0.5 * rho * (u * u + v * v + w * w) - 0.5 * (bX * bX + bY * bY + bZ * bZ));
    out[RHO] = rho;
    out[MX] = rho * 0.0; out[MY] = rho * 0.0; out[MZ] = rho * 0.0;
    out[BXF] = bX; out[BYF] = 0.0; out[BZF] = bZ;
    out[EN] = p / (gm - 1.0) + 0.5 * rho * (0.0 * 0.0 + 0.0 * 0.0 + 0.0 * 0.0) + 0.5 * (bX * bX + 0.0 * 0.0 + bZ * bZ);
}

/* The line-tied state of the flare's x = xmin wall (boundary.cu:212-229):
   as the wall state but keeping the cell's v. */
static void mc_flare_state(const double *c, double gm, double *out)
{
    double rho = c[RHO];
    double u = c[MX] / rho, v = c[MY] / rho, w = c[MZ] / rho;
    double bX = c[BXF], bY = c[BYF], bZ = c[BZF], e = c[EN];
    double p = (gm - 1.0) * (e - 0.5 * rho * (u * u + v * v + w * w) - 0.5 * (bX * bX + bY * bY + bZ * bZ));
    out[RHO] = rho;
    out[MX] = rho * 0.0; out[MY] = rho * v; out[MZ] = rho * 0.0;
    out[BXF] = bX; out[BYF] = 0.0; out[BZF] = bZ;
    out[EN] = p / (gm - 1.0) + 0.5 * rho * (0.0 * 0.0 + v * v + 0.0 * 0.0) + 0.5 * (bX * bX + 0.0 * 0.0 + bZ * bZ);
}

/* boundary.cu:196-245 flareBoundaryX2nd_U: line-tied at x = xmin, copies of
   the last interior column at x = xmax; every row.  With flare = 0 both
   sides are copies (the zero-gradient wall). */
static void mc_x_pass(const orc_params *p, double *U, int flare)
{
    const int nx = p->nx, ny = p->ny;
    for (int j = 0; j < ny; ++j) {
        double wl[NV];
        const double *c3 = &U[(j + 3 * ny) * NV];
        if (flare) mc_flare_state(c3, p->gamma, wl);
        else memcpy(wl, c3, sizeof(wl));
        for (int g = 0; g < 3; ++g) memcpy(&U[(j + g * ny) * NV], wl, sizeof(wl));
        double wr[NV];
        memcpy(wr, &U[(j + (nx - 4) * ny) * NV], sizeof(wr));
        for (int g = 0; g < 3; ++g) memcpy(&U[(j + (nx - 1 - g) * ny) * NV], wr, sizeof(wr));
    }
}

/* boundary.cu:48-119 wallBoundaryY2nd_U (wall = 1) and boundary.cu:292-337
   symmetricBoundaryY2nd_U, the zero-gradient copy (wall = 0); every column. */
static void mc_y_pass(const orc_params *p, double *U, int wall)
{
    const int nx = p->nx, ny = p->ny;
    for (int i = 0; i < nx; ++i) {
        double lo[NV], hi[NV];
        const double *c3 = &U[(3 + i * ny) * NV], *cn = &U[(ny - 4 + i * ny) * NV];
        if (wall) { mc_wall_state(c3, p->gamma, lo); mc_wall_state(cn, p->gamma, hi); }
        else { memcpy(lo, c3, sizeof(lo)); memcpy(hi, cn, sizeof(hi)); }
        for (int g = 0; g < 3; ++g) {
            memcpy(&U[(g + i * ny) * NV], lo, sizeof(lo));
            memcpy(&U[(ny - 1 - g + i * ny) * NV], hi, sizeof(hi));
        }
    }
}

/* The x pass then the y pass, as every oneStepRK2 variant calls them
   (TP/TS resistiveMHD_2D.cu:171-172,193-194; the periodic-x / symmetric-y
   composition is lib_ResistiveMHD_2D_GPU_single/resistiveMHD_2D.cu:229-230,252-253). */
void orc_boundary(const orc_params *p, double *U)
{
    const int bcy = p->bc_y < 0 ? p->bc : p->bc_y;
    switch (p->bc) {
    case ORC_BC_SYMMETRIC: symmetric_x(p, U); break;
    case ORC_BC_ZERO_GRADIENT: mc_x_pass(p, U, 0); break;
    case ORC_BC_FLARE: mc_x_pass(p, U, 1); break;
    default: periodic_x(p, U); break;
    }
    switch (bcy) {
    case ORC_BC_SYMMETRIC: symmetric_y(p, U); break;
    case ORC_BC_ZERO_GRADIENT: mc_y_pass(p, U, 0); break;
    case ORC_BC_WALL: mc_y_pass(p, U, 1); break;
    default: periodic_y(p, U); break;
    }
}

size_t orc_work_doubles(int nx, int ny)
{
    size_t N = (size_t)nx * ny;
    /* UBar, T, F, G, dQ, dQL, dQR (8 each) + bXOld, bYOld, tmp, Ez,
       and for CT-Contact the 12 per-cell EMF inputs of the two stages */
    return N * (7 * 8 + 4 + 12);
}

/* resistiveMHD_2D.cu:133-195 oneStepRK2.  U is updated in place; work must
   hold orc_work_doubles(nx, ny) doubles.  Ustar (may be NULL) receives the
   stage-1 state after its boundary pass, the state stage 2 reads.  Returns
   the dt used. */
static double step_impl(const orc_params *p, double *U, double *work, double *Ustar)
{
    const int nx = p->nx, ny = p->ny, N = nx * ny;
    double *UBar = work;
    double *T = UBar + (size_t)N * 8;
    double *F = T + (size_t)N * 8;
    double *G = F + (size_t)N * 8;
    double *dQ = G + (size_t)N * 8;
    double *dQL = dQ + (size_t)N * 8;
    double *dQR = dQL + (size_t)N * 8;
    double *bXOld = dQR + (size_t)N * 8;
    double *bYOld = bXOld + N;
    double *tmp = bYOld + N;
    double *Ez = tmp + N;

    for (int k = 0; k < N; ++k) { bXOld[k] = U[k * NV + BXF]; bYOld[k] = U[k * NV + BYF]; }
    memcpy(UBar, U, (size_t)N * NV * sizeof(double));

    const double dt = orc_calc_dt(p, U);
    const double dx = p->dx, dy = p->dy;

    shift_to_center(p, U, tmp);
    flux_x(p, U, F, dQ, dQL, dQR);
    flux_y(p, U, G, T, dQ, dQL, dQR);
    back_to_face(p, U, tmp);

    /* oneStepFirstFunctor over k in [ny, N). */
    #pragma omp parallel for schedule(static)
    for (int k = ny; k < N; ++k) {
        const double *u = &U[k * NV];
        const double *f = &F[k * 8], *fm = &F[(k - ny) * 8];
        const double *g = &G[k * 8], *gm = &G[(k - 1) * 8];
        double *ub = &UBar[k * NV];
        for (int c = 0; c < 8; ++c)
            ub[c] = u[c] - dt / dx * (f[c] - fm[c]) - dt / dy * (g[c] - gm[c]);
    }

    corner_ez(p, F, G, Ez);
    ct_update(p, bXOld, bYOld, Ez, dt, UBar);
    orc_boundary(p, UBar);
    if (Ustar) memcpy(Ustar, UBar, (size_t)N * NV * sizeof(double));

    shift_to_center(p, UBar, tmp);
    flux_x(p, UBar, F, dQ, dQL, dQR);
    flux_y(p, UBar, G, T, dQ, dQL, dQR);
    back_to_face(p, UBar, tmp);

    /* oneStepSecondFunctor over k in [ny, N). */
    #pragma omp parallel for schedule(static)
    for (int k = ny; k < N; ++k) {
        double *u = &U[k * NV];
        const double *ub = &UBar[k * NV];
        const double *f = &F[k * 8], *fm = &F[(k - ny) * 8];
        const double *g = &G[k * 8], *gm = &G[(k - 1) * 8];
        for (int c = 0; c < 8; ++c)
            u[c] = 0.5 * (u[c] + ub[c]
                 - dt / dx * (f[c] - fm[c])
                 - dt / dy * (g[c] - gm[c]));
    }

    /* CT again with the stage-1 corner EMF (setOldFlux2D is not called for
       stage 2). */
    ct_update(p, bXOld, bYOld, Ez, dt, U);
    orc_boundary(p, U);
    return dt;
}

double orc_step(const orc_params *p, double *U, double *work)
{
    return step_impl(p, U, work, NULL);
}

/* CT-Contact inputs of one stage, per cell (ResistiveMHD_multiGPU_cuda/
   ResistiveMHD2D_GPU/ct.cu:26-65 setFlux_kernel): the numerical induction
   fluxes F.f5, G.f4, the mass fluxes F.f0, G.f0, and the cell's reference
   EMF u*bY - v*bX - eta*jZ (with centred face B and the mean of the four
   corner curls of U's face B) as the x flux and its negative as the y flux,
   for 0 < i < nx-1, 0 < j < ny-1.  Entries outside are left NaN. */
static void contact_set_flux(const orc_params *p, const double *F, const double *G, const double *U,
                             double *NF5, double *NG4, double *CF5, double *CG4, double *NF0, double *NG0)
{
    const int nx = p->nx, ny = p->ny, N = nx * ny;
    const double dx = p->dx, dy = p->dy;
    for (int k = 0; k < N; ++k) NF5[k] = NG4[k] = CF5[k] = CG4[k] = NF0[k] = NG0[k] = NAN;
    for (int i = 1; i < nx - 1; ++i) {
        for (int j = 1; j < ny - 1; ++j) {
            const int index = j + i * ny;
#define BXAT(k) U[(k) * NV + BXF]
#define BYAT(k) U[(k) * NV + BYF]
            double rho = U[index * NV + RHO];
            double u = U[index * NV + MX] / rho;
            double v = U[index * NV + MY] / rho;
            double bX = 0.5 * (BXAT(index) + BXAT(index - ny));
            double bY = 0.5 * (BYAT(index) + BYAT(index - 1));
            double jZ = 0.25 * (
                (BYAT(index + ny) - BYAT(index)) / dx - (BXAT(index + 1) - BXAT(index)) / dy
              + (BYAT(index - 1 + ny) - BYAT(index - 1)) / dx - (BXAT(index) - BXAT(index - 1)) / dy
              + (BYAT(index - 1) - BYAT(index - 1 - ny)) / dx - (BXAT(index - ny) - BXAT(index - ny - 1)) / dy
              + (BYAT(index) - BYAT(index - ny)) / dx - (BXAT(index + 1 - ny) - BXAT(index - ny)) / dy);
#undef BXAT
#undef BYAT
            double eta = eta_at(p, i, j);
            NF5[index] = F[index * 8 + 5];
            NG4[index] = G[index * 8 + 4];
            CF5[index] = u * bY - v * bX - eta * jZ;
            CG4[index] = -(u * bY - v * bX - eta * jZ);
            NF0[index] = F[index * 8 + 0];
            NG0[index] = G[index * 8 + 0];
        }
    }
}

/* MC sign(): (x > 0) - (x < 0) as an int (sign.cu). */
static inline int isgn(double x) { return (x > 0.0) - (x < 0.0); }

/* One stage's CT-Contact corner EMF at corner (i+1/2, j+1/2) (ct.cu:147-169):
   the arithmetic mean of the four numerical induction fluxes plus the
   upwinded corrections selected by the signs of the mass fluxes. */
static double contact_corner(int index, int ny, const double *NF5, const double *NG4, const double *CF5,
                             const double *CG4, const double *NF0, const double *NG0)
{
    double avg = 0.25 * (-NF5[index] - NF5[index + 1] + NG4[index] + NG4[index + ny]);
    double eS = (1.0 + isgn(NF0[index])) * (NG4[index] - CG4[index])
              + (1.0 - isgn(NF0[index])) * (NG4[index + ny] - CG4[index + ny]);
    double eN = (1.0 + isgn(NF0[index + 1])) * (CG4[index + 1] - NG4[index])
              + (1.0 - isgn(NF0[index + 1])) * (CG4[index + 1 + ny] - NG4[index + ny]);
    double eW = -(1.0 + isgn(NG0[index])) * (NF5[index] - CF5[index])
              - (1.0 - isgn(NG0[index])) * (NF5[index + 1] - CF5[index + 1]);
    double eE = -(1.0 + isgn(NG0[index + ny])) * (CF5[index + ny] - NF5[index])
              - (1.0 - isgn(NG0[index + ny])) * (CF5[index + 1 + ny] - NF5[index + 1]);
    return avg + 0.125 * (eS - eN + eW - eE);
}

/* Corner EMFs of the CT-Contact step (ct.cu:124-200 getEZVector_kernel):
   the mean of the two stages' contact EMFs at every corner (i+1/2, j+1/2)
   with i < nx-1, j < ny-1; NaN elsewhere.  o and n point to the six
   per-cell input planes of each stage (NF5, NG4, CF5, CG4, NF0, NG0 in a row
   of nx*ny doubles each). */
static void contact_ez(const orc_params *p, const double *o, const double *n, double *Ez)
{
    const int nx = p->nx, ny = p->ny, N = nx * ny;
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) {
            const int index = j + i * ny;
            if (i < nx - 1 && j < ny - 1) {
                double eOld = contact_corner(index, ny, o, o + N, o + 2 * N, o + 3 * N, o + 4 * N, o + 5 * N);
                double eNow = contact_corner(index, ny, n, n + N, n + 2 * N, n + 3 * N, n + 4 * N, n + 5 * N);
                Ez[index] = 0.5 * (eOld + eNow);
            } else {
                Ez[index] = NAN;
            }
        }
}

/* The step with the CT-Contact EMF of the multi-GPU library
   (ResistiveMHD2D_GPU/resistiveMHD2D.cu:147-221 oneStepRK2 ordering,
   ct.cu:26-257): both stages update B by flux differences like every other
   field, from the face B that shift + back-to-face left in U; the reference
   EMFs of stage 1 are taken from U after that smoothing and those of stage 2
   from the step's output after its boundary pass; one CT from the step
   input's faces with the mean of the two stages' contact EMFs ends the
   step, followed by the boundary pass.  Fluxes (HLLD, MUSCL, the resistive
   hook), the update ranges and dt are this library's (resistiveMHD_2D.cu
   of the single-GPU library).  Returns the dt used. */
double orc_step_contact(const orc_params *p, double *U, double *work)
{
    const int nx = p->nx, ny = p->ny, N = nx * ny;
    double *UBar = work;
    double *T = UBar + (size_t)N * 8;
    double *F = T + (size_t)N * 8;
    double *G = F + (size_t)N * 8;
    double *dQ = G + (size_t)N * 8;
    double *dQL = dQ + (size_t)N * 8;
    double *dQR = dQL + (size_t)N * 8;
    double *bXOld = dQR + (size_t)N * 8;
    double *bYOld = bXOld + N;
    double *tmp = bYOld + N;
    double *Ez = tmp + N;
    double *oNF5 = Ez + N, *oNG4 = oNF5 + N, *oCF5 = oNG4 + N, *oCG4 = oCF5 + N, *oNF0 = oCG4 + N, *oNG0 = oNF0 + N;
    double *nNF5 = oNG0 + N, *nNG4 = nNF5 + N, *nCF5 = nNG4 + N, *nCG4 = nCF5 + N, *nNF0 = nCG4 + N, *nNG0 = nNF0 + N;

    for (int k = 0; k < N; ++k) { bXOld[k] = U[k * NV + BXF]; bYOld[k] = U[k * NV + BYF]; }
    memcpy(UBar, U, (size_t)N * NV * sizeof(double));

    const double dt = orc_calc_dt(p, U);
    const double dx = p->dx, dy = p->dy;

    shift_to_center(p, U, tmp);
    flux_x(p, U, F, dQ, dQL, dQR);
    flux_y(p, U, G, T, dQ, dQL, dQR);
    back_to_face(p, U, tmp);
    contact_set_flux(p, F, G, U, oNF5, oNG4, oCF5, oCG4, oNF0, oNG0);

    for (int k = ny; k < N; ++k) {
        const double *u = &U[k * NV];
        const double *f = &F[k * 8], *fm = &F[(k - ny) * 8];
        const double *g = &G[k * 8], *gm = &G[(k - 1) * 8];
        double *ub = &UBar[k * NV];
        for (int c = 0; c < 8; ++c)
            ub[c] = u[c] - dt / dx * (f[c] - fm[c]) - dt / dy * (g[c] - gm[c]);
    }
    orc_boundary(p, UBar);

    shift_to_center(p, UBar, tmp);
    flux_x(p, UBar, F, dQ, dQL, dQR);
    flux_y(p, UBar, G, T, dQ, dQL, dQR);
    back_to_face(p, UBar, tmp);

    for (int k = ny; k < N; ++k) {
        double *u = &U[k * NV];
        const double *ub = &UBar[k * NV];
        const double *f = &F[k * 8], *fm = &F[(k - ny) * 8];
        const double *g = &G[k * 8], *gm = &G[(k - 1) * 8];
        for (int c = 0; c < 8; ++c)
            u[c] = 0.5 * (u[c] + ub[c]
                 - dt / dx * (f[c] - fm[c])
                 - dt / dy * (g[c] - gm[c]));
    }
    orc_boundary(p, U);
    contact_set_flux(p, F, G, U, nNF5, nNG4, nCF5, nCG4, nNF0, nNG0);
    contact_ez(p, oNF5, nNF5, Ez);
    ct_update(p, bXOld, bYOld, Ez, dt, U);
    orc_boundary(p, U);
    return dt;
}

size_t orc_contact_ct_work_doubles(int nx, int ny) { return (size_t)13 * nx * ny; }

/* The closing constrained transport of the CT-Contact step on given inputs:
   the contact inputs of the first stage from (Fold, Gold, Uold), those of
   the second from (Fnow, Gnow, U), the corner EMF 0.5 (eOld + eNow), and the
   CT of U's face B from bXOld, bYOld with dt, in place in U (which holds the
   second stage's state on entry).  This is the composition
   CT::setOldFlux2D, CT::setNowFlux2D, CT::divBClean of the multi-GPU library
   (ResistiveMHD2D_GPU/ct.cu:26-257, called at resistiveMHD2D.cu:177,212-214)
   that orc_step_contact ends with; exposed so that it can be checked against
   that library's own code. */
void orc_contact_ct(const orc_params *p, const double *Uold, const double *Fold, const double *Gold,
                    const double *Fnow, const double *Gnow, const double *bXOld, const double *bYOld, double dt,
                    double *U, double *work)
{
    const int N = p->nx * p->ny;
    double *Ez = work;
    double *oNF5 = Ez + N, *oNG4 = oNF5 + N, *oCF5 = oNG4 + N, *oCG4 = oCF5 + N, *oNF0 = oCG4 + N, *oNG0 = oNF0 + N;
    double *nNF5 = oNG0 + N, *nNG4 = nNF5 + N, *nCF5 = nNG4 + N, *nCG4 = nCF5 + N, *nNF0 = nCG4 + N, *nNG0 = nNF0 + N;
    contact_set_flux(p, Fold, Gold, Uold, oNF5, oNG4, oCF5, oCG4, oNF0, oNG0);
    contact_set_flux(p, Fnow, Gnow, U, nNF5, nNG4, nCF5, nCG4, nNF0, nNG0);
    contact_ez(p, oNF5, nNF5, Ez);
    ct_update(p, bXOld, bYOld, Ez, dt, U);
}

/* Runs nsteps steps; dts (may be NULL) receives each step's dt.  Returns 0,
   or 1 + the step index at which the crash check (NaN energy) fired, after
   which no further step is taken, as the reference drivers do. */
/* nsteps stage-1-EMF steps as orc_run takes them, keeping the trajectory a
   discrete adjoint of the steps reverses: Un + s*nx*ny*8 receives the state
   step s starts from and Ustar + s*nx*ny*8 its stage-1 state after the
   boundary pass.  dts receives each step's dt.  Returns as orc_run. */
int orc_run_keep_stages(const orc_params *p, double *U, int nsteps, double *dts, double *Un, double *Ustar)
{
    const size_t sd = (size_t)p->nx * p->ny * NV;
    size_t nw = orc_work_doubles(p->nx, p->ny);
    double *work = (double *)malloc(nw * sizeof(double));
    if (!work) return -1;
    int rc = 0;
    for (int s = 0; s < nsteps; ++s) {
        memcpy(Un + (size_t)s * sd, U, sd * sizeof(double));
        dts[s] = step_impl(p, U, work, Ustar + (size_t)s * sd);
        if (orc_is_crashed(p, U)) { rc = 1 + s; break; }
    }
    free(work);
    return rc;
}

int orc_run(const orc_params *p, double *U, int nsteps, double *dts)
{
    size_t nw = orc_work_doubles(p->nx, p->ny);
    double *work = (double *)malloc(nw * sizeof(double));
    if (!work) return -1;
    int rc = 0;
    for (int s = 0; s < nsteps; ++s) {
        double dt = p->ct_contact ? orc_step_contact(p, U, work) : orc_step(p, U, work);
        if (dts) dts[s] = dt;
        if (orc_is_crashed(p, U)) { rc = 1 + s; break; }
    }
    free(work);
    return rc;
}
