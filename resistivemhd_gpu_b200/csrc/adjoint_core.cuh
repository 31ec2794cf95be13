// adjoint_core.cuh -- reverse-mode derivatives of the per-interface
// arithmetic of the step: primitive recovery, MUSCL-minmod reconstruction
// and the HLLD flux.  Plain C++ on doubles, usable from device code and from
// host code.
//
// Each function recomputes its forward values in the evaluation order of
// the reference (hlld.cu:35-565, muscl.cu:6-126, minmod.hpp:6-16,
// calculate_half_Q.cu:4-38), so the branches it takes -- minmod's choice,
// thrust::min/max, the HLLD region indicators -- are the ones the forward
// step took, and then propagates adjoints backwards through the branch
// taken.  Derivatives are those of the exact formulas (e.g. cs*cs is
// differentiated as gamma*p/rho); where a formula is not differentiable
// (sqrt at 0) the derivative of that term is taken as 0.
#pragma once

#include <math.h>

#if defined(__CUDACC__)
#define ADJ_FN __host__ __device__ __forceinline__
#else
#define ADJ_FN inline
#endif

namespace rmhd2d {
namespace adj {

// BasicParameter order (basic_parameter_struct.hpp:5-27).
enum { QR = 0, QU = 1, QV = 2, QW = 3, QBX = 4, QBY = 5, QBZ = 6, QP = 7 };

// The seven reconstructed components, in the reference's loop order.
ADJ_FN int recon_comp(int n) { return n < 4 ? n : n + 1; }

ADJ_FN double sgn_d(double x) { return (double)((x > 0.0) - (x < 0.0)); }

// calculate_half_Q.cu:4-38 for a cell c (sweep order rho, m_n, m_t1, m_t2,
// b_n, b_t1, b_t2, e) and its neighbour's b_n.
ADJ_FN void basic_param(const double *c, double bn_next, double gm, double *q)
{
    const double rho = c[0];
    const double u = c[1] / rho, v = c[2] / rho, w = c[3] / rho;
    const double bX = c[4], bY = c[5], bZ = c[6], e = c[7];
    q[QP] = (gm - 1.0) * (e - 0.5 * (rho * (u * u + v * v + w * w)) - 0.5 * (bX * bX + bY * bY + bZ * bZ));
    q[QR] = rho;
    q[QU] = u;
    q[QV] = v;
    q[QW] = w;
    q[QBX] = 0.5 * (bX + bn_next);
    q[QBY] = bY;
    q[QBZ] = bZ;
}

// Reverse of basic_param: qb (8 adjoints of q) -> cb (8 adjoints of the cell,
// accumulated).  The b_n of the next cell receives 0.5 * qb[QBX], which the
// caller routes.
ADJ_FN void basic_param_adj(const double *c, double gm, const double *qb, double *cb)
{
    const double rho = c[0];
    const double ir = 1.0 / rho;
    const double u = c[1] * ir, v = c[2] * ir, w = c[3] * ir;
    const double g1 = gm - 1.0;
    const double pb = qb[QP];
    cb[0] += qb[QR] - (qb[QU] * u + qb[QV] * v + qb[QW] * w) * ir + pb * g1 * 0.5 * (u * u + v * v + w * w);
    cb[1] += qb[QU] * ir - pb * g1 * u;
    cb[2] += qb[QV] * ir - pb * g1 * v;
    cb[3] += qb[QW] * ir - pb * g1 * w;
    cb[4] += 0.5 * qb[QBX] - pb * g1 * c[4];
    cb[5] += qb[QBY] - pb * g1 * c[5];
    cb[6] += qb[QBZ] - pb * g1 * c[6];
    cb[7] += pb * g1;
}

// minmod.hpp:6-16 with the branch taken: 0 constant (sign change or below
// EPS), 1 the first argument, 2 the second.
ADJ_FN double minmod_sel(double x, double y, double eps, int &sel)
{
    const int s = (x > 0) - (x < 0);
    const double ax = fabs(x);
    const double sy = (double)s * y;
    const bool pick_y = sy < ax;          // thrust::min(ax, s*y)
    const double in = pick_y ? sy : ax;
    const bool clamp = in < eps;          // thrust::max(in, EPS)
    sel = (s == 0 || clamp) ? 0 : (pick_y ? 2 : 1);
    return (double)s * (clamp ? eps : in);
}

// muscl.cu:6-30 / 66-90: interface states from dQ of cells m-1, m, m+1, m+2
// (pointers q0..q3); the 14 minmod branches are packed 2 bits each (left
// components in bits 0..13, right in 14..27).
ADJ_FN unsigned muscl_states(const double *q0, const double *q1, const double *q2, const double *q3, double eps,
                             double *L, double *R)
{
    unsigned bits = 0u;
#pragma unroll
    for (int n = 0; n < 7; ++n) {
        const int c = recon_comp(n);
        int sl, sr;
        L[c] = q1[c] + 0.5 * minmod_sel(q1[c] - q0[c], q2[c] - q1[c], eps, sl);
        R[c] = q2[c] - 0.5 * minmod_sel(q2[c] - q1[c], q3[c] - q2[c], eps, sr);
        bits |= (unsigned)sl << (2 * n);
        bits |= (unsigned)sr << (14 + 2 * n);
    }
    L[QBX] = q1[QBX];
    R[QBX] = q1[QBX];
    return bits;
}

struct St {
    double rho, u, v, w, bX, bY, bZ, e, pT;
};

// Reverse of getOneFlux (hlld.cu:448-467).
ADJ_FN void one_flux_adj(const St &s, const double *fb, St &sb)
{
    const double rho = s.rho, u = s.u, v = s.v, w = s.w, bX = s.bX, bY = s.bY, bZ = s.bZ;
    sb.rho += fb[0] * u + fb[1] * u * u + fb[2] * u * v + fb[3] * u * w;
    sb.u += fb[0] * rho + fb[1] * 2.0 * rho * u + fb[2] * rho * v + fb[3] * rho * w + fb[5] * bY + fb[6] * bZ
          + fb[7] * (s.e + s.pT);
    sb.v += fb[2] * rho * u - fb[5] * bX;
    sb.w += fb[3] * rho * u - fb[6] * bX;
    sb.pT += fb[1] + fb[7] * u;
    sb.e += fb[7] * u;
    const double vb = bX * u + bY * v + bZ * w;
    sb.bX += -fb[1] * 2.0 * bX - fb[2] * bY - fb[3] * bZ - fb[5] * v - fb[6] * w - fb[7] * vb;
    sb.bY += -fb[2] * bX + fb[5] * u;
    sb.bZ += -fb[3] * bX + fb[6] * u;
    const double t = -fb[7] * bX;   // adjoint of bX*u + bY*v + bZ*w
    sb.bX += t * u;
    sb.u += t * bX;
    sb.bY += t * v;
    sb.v += t * bY;
    sb.bZ += t * w;
    sb.w += t * bZ;
}

// Reverse of the fast magnetosonic speed
// cf = sqrt((cs2 + ca2 + sqrt((cs2 + ca2)^2 - 4 cs2 va2)) / 2),
// cs2 = gm p / rho, ca2 = |B|^2 / rho, va2 = bX^2 / rho (hlld.cu:290-310).
ADJ_FN void fast_speed_adj(double rho, double bX, double bY, double bZ, double p, double gm, double cf, double cfb,
                           double &rhob, double &bXb, double &bYb, double &bZb, double &pb)
{
    if (cfb == 0.0 || !(cf > 0.0)) return;
    const double ir = 1.0 / rho;
    const double cs2 = gm * p * ir, B2 = bX * bX + bY * bY + bZ * bZ, ca2 = B2 * ir, va2 = bX * bX * ir;
    const double s = cs2 + ca2;
    const double disc = s * s - 4.0 * cs2 * va2;
    const double rd = disc > 0.0 ? sqrt(disc) : 0.0;
    const double tb = cfb / (2.0 * cf);
    double sb = 0.5 * tb;
    const double db = rd > 0.0 ? 0.5 * tb / (2.0 * rd) : 0.0;
    sb += 2.0 * s * db;
    const double cs2b = sb - 4.0 * va2 * db;
    const double ca2b = sb;
    const double va2b = -4.0 * cs2 * db;
    pb += gm * ir * cs2b;
    rhob -= (cs2 * cs2b + ca2 * ca2b + va2 * va2b) * ir;
    const double B2b = ca2b * ir;
    bXb += 2.0 * bX * (B2b + va2b * ir);
    bYb += 2.0 * bY * B2b;
    bZb += 2.0 * bZ * B2b;
}

// Adjoints of the star / double-star quantities of one side of the fan.
struct SideBar {
    double rho1, v1, w1, bY1, bZ1, e1;
};

// Reverse of the HLLD flux (hlld.cu:35-131 CalculateFluxFunctor,
// hlld.cu:256-444 calculateHLLDParameterFunctor, hlld.cu:448-565
// setFluxFunctor): given fb = dJ/dflux, accumulates dJ/dL into Lb and dJ/dR
// into Rb (8 components each, BasicParameter order).  The flux is the
// indicator-weighted sum of six candidate fluxes; each selected candidate
// passes fb back through its state.
ADJ_FN void hlld_flux_adj(const double *L, const double *R, double gm, double EPS, const double *fb, double *Lb,
                          double *Rb)
{
    // ---- forward, in the reference's evaluation order ----
    const double rhoL = L[QR], uL = L[QU], vL = L[QV], wL = L[QW];
    const double bXL = L[QBX], bYL = L[QBY], bZL = L[QBZ], pL = L[QP];
    const double rhoR = R[QR], uR = R[QU], vR = R[QV], wR = R[QW];
    const double bXR = R[QBX], bYR = R[QBY], bZR = R[QBZ], pR = R[QP];

    const double eL = pL / (gm - 1.0) + 0.5 * rhoL * (uL * uL + vL * vL + wL * wL)
                    + 0.5 * (bXL * bXL + bYL * bYL + bZL * bZL);
    const double pTL = pL + 0.5 * (bXL * bXL + bYL * bYL + bZL * bZL);
    const double eR = pR / (gm - 1.0) + 0.5 * rhoR * (uR * uR + vR * vR + wR * wR)
                    + 0.5 * (bXR * bXR + bYR * bYR + bZR * bZR);
    const double pTR = pR + 0.5 * (bXR * bXR + bYR * bYR + bZR * bZR);

    double cfL, cfR;
    {
        const double cs = sqrt(gm * pL / rhoL), ca = sqrt((bXL * bXL + bYL * bYL + bZL * bZL) / rhoL);
        const double va = sqrt(bXL * bXL / rhoL);
        cfL = sqrt(0.5 * (cs * cs + ca * ca + sqrt((cs * cs + ca * ca) * (cs * cs + ca * ca) - 4.0 * cs * cs * va * va)));
    }
    {
        const double cs = sqrt(gm * pR / rhoR), ca = sqrt((bXR * bXR + bYR * bYR + bZR * bZR) / rhoR);
        const double va = sqrt(bXR * bXR / rhoR);
        cfR = sqrt(0.5 * (cs * cs + ca * ca + sqrt((cs * cs + ca * ca) * (cs * cs + ca * ca) - 4.0 * cs * cs * va * va)));
    }
    // thrust::min(a, b) = b < a ? b : a, thrust::max(a, b) = a < b ? b : a
    const bool umin_R = uR < uL, umax_R = uL < uR, cfm_R = cfL < cfR;
    const double umin = umin_R ? uR : uL, umax = umax_R ? uR : uL, cfm = cfm_R ? cfR : cfL;
    const double SL0 = umin - cfm, SR0 = umax + cfm;
    const bool SL_clamped = 0.0 < SL0, SR_clamped = SR0 < 0.0;
    const double SL = SL_clamped ? 0.0 : SL0, SR = SR_clamped ? 0.0 : SR0;

    const double aL = SL - uL, aR = SR - uR;
    const double den = aR * rhoR - aL * rhoL + EPS;
    const double SM = (aR * rhoR * uR - aL * rhoL * uL - pTR + pTL) / den;
    const double pT1 = (aR * rhoR * pTL - aL * rhoL * pTR + rhoL * rhoR * aR * aL * (uR - uL)) / den;

    const double dSL = SL - SM + EPS;
    const double rho1L = rhoL * aL / dSL;
    const double DL = rhoL * aL * (SL - SM) - bXL * bXL + EPS;
    const double NL = rhoL * aL * aL - bXL * bXL;
    const double v1L = vL - bXL * bYL * (SM - uL) / DL;
    const double w1L = wL - bXL * bZL * (SM - uL) / DL;
    const double bY1L = bYL * NL / DL;
    const double bZ1L = bZL * NL / DL;
    const double vbL = uL * bXL + vL * bYL + wL * bZL;
    const double vb1L = SM * bXL + v1L * bY1L + w1L * bZ1L;
    const double e1L = (aL * eL - pTL * uL + pT1 * SM + bXL * (vbL - vb1L)) / dSL;

    const double dSR = SR - SM + EPS;
    const double rho1R = rhoR * aR / dSR;
    const double DR = rhoR * aR * (SR - SM) - bXR * bXR + EPS;
    const double NR = rhoR * aR * aR - bXR * bXR;
    const double v1R = vR - bXR * bYR * (SM - uR) / DR;
    const double w1R = wR - bXR * bZR * (SM - uR) / DR;
    const double bY1R = bYR * NR / DR;
    const double bZ1R = bZR * NR / DR;
    const double vbR = uR * bXR + vR * bYR + wR * bZR;
    const double vb1R = SM * bXR + v1R * bY1R + w1R * bZ1R;
    const double e1R = (aR * eR - pTR * uR + pT1 * SM + bXR * (vbR - vb1R)) / dSR;

    const double S1L = SM - sqrt(bXL * bXL / rho1L);
    const double S1R = SM + sqrt(bXR * bXR / rho1R);

    const double sg = sgn_d(bXL);
    const double sqL = sqrt(rho1L), sqR = sqrt(rho1R), sqLR = sqrt(rho1L * rho1R);
    const double dd = sqL + sqR + EPS;
    const double v2 = (sqL * v1L + sqR * v1R + (bY1R - bY1L) * sg) / dd;
    const double w2 = (sqL * w1L + sqR * w1R + (bZ1R - bZ1L) * sg) / dd;
    const double bY2 = (sqL * bY1R + sqR * bY1L + sqLR * (v1R - v1L) * sg) / dd;
    const double bZ2 = (sqL * bZ1R + sqR * bZ1L + sqLR * (w1R - w1L) * sg) / dd;
    const double vb2L = SM * bXL + v2 * bY2 + w2 * bZ2;
    const double vb2R = SM * bXR + v2 * bY2 + w2 * bZ2;
    const double sgL = sgn_d(bXL), sgR = sgn_d(bXR);
    const double e2L = e1L - sqL * (vb1L - vb2L) * sgL;
    const double e2R = e1R + sqR * (vb1R - vb2R) * sgR;

    const bool iOL = SL > 0.0;
    const bool iML = (SL <= 0.0) && (0.0 < S1L);
    const bool iIL = (S1L <= 0.0) && (0.0 < SM);
    const bool iOR = SR <= 0.0;
    const bool iMR = (S1R <= 0.0) && (0.0 < SR);
    const bool iIR = (SM <= 0.0) && (0.0 < S1R);

    // ---- reverse ----
    St OLb{}, ORb{};
    SideBar Lsb{}, Rsb{};
    double SMb = 0.0, pT1b = 0.0, v2b = 0.0, w2b = 0.0, bY2b = 0.0, bZ2b = 0.0, e2Lb = 0.0, e2Rb = 0.0;
    double bXLb = 0.0, bXRb = 0.0;
    {
        St b{};
        if (iOL) one_flux_adj(St{rhoL, uL, vL, wL, bXL, bYL, bZL, eL, pTL}, fb, OLb);
        if (iOR) one_flux_adj(St{rhoR, uR, vR, wR, bXR, bYR, bZR, eR, pTR}, fb, ORb);
        if (iML) {
            b = St{};
            one_flux_adj(St{rho1L, SM, v1L, w1L, bXL, bY1L, bZ1L, e1L, pT1}, fb, b);
            Lsb.rho1 += b.rho; SMb += b.u; Lsb.v1 += b.v; Lsb.w1 += b.w; bXLb += b.bX;
            Lsb.bY1 += b.bY; Lsb.bZ1 += b.bZ; Lsb.e1 += b.e; pT1b += b.pT;
        }
        if (iIL) {
            b = St{};
            one_flux_adj(St{rho1L, SM, v2, w2, bXL, bY2, bZ2, e2L, pT1}, fb, b);
            Lsb.rho1 += b.rho; SMb += b.u; v2b += b.v; w2b += b.w; bXLb += b.bX;
            bY2b += b.bY; bZ2b += b.bZ; e2Lb += b.e; pT1b += b.pT;
        }
        if (iMR) {
            b = St{};
            one_flux_adj(St{rho1R, SM, v1R, w1R, bXR, bY1R, bZ1R, e1R, pT1}, fb, b);
            Rsb.rho1 += b.rho; SMb += b.u; Rsb.v1 += b.v; Rsb.w1 += b.w; bXRb += b.bX;
            Rsb.bY1 += b.bY; Rsb.bZ1 += b.bZ; Rsb.e1 += b.e; pT1b += b.pT;
        }
        if (iIR) {
            b = St{};
            one_flux_adj(St{rho1R, SM, v2, w2, bXR, bY2, bZ2, e2R, pT1}, fb, b);
            Rsb.rho1 += b.rho; SMb += b.u; v2b += b.v; w2b += b.w; bXRb += b.bX;
            bY2b += b.bY; bZ2b += b.bZ; e2Rb += b.e; pT1b += b.pT;
        }
    }

    // double-star energies
    double sqLb = 0.0, sqRb = 0.0, sqLRb = 0.0, ddb = 0.0, vb1Lb = 0.0, vb1Rb = 0.0;
    {
        Rsb.e1 += e2Rb;
        sqRb += e2Rb * (vb1R - vb2R) * sgR;
        vb1Rb += e2Rb * sqR * sgR;
        const double vb2Rb = -e2Rb * sqR * sgR;
        Lsb.e1 += e2Lb;
        sqLb -= e2Lb * (vb1L - vb2L) * sgL;
        vb1Lb -= e2Lb * sqL * sgL;
        const double vb2Lb = e2Lb * sqL * sgL;
        SMb += vb2Rb * bXR + vb2Lb * bXL;
        bXRb += vb2Rb * SM;
        bXLb += vb2Lb * SM;
        const double vb2b = vb2Rb + vb2Lb;   // v2*bY2 + w2*bZ2 is shared
        v2b += vb2b * bY2;
        bY2b += vb2b * v2;
        w2b += vb2b * bZ2;
        bZ2b += vb2b * w2;
    }
    // double-star state
    {
        double nb = bZ2b / dd;
        ddb -= bZ2b * bZ2 / dd;
        sqLb += nb * bZ1R; Rsb.bZ1 += nb * sqL; sqRb += nb * bZ1L; Lsb.bZ1 += nb * sqR;
        sqLRb += nb * (w1R - w1L) * sg; Rsb.w1 += nb * sqLR * sg; Lsb.w1 -= nb * sqLR * sg;

        nb = bY2b / dd;
        ddb -= bY2b * bY2 / dd;
        sqLb += nb * bY1R; Rsb.bY1 += nb * sqL; sqRb += nb * bY1L; Lsb.bY1 += nb * sqR;
        sqLRb += nb * (v1R - v1L) * sg; Rsb.v1 += nb * sqLR * sg; Lsb.v1 -= nb * sqLR * sg;

        nb = w2b / dd;
        ddb -= w2b * w2 / dd;
        sqLb += nb * w1L; Lsb.w1 += nb * sqL; sqRb += nb * w1R; Rsb.w1 += nb * sqR;
        Rsb.bZ1 += nb * sg; Lsb.bZ1 -= nb * sg;

        nb = v2b / dd;
        ddb -= v2b * v2 / dd;
        sqLb += nb * v1L; Lsb.v1 += nb * sqL; sqRb += nb * v1R; Rsb.v1 += nb * sqR;
        Rsb.bY1 += nb * sg; Lsb.bY1 -= nb * sg;

        sqLb += ddb;
        sqRb += ddb;
        if (sqLR > 0.0) {
            const double t = sqLRb / (2.0 * sqLR);
            Lsb.rho1 += t * rho1R;
            Rsb.rho1 += t * rho1L;
        }
        if (sqL > 0.0) Lsb.rho1 += sqLb / (2.0 * sqL);
        if (sqR > 0.0) Rsb.rho1 += sqRb / (2.0 * sqR);
    }

    double rhoLb = OLb.rho, uLb = OLb.u, vLb = OLb.v, wLb = OLb.w, bYLb = OLb.bY, bZLb = OLb.bZ, eLb = OLb.e,
           pTLb = OLb.pT;
    double rhoRb = ORb.rho, uRb = ORb.u, vRb = ORb.v, wRb = ORb.w, bYRb = ORb.bY, bZRb = ORb.bZ, eRb = ORb.e,
           pTRb = ORb.pT;
    bXLb += OLb.bX;
    bXRb += ORb.bX;
    double aLb = 0.0, aRb = 0.0, SLb = 0.0, SRb = 0.0;

    // one side of the star region (right: s = +1 uses SR, aR, ...)
    auto star_side = [&](const SideBar &sb, double rho, double u, double v, double w, double bX, double bY, double bZ,
                         double e, double pT, double S, double a, double dS, double rho1, double D, double N,
                         double v1, double w1, double bY1, double bZ1, double vb, double vb1, double e1,
                         double vb1b_in, double &rhob, double &ub, double &vbr, double &wb, double &bXb,
                         double &bYb, double &bZb, double &eb, double &pTb, double &Sb, double &ab) {
        // e1 = (a e - pT u + pT1 SM + bX (vb - vb1)) / dS
        const double nb = sb.e1 / dS;
        double dSb = -sb.e1 * e1 / dS;
        ab += nb * e;
        eb += nb * a;
        pTb -= nb * u;
        ub -= nb * pT;
        pT1b += nb * SM;
        SMb += nb * pT1;
        bXb += nb * (vb - vb1);
        const double vbb = nb * bX;
        const double vb1b = vb1b_in - nb * bX;
        // vb1 = SM bX + v1 bY1 + w1 bZ1
        SMb += vb1b * bX;
        bXb += vb1b * SM;
        const double v1b = sb.v1 + vb1b * bY1;
        const double bY1b = sb.bY1 + vb1b * v1;
        const double w1b = sb.w1 + vb1b * bZ1;
        const double bZ1b = sb.bZ1 + vb1b * w1;
        // vb = u bX + v bY + w bZ
        ub += vbb * bX;
        bXb += vbb * u;
        vbr += vbb * bY;
        bYb += vbb * v;
        wb += vbb * bZ;
        bZb += vbb * w;
        // bZ1 = bZ N / D, bY1 = bY N / D
        bZb += bZ1b * N / D;
        double Nb = bZ1b * bZ / D;
        double Db = -bZ1b * bZ1 / D;
        bYb += bY1b * N / D;
        Nb += bY1b * bY / D;
        Db -= bY1b * bY1 / D;
        // w1 = w - bX bZ (SM - u) / D, v1 = v - bX bY (SM - u) / D
        const double q = (SM - u) / D;
        wb += w1b;
        bXb -= w1b * bZ * q;
        bZb -= w1b * bX * q;
        SMb -= w1b * bX * bZ / D;
        ub += w1b * bX * bZ / D;
        Db += w1b * bX * bZ * q / D;
        vbr += v1b;
        bXb -= v1b * bY * q;
        bYb -= v1b * bX * q;
        SMb -= v1b * bX * bY / D;
        ub += v1b * bX * bY / D;
        Db += v1b * bX * bY * q / D;
        // N = rho a a - bX bX
        rhob += Nb * a * a;
        ab += Nb * 2.0 * rho * a;
        bXb -= Nb * 2.0 * bX;
        // D = rho a (S - SM) - bX bX + EPS
        rhob += Db * a * (S - SM);
        ab += Db * rho * (S - SM);
        Sb += Db * rho * a;
        SMb -= Db * rho * a;
        bXb -= Db * 2.0 * bX;
        // rho1 = rho a / dS
        rhob += sb.rho1 * a / dS;
        ab += sb.rho1 * rho / dS;
        dSb -= sb.rho1 * rho1 / dS;
        // dS = S - SM + EPS
        Sb += dSb;
        SMb -= dSb;
    };
    star_side(Rsb, rhoR, uR, vR, wR, bXR, bYR, bZR, eR, pTR, SR, aR, dSR, rho1R, DR, NR, v1R, w1R, bY1R, bZ1R, vbR,
              vb1R, e1R, vb1Rb, rhoRb, uRb, vRb, wRb, bXRb, bYRb, bZRb, eRb, pTRb, SRb, aRb);
    star_side(Lsb, rhoL, uL, vL, wL, bXL, bYL, bZL, eL, pTL, SL, aL, dSL, rho1L, DL, NL, v1L, w1L, bY1L, bZ1L, vbL,
              vb1L, e1L, vb1Lb, rhoLb, uLb, vLb, wLb, bXLb, bYLb, bZLb, eLb, pTLb, SLb, aLb);

    // pT1 = (aR rhoR pTL - aL rhoL pTR + rhoL rhoR aR aL (uR - uL)) / den
    double denb;
    {
        const double nb = pT1b / den;
        denb = -pT1b * pT1 / den;
        const double du = uR - uL;
        aRb += nb * (rhoR * pTL + rhoL * rhoR * aL * du);
        rhoRb += nb * (aR * pTL + rhoL * aR * aL * du);
        pTLb += nb * aR * rhoR;
        aLb += nb * (-rhoL * pTR + rhoL * rhoR * aR * du);
        rhoLb += nb * (-aL * pTR + rhoR * aR * aL * du);
        pTRb -= nb * aL * rhoL;
        uRb += nb * rhoL * rhoR * aR * aL;
        uLb -= nb * rhoL * rhoR * aR * aL;
    }
    // SM = (aR rhoR uR - aL rhoL uL - pTR + pTL) / den
    {
        const double nb = SMb / den;
        denb -= SMb * SM / den;
        aRb += nb * rhoR * uR;
        rhoRb += nb * aR * uR;
        uRb += nb * aR * rhoR;
        aLb -= nb * rhoL * uL;
        rhoLb -= nb * aL * uL;
        uLb -= nb * aL * rhoL;
        pTRb -= nb;
        pTLb += nb;
    }
    // den = aR rhoR - aL rhoL + EPS
    aRb += denb * rhoR;
    rhoRb += denb * aR;
    aLb -= denb * rhoL;
    rhoLb -= denb * aL;
    // aR = SR - uR, aL = SL - uL
    SRb += aRb;
    uRb -= aRb;
    SLb += aLb;
    uLb -= aLb;
    // clamps, then SL0 = umin - cfm, SR0 = umax + cfm
    const double SL0b = SL_clamped ? 0.0 : SLb;
    const double SR0b = SR_clamped ? 0.0 : SRb;
    const double cfmb = SR0b - SL0b;
    if (umin_R) uRb += SL0b; else uLb += SL0b;
    if (umax_R) uRb += SR0b; else uLb += SR0b;
    double cfLb = 0.0, cfRb = 0.0;
    if (cfm_R) cfRb = cfmb; else cfLb = cfmb;
    double pLb = 0.0, pRb = 0.0;
    fast_speed_adj(rhoL, bXL, bYL, bZL, pL, gm, cfL, cfLb, rhoLb, bXLb, bYLb, bZLb, pLb);
    fast_speed_adj(rhoR, bXR, bYR, bZR, pR, gm, cfR, cfRb, rhoRb, bXRb, bYRb, bZRb, pRb);
    // pT = p + |B|^2 / 2 ; e = p / (gm - 1) + rho |u|^2 / 2 + |B|^2 / 2
    pLb += pTLb + eLb / (gm - 1.0);
    rhoLb += eLb * 0.5 * (uL * uL + vL * vL + wL * wL);
    uLb += eLb * rhoL * uL;
    vLb += eLb * rhoL * vL;
    wLb += eLb * rhoL * wL;
    bXLb += (pTLb + eLb) * bXL;
    bYLb += (pTLb + eLb) * bYL;
    bZLb += (pTLb + eLb) * bZL;
    pRb += pTRb + eRb / (gm - 1.0);
    rhoRb += eRb * 0.5 * (uR * uR + vR * vR + wR * wR);
    uRb += eRb * rhoR * uR;
    vRb += eRb * rhoR * vR;
    wRb += eRb * rhoR * wR;
    bXRb += (pTRb + eRb) * bXR;
    bYRb += (pTRb + eRb) * bYR;
    bZRb += (pTRb + eRb) * bZR;

    Lb[QR] += rhoLb; Lb[QU] += uLb; Lb[QV] += vLb; Lb[QW] += wLb;
    Lb[QBX] += bXLb; Lb[QBY] += bYLb; Lb[QBZ] += bZLb; Lb[QP] += pLb;
    Rb[QR] += rhoRb; Rb[QU] += uRb; Rb[QV] += vRb; Rb[QW] += wRb;
    Rb[QBX] += bXRb; Rb[QBY] += bYRb; Rb[QBZ] += bZRb; Rb[QP] += pRb;
}

}  // namespace adj
}  // namespace rmhd2d
