// adjoint_core.cuh -- reverse-mode derivatives of the per-interface
// arithmetic of the step: primitive recovery, MUSCL-minmod reconstruction
// and the HLLD flux.  Plain C++ on doubles, usable from device code and from
// host code.
//
// Each function recomputes the forward values it needs.  The values that
// decide a branch -- the primitives, the reconstructed states, minmod's
// choice, the wave speeds SL, SR, SM, S1L, S1R and with them the HLLD
// region -- are evaluated in the reference's order with explicitly rounded
// operations (never contracted into fused multiply-adds, whatever the
// compiler flags), so the branches taken are the ones the FP64 forward step
// took (hlld.cu:35-565, muscl.cu:6-126, minmod.hpp:6-16,
// calculate_half_Q.cu:4-38).  Adjoints are then propagated backwards
// through the branch taken, with reciprocals in place of divisions.
// Derivatives are those of the exact formulas (cs*cs is differentiated as
// gamma*p/rho); where a formula is not differentiable (sqrt at 0) the
// derivative of that term is taken as 0.
#pragma once

#include <math.h>

#if defined(__CUDACC__)
#define ADJ_FN __host__ __device__ __forceinline__
#else
#define ADJ_FN inline
#endif

// Correctly rounded single operations, kept out of any contraction.  A host
// build that models the device's rounding (contracting everything else)
// defines RMHD_ADJ_HOST_RN and supplies __dadd_rn and the others.
#if defined(__CUDA_ARCH__) || defined(RMHD_ADJ_HOST_RN)
#define XADD(a, b) __dadd_rn((a), (b))
#define XSUB(a, b) __dsub_rn((a), (b))
#define XMUL(a, b) __dmul_rn((a), (b))
#define XDIV(a, b) __ddiv_rn((a), (b))
#define XSQRT(a) __dsqrt_rn(a)
#else
#define XADD(a, b) ((a) + (b))
#define XSUB(a, b) ((a) - (b))
#define XMUL(a, b) ((a) * (b))
#define XDIV(a, b) ((a) / (b))
#define XSQRT(a) sqrt(a)
#endif

namespace rmhd2d {
namespace adj {

// BasicParameter order (basic_parameter_struct.hpp:5-27).
enum { QR = 0, QU = 1, QV = 2, QW = 3, QBX = 4, QBY = 5, QBZ = 6, QP = 7 };

// The seven reconstructed components, in the reference's loop order.
ADJ_FN int recon_comp(int n) { return n < 4 ? n : n + 1; }

ADJ_FN double sgn_d(double x) { return (double)((x > 0.0) - (x < 0.0)); }

// 1/a for the reverse sweep: on the device the hardware seed refined by two
// Newton-Raphson steps x' = x + x (1 - a x) (each squares the relative
// error), on the host a division.
ADJ_FN double adj_rcp(double a)
{
#if defined(__CUDA_ARCH__)
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(a));
    double e = fma(-a, r, 1.0);
    r = fma(r, e, r);
    e = fma(-a, r, 1.0);
    return fma(r, e, r);
#else
    return 1.0 / a;
#endif
}

// calculate_half_Q.cu:4-38 for a cell c (sweep order rho, m_n, m_t1, m_t2,
// b_n, b_t1, b_t2, e) and its neighbour's b_n.
ADJ_FN void basic_param(const double *c, double bn_next, double gm, double *q)
{
    const double rho = c[0];
    const double u = XDIV(c[1], rho), v = XDIV(c[2], rho), w = XDIV(c[3], rho);
    const double bX = c[4], bY = c[5], bZ = c[6], e = c[7];
    const double k2 = XADD(XADD(XMUL(u, u), XMUL(v, v)), XMUL(w, w));
    const double b2 = XADD(XADD(XMUL(bX, bX), XMUL(bY, bY)), XMUL(bZ, bZ));
    q[QP] = XMUL(XSUB(gm, 1.0), XSUB(XSUB(e, XMUL(0.5, XMUL(rho, k2))), XMUL(0.5, b2)));
    q[QR] = rho;
    q[QU] = u;
    q[QV] = v;
    q[QW] = w;
    q[QBX] = XMUL(0.5, XADD(bX, bn_next));
    q[QBY] = bY;
    q[QBZ] = bZ;
}

// Reverse of basic_param from its outputs q and the cell's own b_n: qb (8
// adjoints of q) -> cb (8 adjoints of the cell, accumulated).  The b_n of
// the next cell receives 0.5 * qb[QBX], which the caller routes.
ADJ_FN void basic_param_adj(const double *q, double bn_own, double gm, const double *qb, double *cb)
{
    const double ir = adj_rcp(q[QR]);
    const double u = q[QU], v = q[QV], w = q[QW];
    const double g1 = gm - 1.0;
    const double pb = qb[QP] * g1;
    cb[0] += qb[QR] - (qb[QU] * u + qb[QV] * v + qb[QW] * w) * ir + pb * 0.5 * (u * u + v * v + w * w);
    cb[1] += qb[QU] * ir - pb * u;
    cb[2] += qb[QV] * ir - pb * v;
    cb[3] += qb[QW] * ir - pb * w;
    cb[4] += 0.5 * qb[QBX] - pb * bn_own;
    cb[5] += qb[QBY] - pb * q[QBY];
    cb[6] += qb[QBZ] - pb * q[QBZ];
    cb[7] += pb;
}

// minmod.hpp:6-16 with the branch taken: 0 constant (sign change or below
// EPS), 1 the first argument, 2 the second.
ADJ_FN double minmod_sel(double x, double y, double eps, int &sel)
{
    const int s = (x > 0) - (x < 0);
    const double ax = fabs(x);
    const double sy = XMUL((double)s, y);
    const bool pick_y = sy < ax;          // thrust::min(ax, s*y)
    const double in = pick_y ? sy : ax;
    const bool clamp = in < eps;          // thrust::max(in, EPS)
    sel = (s == 0 || clamp) ? 0 : (pick_y ? 2 : 1);
    return XMUL((double)s, clamp ? eps : in);
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
        L[c] = XADD(q1[c], XMUL(0.5, minmod_sel(XSUB(q1[c], q0[c]), XSUB(q2[c], q1[c]), eps, sl)));
        R[c] = XSUB(q2[c], XMUL(0.5, minmod_sel(XSUB(q2[c], q1[c]), XSUB(q3[c], q2[c]), eps, sr)));
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
    const double t = -fb[7] * bX;   // adjoint of bX*u + bY*v + bZ*w
    sb.rho += u * (fb[0] + fb[1] * u + fb[2] * v + fb[3] * w);
    sb.u += rho * (fb[0] + 2.0 * fb[1] * u + fb[2] * v + fb[3] * w) + fb[5] * bY + fb[6] * bZ
          + fb[7] * (s.e + s.pT) + t * bX;
    sb.v += fb[2] * rho * u - fb[5] * bX + t * bY;
    sb.w += fb[3] * rho * u - fb[6] * bX + t * bZ;
    sb.pT += fb[1] + fb[7] * u;
    sb.e += fb[7] * u;
    sb.bX += -2.0 * fb[1] * bX - fb[2] * bY - fb[3] * bZ - fb[5] * v - fb[6] * w - fb[7] * (bX * u + bY * v + bZ * w)
           + t * u;
    sb.bY += -fb[2] * bX + fb[5] * u + t * v;
    sb.bZ += -fb[3] * bX + fb[6] * u + t * w;
}

// The fast magnetosonic speed cf = sqrt((cs2 + ca2 + sqrt((cs2 + ca2)^2 -
// 4 cs2 va2)) / 2), cs = sqrt(gm p / rho), ca = |B| / sqrt(rho),
// va = |bX| / sqrt(rho) (hlld.cu:290-310), in the reference's order.
ADJ_FN double fast_speed(double rho, double bX, double b2, double p, double gm)
{
    const double cs = XSQRT(XDIV(XMUL(gm, p), rho));
    const double ca = XSQRT(XDIV(b2, rho));
    const double va = XSQRT(XDIV(XMUL(bX, bX), rho));
    const double s = XADD(XMUL(cs, cs), XMUL(ca, ca));
    const double inner = XSUB(XMUL(s, s), XMUL(XMUL(XMUL(XMUL(4.0, cs), cs), va), va));
    return XSQRT(XMUL(0.5, XADD(s, XSQRT(inner))));
}

// Reverse of fast_speed.
ADJ_FN void fast_speed_adj(double rho, double bX, double bY, double bZ, double p, double gm, double cf, double cfb,
                           double &rhob, double &bXb, double &bYb, double &bZb, double &pb)
{
    if (cfb == 0.0 || !(cf > 0.0)) return;
    const double ir = adj_rcp(rho);
    const double cs2 = gm * p * ir, B2 = bX * bX + bY * bY + bZ * bZ, ca2 = B2 * ir, va2 = bX * bX * ir;
    const double s = cs2 + ca2;
    const double disc = s * s - 4.0 * cs2 * va2;
    const double rd = disc > 0.0 ? sqrt(disc) : 0.0;
    const double tb = 0.5 * cfb * adj_rcp(cf);
    double sb = 0.5 * tb;
    const double db = rd > 0.0 ? 0.25 * tb * adj_rcp(rd) : 0.0;
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

// Adjoints of the star quantities of one side of the fan.
struct SideBar {
    double rho1, v1, w1, bY1, bZ1, e1;
};

// Reverse of one side's star state (hlld.cu:330-392), s = L or R.
struct Side {
    double rho, u, v, w, bX, bY, bZ, e, pT;   // outer state
    double S, a, idS, rho1, iD, N, v1, w1, bY1, bZ1, vb, vb1, e1;
};

ADJ_FN void star_side_adj(const Side &x, const SideBar &sb, double vb1b_in, double SM, double pT1, double &SMb,
                          double &pT1b, St &ob, double &Sb, double &ab)
{
    // e1 = (a e - pT u + pT1 SM + bX (vb - vb1)) / dS
    const double nb = sb.e1 * x.idS;
    double dSb = -sb.e1 * x.e1 * x.idS;
    ab += nb * x.e;
    ob.e += nb * x.a;
    ob.pT -= nb * x.u;
    ob.u -= nb * x.pT;
    pT1b += nb * SM;
    SMb += nb * pT1;
    ob.bX += nb * (x.vb - x.vb1);
    const double vbb = nb * x.bX;
    const double vb1b = vb1b_in - nb * x.bX;
    // vb1 = SM bX + v1 bY1 + w1 bZ1
    SMb += vb1b * x.bX;
    ob.bX += vb1b * SM;
    const double v1b = sb.v1 + vb1b * x.bY1;
    const double bY1b = sb.bY1 + vb1b * x.v1;
    const double w1b = sb.w1 + vb1b * x.bZ1;
    const double bZ1b = sb.bZ1 + vb1b * x.w1;
    // vb = u bX + v bY + w bZ
    ob.u += vbb * x.bX;
    ob.bX += vbb * x.u;
    ob.v += vbb * x.bY;
    ob.bY += vbb * x.v;
    ob.w += vbb * x.bZ;
    ob.bZ += vbb * x.w;
    // bZ1 = bZ N / D, bY1 = bY N / D
    ob.bZ += bZ1b * x.N * x.iD;
    ob.bY += bY1b * x.N * x.iD;
    const double Nb = (bZ1b * x.bZ + bY1b * x.bY) * x.iD;
    double Db = -(bZ1b * x.bZ1 + bY1b * x.bY1) * x.iD;
    // w1 = w - bX bZ (SM - u) / D, v1 = v - bX bY (SM - u) / D
    const double q = (SM - x.u) * x.iD;
    ob.w += w1b;
    ob.v += v1b;
    const double tw = w1b * x.bZ + v1b * x.bY;   // shared bX (SM - u) / D factor
    ob.bX -= tw * q;
    ob.bZ -= w1b * x.bX * q;
    ob.bY -= v1b * x.bX * q;
    SMb -= tw * x.bX * x.iD;
    ob.u += tw * x.bX * x.iD;
    Db += tw * x.bX * q * x.iD;
    // N = rho a a - bX bX ; D = rho a (S - SM) - bX bX + EPS
    const double SmM = x.S - SM;
    ob.rho += Nb * x.a * x.a + Db * x.a * SmM;
    ab += Nb * 2.0 * x.rho * x.a + Db * x.rho * SmM;
    ob.bX -= (Nb + Db) * 2.0 * x.bX;
    Sb += Db * x.rho * x.a;
    SMb -= Db * x.rho * x.a;
    // rho1 = rho a / dS ; dS = S - SM + EPS
    ob.rho += sb.rho1 * x.a * x.idS;
    ab += sb.rho1 * x.rho * x.idS;
    dSb -= sb.rho1 * x.rho1 * x.idS;
    Sb += dSb;
    SMb -= dSb;
}

// Reverse of the HLLD flux (hlld.cu:35-131 CalculateFluxFunctor,
// hlld.cu:256-444 calculateHLLDParameterFunctor, hlld.cu:448-565
// setFluxFunctor): given fb = dJ/dflux, accumulates dJ/dL into Lb and dJ/dR
// into Rb (8 components each, BasicParameter order).  The flux is the
// indicator-weighted sum of six candidate fluxes; each selected candidate
// passes fb back through its state.
ADJ_FN void hlld_flux_adj(const double *L, const double *R, double gm, double EPS, const double *fb, double *Lb,
                          double *Rb)
{
    // ---- forward: branch-deciding values, exactly rounded ----
    Side l, r;
    l.rho = L[QR]; l.u = L[QU]; l.v = L[QV]; l.w = L[QW]; l.bX = L[QBX]; l.bY = L[QBY]; l.bZ = L[QBZ];
    r.rho = R[QR]; r.u = R[QU]; r.v = R[QV]; r.w = R[QW]; r.bX = R[QBX]; r.bY = R[QBY]; r.bZ = R[QBZ];
    const double pL = L[QP], pR = R[QP];
    const double b2L = XADD(XADD(XMUL(l.bX, l.bX), XMUL(l.bY, l.bY)), XMUL(l.bZ, l.bZ));
    const double b2R = XADD(XADD(XMUL(r.bX, r.bX), XMUL(r.bY, r.bY)), XMUL(r.bZ, r.bZ));
    l.pT = XADD(pL, XMUL(0.5, b2L));
    r.pT = XADD(pR, XMUL(0.5, b2R));
    const double cfL = fast_speed(l.rho, l.bX, b2L, pL, gm);
    const double cfR = fast_speed(r.rho, r.bX, b2R, pR, gm);
    // thrust::min(a, b) = b < a ? b : a, thrust::max(a, b) = a < b ? b : a
    const bool umin_R = r.u < l.u, umax_R = l.u < r.u, cfm_R = cfL < cfR;
    const double umin = umin_R ? r.u : l.u, umax = umax_R ? r.u : l.u, cfm = cfm_R ? cfR : cfL;
    const double SL0 = XSUB(umin, cfm), SR0 = XADD(umax, cfm);
    const bool SL_clamped = 0.0 < SL0, SR_clamped = SR0 < 0.0;
    l.S = SL_clamped ? 0.0 : SL0;
    r.S = SR_clamped ? 0.0 : SR0;
    l.a = XSUB(l.S, l.u);
    r.a = XSUB(r.S, r.u);
    const double den = XADD(XSUB(XMUL(r.a, r.rho), XMUL(l.a, l.rho)), EPS);
    const double SM = XDIV(XADD(XSUB(XSUB(XMUL(XMUL(r.a, r.rho), r.u), XMUL(XMUL(l.a, l.rho), l.u)), r.pT), l.pT), den);
    const double dSL = XADD(XSUB(l.S, SM), EPS), dSR = XADD(XSUB(r.S, SM), EPS);
    l.rho1 = XDIV(XMUL(l.rho, l.a), dSL);
    r.rho1 = XDIV(XMUL(r.rho, r.a), dSR);
    const double S1L = XSUB(SM, XSQRT(XDIV(XMUL(l.bX, l.bX), l.rho1)));
    const double S1R = XADD(SM, XSQRT(XDIV(XMUL(r.bX, r.bX), r.rho1)));
    const bool iOL = l.S > 0.0;
    const bool iML = (l.S <= 0.0) && (0.0 < S1L);
    const bool iIL = (S1L <= 0.0) && (0.0 < SM);
    const bool iOR = r.S <= 0.0;
    const bool iMR = (S1R <= 0.0) && (0.0 < r.S);
    const bool iIR = (SM <= 0.0) && (0.0 < S1R);

    // ---- forward: the rest of the fan ----
    const double ig1 = 1.0 / (gm - 1.0);
    l.e = pL * ig1 + 0.5 * l.rho * (l.u * l.u + l.v * l.v + l.w * l.w) + 0.5 * b2L;
    r.e = pR * ig1 + 0.5 * r.rho * (r.u * r.u + r.v * r.v + r.w * r.w) + 0.5 * b2R;
    const double iden = adj_rcp(den);
    const double du = r.u - l.u;
    const double pT1 = (r.a * r.rho * l.pT - l.a * l.rho * r.pT + l.rho * r.rho * r.a * l.a * du) * iden;
    l.idS = adj_rcp(dSL);
    r.idS = adj_rcp(dSR);
    auto star = [&](Side &x) {
        // D and N in the forward's rounding: where the fast and Alfven waves
        // meet, both are differences of nearly equal terms, and the ratios
        // N / D and (SM - u) / D linearised at contracted values differ
        // from the forward's at the 1e-6 level.
        x.iD = adj_rcp(XADD(XSUB(XMUL(XMUL(x.rho, x.a), XSUB(x.S, SM)), XMUL(x.bX, x.bX)), EPS));
        x.N = XSUB(XMUL(XMUL(x.rho, x.a), x.a), XMUL(x.bX, x.bX));
        const double q = (SM - x.u) * x.iD;
        x.v1 = x.v - x.bX * x.bY * q;
        x.w1 = x.w - x.bX * x.bZ * q;
        x.bY1 = x.bY * x.N * x.iD;
        x.bZ1 = x.bZ * x.N * x.iD;
        x.vb = x.u * x.bX + x.v * x.bY + x.w * x.bZ;
        x.vb1 = SM * x.bX + x.v1 * x.bY1 + x.w1 * x.bZ1;
        x.e1 = (x.a * x.e - x.pT * x.u + pT1 * SM + x.bX * (x.vb - x.vb1)) * x.idS;
    };
    star(l);
    star(r);
    const double sg = sgn_d(l.bX), sgL = sg, sgR = sgn_d(r.bX);
    const double sqL = sqrt(l.rho1), sqR = sqrt(r.rho1), sqLR = sqL * sqR;
    const double idd = adj_rcp(sqL + sqR + EPS);
    const double v2 = (sqL * l.v1 + sqR * r.v1 + (r.bY1 - l.bY1) * sg) * idd;
    const double w2 = (sqL * l.w1 + sqR * r.w1 + (r.bZ1 - l.bZ1) * sg) * idd;
    const double bY2 = (sqL * r.bY1 + sqR * l.bY1 + sqLR * (r.v1 - l.v1) * sg) * idd;
    const double bZ2 = (sqL * r.bZ1 + sqR * l.bZ1 + sqLR * (r.w1 - l.w1) * sg) * idd;
    const double vb2s = v2 * bY2 + w2 * bZ2;
    const double vb2L = SM * l.bX + vb2s, vb2R = SM * r.bX + vb2s;
    const double e2L = l.e1 - sqL * (l.vb1 - vb2L) * sgL;
    const double e2R = r.e1 + sqR * (r.vb1 - vb2R) * sgR;

    // ---- reverse ----
    St Lo{}, Ro{};                 // adjoints of the outer states (rho, u, ..., e, pT)
    SideBar Lsb{}, Rsb{};
    double SMb = 0.0, pT1b = 0.0, v2b = 0.0, w2b = 0.0, bY2b = 0.0, bZ2b = 0.0, e2Lb = 0.0, e2Rb = 0.0;
    // the fan region (at most one of ML, IL, IR, MR) through one flux reverse
    const int cand = iML ? 1 : (iIL ? 2 : (iIR ? 3 : (iMR ? 4 : 0)));
    if (cand) {
        const bool left = cand <= 2, dbl = cand == 2 || cand == 3;
        St st;
        st.rho = left ? l.rho1 : r.rho1;
        st.u = SM;
        st.v = dbl ? v2 : (left ? l.v1 : r.v1);
        st.w = dbl ? w2 : (left ? l.w1 : r.w1);
        st.bX = left ? l.bX : r.bX;
        st.bY = dbl ? bY2 : (left ? l.bY1 : r.bY1);
        st.bZ = dbl ? bZ2 : (left ? l.bZ1 : r.bZ1);
        st.e = cand == 1 ? l.e1 : (cand == 2 ? e2L : (cand == 3 ? e2R : r.e1));
        st.pT = pT1;
        St b{};
        one_flux_adj(st, fb, b);
        SMb += b.u;
        pT1b += b.pT;
        const double kl = left ? 1.0 : 0.0, kr = 1.0 - kl;        // side
        const double k2 = dbl ? 1.0 : 0.0, k1 = 1.0 - k2;         // double star / star
        Lsb.rho1 += kl * b.rho;
        Rsb.rho1 += kr * b.rho;
        Lo.bX += kl * b.bX;
        Ro.bX += kr * b.bX;
        v2b += k2 * b.v; w2b += k2 * b.w; bY2b += k2 * b.bY; bZ2b += k2 * b.bZ;
        e2Lb += (cand == 2 ? 1.0 : 0.0) * b.e;
        e2Rb += (cand == 3 ? 1.0 : 0.0) * b.e;
        Lsb.v1 += kl * k1 * b.v; Lsb.w1 += kl * k1 * b.w; Lsb.bY1 += kl * k1 * b.bY; Lsb.bZ1 += kl * k1 * b.bZ;
        Lsb.e1 += kl * k1 * b.e;
        Rsb.v1 += kr * k1 * b.v; Rsb.w1 += kr * k1 * b.w; Rsb.bY1 += kr * k1 * b.bY; Rsb.bZ1 += kr * k1 * b.bZ;
        Rsb.e1 += kr * k1 * b.e;
    }
    if (iOR) one_flux_adj(St{r.rho, r.u, r.v, r.w, r.bX, r.bY, r.bZ, r.e, r.pT}, fb, Ro);
    if (iOL) one_flux_adj(St{l.rho, l.u, l.v, l.w, l.bX, l.bY, l.bZ, l.e, l.pT}, fb, Lo);

    // double-star energies and state
    double sqLb = 0.0, sqRb = 0.0, sqLRb = 0.0, ddb = 0.0, vb1Lb, vb1Rb;
    {
        Rsb.e1 += e2Rb;
        sqRb += e2Rb * (r.vb1 - vb2R) * sgR;
        vb1Rb = e2Rb * sqR * sgR;
        const double vb2Rb = -vb1Rb;
        Lsb.e1 += e2Lb;
        sqLb -= e2Lb * (l.vb1 - vb2L) * sgL;
        vb1Lb = -e2Lb * sqL * sgL;
        const double vb2Lb = -vb1Lb;
        SMb += vb2Rb * r.bX + vb2Lb * l.bX;
        Ro.bX += vb2Rb * SM;
        Lo.bX += vb2Lb * SM;
        const double vb2b = vb2Rb + vb2Lb;
        v2b += vb2b * bY2;
        bY2b += vb2b * v2;
        w2b += vb2b * bZ2;
        bZ2b += vb2b * w2;

        double nb = bZ2b * idd;
        ddb -= bZ2b * bZ2 * idd;
        sqLb += nb * r.bZ1; Rsb.bZ1 += nb * sqL; sqRb += nb * l.bZ1; Lsb.bZ1 += nb * sqR;
        sqLRb += nb * (r.w1 - l.w1) * sg; Rsb.w1 += nb * sqLR * sg; Lsb.w1 -= nb * sqLR * sg;

        nb = bY2b * idd;
        ddb -= bY2b * bY2 * idd;
        sqLb += nb * r.bY1; Rsb.bY1 += nb * sqL; sqRb += nb * l.bY1; Lsb.bY1 += nb * sqR;
        sqLRb += nb * (r.v1 - l.v1) * sg; Rsb.v1 += nb * sqLR * sg; Lsb.v1 -= nb * sqLR * sg;

        nb = w2b * idd;
        ddb -= w2b * w2 * idd;
        sqLb += nb * l.w1; Lsb.w1 += nb * sqL; sqRb += nb * r.w1; Rsb.w1 += nb * sqR;
        Rsb.bZ1 += nb * sg; Lsb.bZ1 -= nb * sg;

        nb = v2b * idd;
        ddb -= v2b * v2 * idd;
        sqLb += nb * l.v1; Lsb.v1 += nb * sqL; sqRb += nb * r.v1; Rsb.v1 += nb * sqR;
        Rsb.bY1 += nb * sg; Lsb.bY1 -= nb * sg;

        // sqLR = sqL sqR, dd = sqL + sqR + EPS, sq = sqrt(rho1)
        sqLb += ddb + sqLRb * sqR;
        sqRb += ddb + sqLRb * sqL;
        if (sqL > 0.0) Lsb.rho1 += 0.5 * sqLb * adj_rcp(sqL);
        if (sqR > 0.0) Rsb.rho1 += 0.5 * sqRb * adj_rcp(sqR);
    }

    double SLb = 0.0, SRb = 0.0, aLb = 0.0, aRb = 0.0;
    star_side_adj(r, Rsb, vb1Rb, SM, pT1, SMb, pT1b, Ro, SRb, aRb);
    star_side_adj(l, Lsb, vb1Lb, SM, pT1, SMb, pT1b, Lo, SLb, aLb);

    // pT1 = (aR rhoR pTL - aL rhoL pTR + rhoL rhoR aR aL (uR - uL)) / den
    double denb;
    {
        const double nb = pT1b * iden;
        denb = -pT1b * pT1 * iden;
        const double rr = l.rho * r.rho;
        aRb += nb * (r.rho * l.pT + rr * l.a * du);
        Ro.rho += nb * (r.a * l.pT + l.rho * r.a * l.a * du);
        Lo.pT += nb * r.a * r.rho;
        aLb += nb * (-l.rho * r.pT + rr * r.a * du);
        Lo.rho += nb * (-l.a * r.pT + r.rho * r.a * l.a * du);
        Ro.pT -= nb * l.a * l.rho;
        Ro.u += nb * rr * r.a * l.a;
        Lo.u -= nb * rr * r.a * l.a;
    }
    // SM = (aR rhoR uR - aL rhoL uL - pTR + pTL) / den
    {
        const double nb = SMb * iden;
        denb -= SMb * SM * iden;
        aRb += nb * r.rho * r.u;
        Ro.rho += nb * r.a * r.u;
        Ro.u += nb * r.a * r.rho;
        aLb -= nb * l.rho * l.u;
        Lo.rho -= nb * l.a * l.u;
        Lo.u -= nb * l.a * l.rho;
        Ro.pT -= nb;
        Lo.pT += nb;
    }
    // den = aR rhoR - aL rhoL + EPS ; a = S - u
    aRb += denb * r.rho;
    Ro.rho += denb * r.a;
    aLb -= denb * l.rho;
    Lo.rho -= denb * l.a;
    SRb += aRb;
    Ro.u -= aRb;
    SLb += aLb;
    Lo.u -= aLb;
    // clamps, then SL0 = umin - cfm, SR0 = umax + cfm
    const double SL0b = SL_clamped ? 0.0 : SLb;
    const double SR0b = SR_clamped ? 0.0 : SRb;
    const double cfmb = SR0b - SL0b;
    Ro.u += (umin_R ? SL0b : 0.0) + (umax_R ? SR0b : 0.0);
    Lo.u += (umin_R ? 0.0 : SL0b) + (umax_R ? 0.0 : SR0b);
    double pLb = 0.0, pRb = 0.0;
    fast_speed_adj(l.rho, l.bX, l.bY, l.bZ, pL, gm, cfL, cfm_R ? 0.0 : cfmb, Lo.rho, Lo.bX, Lo.bY, Lo.bZ, pLb);
    fast_speed_adj(r.rho, r.bX, r.bY, r.bZ, pR, gm, cfR, cfm_R ? cfmb : 0.0, Ro.rho, Ro.bX, Ro.bY, Ro.bZ, pRb);
    // pT = p + |B|^2 / 2 ; e = p / (gm - 1) + rho |u|^2 / 2 + |B|^2 / 2
    pLb += Lo.pT + Lo.e * ig1;
    pRb += Ro.pT + Ro.e * ig1;
    const double cL = Lo.pT + Lo.e, cR = Ro.pT + Ro.e;

    Lb[QR] += Lo.rho + Lo.e * 0.5 * (l.u * l.u + l.v * l.v + l.w * l.w);
    Lb[QU] += Lo.u + Lo.e * l.rho * l.u;
    Lb[QV] += Lo.v + Lo.e * l.rho * l.v;
    Lb[QW] += Lo.w + Lo.e * l.rho * l.w;
    Lb[QBX] += Lo.bX + cL * l.bX;
    Lb[QBY] += Lo.bY + cL * l.bY;
    Lb[QBZ] += Lo.bZ + cL * l.bZ;
    Lb[QP] += pLb;
    Rb[QR] += Ro.rho + Ro.e * 0.5 * (r.u * r.u + r.v * r.v + r.w * r.w);
    Rb[QU] += Ro.u + Ro.e * r.rho * r.u;
    Rb[QV] += Ro.v + Ro.e * r.rho * r.v;
    Rb[QW] += Ro.w + Ro.e * r.rho * r.w;
    Rb[QBX] += Ro.bX + cR * r.bX;
    Rb[QBY] += Ro.bY + cR * r.bY;
    Rb[QBZ] += Ro.bZ + cR * r.bZ;
    Rb[QP] += pRb;
}

}  // namespace adj
}  // namespace rmhd2d
