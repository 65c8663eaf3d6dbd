// adjoint.cuh -- reverse-mode (adjoint) forms of the step's routines.
//
// Each `*_b` function takes the forward inputs of its routine, recomputes the
// forward intermediates with the same arithmetic (so every branch -- dry/wet
// tests, limiter cases, wall and static-friction decisions, min/max picks --
// is the one the forward pass took), and maps adjoints of the outputs to
// adjoints of the inputs. Material-parameter adjoints are accumulated into
// pb[NPB] (phi in radians, kref, alpha_c, mu). Time steps are data, not
// variables: their adjoints are not formed.
//
// Conventions: a `_b` suffix is an adjoint. Adjoint arguments passed by
// reference are accumulated into (+=) unless the comment says "replaced".
// fmax2(a, b) = a > b ? a : b and fmin2(a, b) = a < b ? a : b, so the
// adjoint of a max/min goes to the operand the forward returned.
#pragma once
#include "stages.cuh"

namespace dclaw {

enum { PB_PHI = 0, PB_KREF = 1, PB_ALPHA = 2, PB_MU = 3, NPB = 4 };

// d sqrt(x) for x = s*s > 0; 0 where the forward value is 0 (the callers'
// zero-depth states are constants of their branch)
DC_HD double dsqrt_b(double s, double sb) { return s > 0.0 ? 0.5 * sb / s : 0.0; }

// ---------------------------------------------------------------------------
// qfix. Inputs (h, hu, hv, hm, p) before qfix; on entry hb..pb hold adjoints
// of the outputs (h, hu, hv, hm, p) and ub, vb, mb adjoints of (u, v, m); on
// return hb..pb are replaced by adjoints of the inputs.
DC_HD void qfix_b(const dclaw_params& P, double h, double hu, double hv, double hm, double p, double gz,
                  double& hb, double& hub, double& hvb, double& hmb, double& pb, double ub, double vb, double mb) {
    if (h <= P.dry_tolerance) {
        hb = 0.0; hub = 0.0; hvb = 0.0; hmb = 0.0; pb = 0.0;
        return;
    }
    double u = hu / h, v = hv / h, m0 = hm / h;
    double m1 = fmax2(m0, 0.0);
    double m = fmin2(m1, 1.0);
    double rho = P.rho_s * m + (1.0 - m) * P.rho_f;
    double pmax = rho * gz * h;
    double p1 = fmax2(0.0, p);
    double pmaxb = 0.0, p1b = 0.0;
    if (pmax < p1) pmaxb = pb; else p1b = pb;
    double pin_b = (0.0 > p) ? 0.0 : p1b;
    double rhob = pmaxb * gz * h;
    double h_b = hb + pmaxb * rho * gz;
    double m_b = mb + rhob * (P.rho_s - P.rho_f);
    h_b += hmb * m;
    m_b += hmb * h;
    double m1b = (m1 < 1.0) ? m_b : 0.0;
    double m0b = (m0 > 0.0) ? m1b : 0.0;
    double hm_b = m0b / h;
    h_b -= m0b * m0 / h;
    double hu_b = hub + ub / h;
    h_b -= ub * u / h;
    double hv_b = hvb + vb / h;
    h_b -= vb * v / h;
    hb = h_b; hub = hu_b; hvb = hv_b; hmb = hm_b; pb = pin_b;
}

// qfix_mp on a wet cell: inputs (h, hm, p); hmb, pb hold adjoints of the
// outputs (hm, p), mb of m; replaced by adjoints of the inputs hm, p; hb += .
DC_HD void qfix_mp_b(const dclaw_params& P, double h, double hm, double p, double gz, double& hb, double& hmb,
                     double& pb, double mb) {
    double m0 = hm / h;
    double m1 = fmax2(m0, 0.0);
    double m = fmin2(m1, 1.0);
    double rho = P.rho_s * m + (1.0 - m) * P.rho_f;
    double pmax = rho * gz * h;
    double p1 = fmax2(0.0, p);
    double pmaxb = 0.0, p1b = 0.0;
    if (pmax < p1) pmaxb = pb; else p1b = pb;
    double pin_b = (0.0 > p) ? 0.0 : p1b;
    double rhob = pmaxb * gz * h;
    hb += pmaxb * rho * gz;
    double m_b = mb + rhob * (P.rho_s - P.rho_f);
    hb += hmb * m;
    m_b += hmb * h;
    double m1b = (m1 < 1.0) ? m_b : 0.0;
    double m0b = (m0 > 0.0) ? m1b : 0.0;
    double hm_b = m0b / h;
    hb -= m0b * m0 / h;
    hmb = hm_b;
    pb = pin_b;
}

// qfix_cmass. Inputs m, p_exc, u, v, rhoh (h, p, rho, hu, hv, hm are
// outputs only). Output adjoints hb, mb, pb, rhob, pexb, hub, hvb, hmb;
// returns input adjoints: mb, pexb replaced; ub, vb, rhohb accumulated.
DC_HD void qfix_cmass_b(const dclaw_params& P, double m, double p_exc, double u, double v, double rhoh, double gz,
                        double hb, double& mb, double pb, double rhob, double& pexb, double hub, double hvb,
                        double hmb, double& ub, double& vb, double& rhohb) {
    double m1 = fmax2(m, 0.0);
    double m2 = fmin2(m1, 1.0);
    double rho = m2 * (P.rho_s - P.rho_f) + P.rho_f;
    double h = rhoh / rho;
    double pe_max = rhoh * gz - P.rho_f * h * gz;
    double pe_min = 0.0 - P.rho_f * h * gz;
    double pe1 = fmax2(pe_min, p_exc);
    double pe2 = fmin2(pe_max, pe1);
    // hu = h u, hv = h v, hm = h m2, p = rho_f gz h + pe2
    double h_b = hb + hub * u + hvb * v + hmb * m2 + pb * P.rho_f * gz;
    ub += hub * h;
    vb += hvb * h;
    double m2b = mb + hmb * h;
    double pe2b = pexb + pb;
    double pe_maxb = 0.0, pe1b = 0.0;
    if (pe_max < pe1) pe_maxb = pe2b; else pe1b = pe2b;
    double pe_minb = 0.0, pin_b = 0.0;
    if (pe_min > p_exc) pe_minb = pe1b; else pin_b = pe1b;
    rhohb += pe_maxb * gz;
    h_b += -pe_maxb * P.rho_f * gz - pe_minb * P.rho_f * gz;
    // h = rhoh / rho
    rhohb += h_b / rho;
    double rho_b = rhob - h_b * h / rho;
    m2b += rho_b * (P.rho_s - P.rho_f);
    double m1b = (m1 < 1.0) ? m2b : 0.0;
    mb = (m > 0.0) ? m1b : 0.0;
    pexb = pin_b;
}

// ---------------------------------------------------------------------------
// setvars. Output adjoints in `ob` (rho, kperm, alphainv, m_eq, tanpsi, tau);
// accumulates input adjoints phib, hb, ub, vb, mb, pb_ and parameters pbar.
template <bool NEED_ALL>
DC_HD void setvars_b(const dclaw_params& P, double phi, double h, double u, double v, double m, double p,
                     double gz, const SetVars& ob, double& phib, double& hb, double& ub, double& vb, double& mb,
                     double& p_b, double* pbar) {
    const double rs = P.rho_s, rf = P.rho_f;
    double rho = m * (rs - rf) + rf;
    double ek = 0.0;
    if (NEED_ALL) ek = em::d_exp(-(m - P.mref) / (0.04));
    double a = rho * gz * h - p;
    double sig_eff = fmax2(0.0, a);
    double sig_0 = 0.0;
    if (P.alphamethod == 0) sig_0 = P.sigma_0;
    else if (P.alphamethod == 1) sig_0 = 0.50 * P.alpha_c * rf * (rs - rf) * gz * h / rho;
    double S = sig_eff + sig_0;
    double alphainv = m * S / P.alpha_c;
    double vnorm = sqrt(sq(u) + sq(v));
    double shear = (h > P.dry_tolerance) ? 2.0 * vnorm / h : 0.0;
    double Nden = rs * sq(shear * P.delta) + sig_eff;
    double Nnum = P.mu * shear;
    double sNd = 0.0, sNn = 0.0, m_eq;
    if (Nnum <= 0.0) m_eq = P.m_crit;
    else {
        sNd = sqrt(Nden);
        sNn = sqrt(Nnum);
        m_eq = P.m_crit * (sNd / (sNd + sNn));
    }
    double x = P.c1 * (m - m_eq);
    double t = em::d_tan(phi + em::d_atan(x));
    double tau0 = sig_eff * t;
    double th = em::d_tanh(100.0 * (m - 0.1));
    // reverse
    double rho_b = ob.rho;
    double m_b = 0.0, h_b = 0.0;
    double tau0b = ob.tau * 0.5 * (1.0 + th);
    double thb = ob.tau * tau0 * 0.5;
    m_b += thb * (1.0 - th * th) * 100.0;
    double sig_effb = tau0b * t;
    double argb = tau0b * sig_eff * (1.0 + t * t);
    phib += argb;
    double xb = ob.tanpsi + argb / (1.0 + x * x);
    m_b += xb * P.c1;
    double m_eqb = ob.m_eq - xb * P.c1;
    double shearb = 0.0;
    if (Nnum > 0.0) {
        double D = sNd + sNn;
        double sNdb = m_eqb * P.m_crit * sNn / (D * D);
        double sNnb = -m_eqb * P.m_crit * sNd / (D * D);
        double Ndenb = dsqrt_b(sNd, sNdb);
        double Nnumb = dsqrt_b(sNn, sNnb);
        pbar[PB_MU] += Nnumb * shear;
        shearb += Nnumb * P.mu;
        shearb += Ndenb * rs * 2.0 * (shear * P.delta) * P.delta;
        sig_effb += Ndenb;
    }
    if (h > P.dry_tolerance) {
        double vnormb = shearb * 2.0 / h;
        h_b -= shearb * shear / h;
        if (vnorm > 0.0) {
            ub += vnormb * u / vnorm;
            vb += vnormb * v / vnorm;
        }
    }
    double alphainvb = ob.alphainv;
    m_b += alphainvb * S / P.alpha_c;
    double Sb = alphainvb * m / P.alpha_c;
    pbar[PB_ALPHA] -= alphainvb * alphainv / P.alpha_c;
    sig_effb += Sb;
    if (P.alphamethod == 1) {
        pbar[PB_ALPHA] += Sb * sig_0 / P.alpha_c;
        h_b += Sb * sig_0 / h;
        rho_b -= Sb * sig_0 / rho;
    }
    if (!(0.0 > a)) {
        rho_b += sig_effb * gz * h;
        h_b += sig_effb * rho * gz;
        p_b -= sig_effb;
    }
    if (NEED_ALL) {
        double kb = ob.kperm;
        pbar[PB_KREF] += kb * ek;
        m_b += kb * P.kref * ek * (-1.0 / 0.04);
    }
    m_b += rho_b * (rs - rf);
    hb += h_b;
    mb += m_b;
}

// ---------------------------------------------------------------------------
// riemanntype: adjoints of (hm, s1m, s2m) to (hL, hR, uL, uR), accumulated.
DC_HD void riemanntype_b(double hL, double hR, double uL, double uR, double drytol, double g, double hmb,
                         double s1mb, double s2mb, double& hLb, double& hRb, double& uLb, double& uRb) {
    double h_min = fmin2(hR, hL);
    double h_max = fmax2(hR, hL);
    double delu = uR - uL;
    double delub = 0.0;
    if (h_min <= drytol) {
        double sb = s1mb + s2mb;
        uRb += sb;
        uLb += sb;
        double cR = sqrt(g * hR), cL = sqrt(g * hL);
        hRb += -2.0 * g * dsqrt_b(cR, sb);
        hLb += 2.0 * g * dsqrt_b(cL, sb);
        return;
    }
    double F_min = delu + 2.0 * (sqrt(g * h_min) - sqrt(g * h_max));
    double F_max = delu + (h_max - h_min) * (sqrt(.5 * g * (h_max + h_min) / (h_max * h_min)));
    double cL = sqrt(g * hL), cR = sqrt(g * hR);
    if (F_min > 0.0) {
        double X = -delu + 2.0 * (cL + cR);
        double Y = fmax2(0.0, X);
        double hm = (1.0 / (16.0 * g)) * sq(Y);
        double sghm = sqrt(g * hm);
        double sghmb = -3.0 * s1mb + 3.0 * s2mb;
        uLb += s1mb;
        hLb += 2.0 * g * dsqrt_b(cL, s1mb);
        uRb += s2mb;
        hRb += -2.0 * g * dsqrt_b(cR, s2mb);
        double hmt = hmb + g * dsqrt_b(sghm, sghmb);
        double Yb = hmt * (1.0 / (16.0 * g)) * 2.0 * Y;
        double Xb = (0.0 > X) ? 0.0 : Yb;
        delub -= Xb;
        hLb += 2.0 * g * dsqrt_b(cL, Xb);
        hRb += 2.0 * g * dsqrt_b(cR, Xb);
    } else if (F_max <= 0.0) {
        double H = h_max;
        double XL = .5 * g * (1.0 / H + 1.0 / hL), XR = .5 * g * (1.0 / H + 1.0 / hR);
        double gL = sqrt(XL), gR = sqrt(XR);
        double F0 = delu + (H - hL) * gL + (H - hR) * gR;
        double T1 = g * (H - hL) / (4.0 * (sq(H)) * gL);
        double T2 = g * (H - hR) / (4.0 * (sq(H)) * gR);
        double dfdh = gL - T1 + gR - T2;
        double sH = sqrt(H);
        double slope = 2.0 * sH * dfdh;
        double Z = sH - F0 / slope;
        double hm = sq(Z);
        double A1 = sqrt((.5 * g) * (1.0 / hm + 1.0 / hL));
        double A2 = sqrt((.5 * g) * (1.0 / hm + 1.0 / hR));
        double sghm = sqrt(g * hm);
        double u1mb = s1mb, u2mb = s2mb;
        double sghmb = -s1mb + s2mb;
        double hmt = hmb + g * dsqrt_b(sghm, sghmb);
        // u1m = uL - (hm - hL) A1
        uLb += u1mb;
        hmt += -u1mb * A1;
        hLb += u1mb * A1;
        double A1b = -u1mb * (hm - hL);
        double X1b = dsqrt_b(A1, A1b);
        hmt += X1b * .5 * g * (-1.0 / (hm * hm));
        hLb += X1b * .5 * g * (-1.0 / (hL * hL));
        // u2m = uR + (hm - hR) A2
        uRb += u2mb;
        hmt += u2mb * A2;
        hRb -= u2mb * A2;
        double A2b = u2mb * (hm - hR);
        double X2b = dsqrt_b(A2, A2b);
        hmt += X2b * .5 * g * (-1.0 / (hm * hm));
        hRb += X2b * .5 * g * (-1.0 / (hR * hR));
        // hm = Z^2, Z = sH - F0/slope
        double Zb = hmt * 2.0 * Z;
        double sHb = Zb;
        double F0b = -Zb / slope;
        double slopeb = Zb * F0 / (slope * slope);
        sHb += slopeb * 2.0 * dfdh;
        double dfdhb = slopeb * 2.0 * sH;
        double Hb = dsqrt_b(sH, sHb);
        double gLb = dfdhb, gRb = dfdhb;
        double T1b = -dfdhb, T2b = -dfdhb;
        // T = g (H - hX) / (4 H^2 gX)
        Hb += T1b * (g / (4.0 * H * H * gL)) * (1.0 - 2.0 * (H - hL) / H);
        hLb += T1b * (-g / (4.0 * H * H * gL));
        gLb += T1b * (-T1 / gL);
        Hb += T2b * (g / (4.0 * H * H * gR)) * (1.0 - 2.0 * (H - hR) / H);
        hRb += T2b * (-g / (4.0 * H * H * gR));
        gRb += T2b * (-T2 / gR);
        // F0
        delub += F0b;
        Hb += F0b * (gL + gR);
        hLb -= F0b * gL;
        hRb -= F0b * gR;
        gLb += F0b * (H - hL);
        gRb += F0b * (H - hR);
        double XLb = dsqrt_b(gL, gLb), XRb = dsqrt_b(gR, gRb);
        Hb += (XLb + XRb) * .5 * g * (-1.0 / (H * H));
        hLb += XLb * .5 * g * (-1.0 / (hL * hL));
        hRb += XRb * .5 * g * (-1.0 / (hR * hR));
        if (hR > hL) hRb += Hb; else hLb += Hb;
    } else {
        // one secant step from h_min: F0 = delu + 2 (sqrt(g h_min) - sqrt(g h_max)) + 0
        double sgmin = sqrt(g * h_min), sgmax = sqrt(g * h_max);
        double F0 = delu + 2.0 * (sgmin - sgmax);
        double dh = h_max - h_min;
        double Q = sqrt(.5 * g * (h_max + h_min) / (h_max * h_min));
        double slope = (F_max - F0) / dh;
        double hm = h_min - F0 / slope;
        double sghm = sqrt(g * hm);
        double sghmb, ab;
        if (hL > hR) {
            ab = s1mb + s2mb;
            sghmb = -3.0 * s1mb - s2mb;
            uLb += ab;
            hLb += 2.0 * g * dsqrt_b(cL, ab);
        } else {
            ab = s1mb + s2mb;
            sghmb = 3.0 * s2mb + s1mb;
            uRb += ab;
            hRb += -2.0 * g * dsqrt_b(cR, ab);
        }
        double hmt = hmb + g * dsqrt_b(sghm, sghmb);
        double hminb = hmt;
        double F0b = -hmt / slope;
        double slopeb = hmt * F0 / (slope * slope);
        double Fmaxb = slopeb / dh;
        F0b -= slopeb / dh;
        double dhb = -slopeb * slope / dh;
        // F_max = delu + dh * Q,  Q = sqrt(.5 g (hmax + hmin) / (hmax hmin))
        delub += Fmaxb;
        dhb += Fmaxb * Q;
        double Qb = Fmaxb * dh;
        double Xq = .5 * g * (h_max + h_min) / (h_max * h_min);
        double Xqb = dsqrt_b(Q, Qb);
        // Xq = .5 g (hmax + hmin) / (hmax hmin) = .5 g (1/hmin + 1/hmax)
        double hmaxb = Xqb * (.5 * g / (h_max * h_min) - Xq / h_max);
        hminb += Xqb * (.5 * g / (h_max * h_min) - Xq / h_min);
        hmaxb += dhb;
        hminb -= dhb;
        delub += F0b;
        hminb += 2.0 * g * dsqrt_b(sgmin, F0b);
        hmaxb += -2.0 * g * dsqrt_b(sgmax, F0b);
        if (hR > hL) { hRb += hmaxb; hLb += hminb; }
        else { hLb += hmaxb; hRb += hminb; }
    }
    uRb += delub;
    uLb -= delub;
}

// ---------------------------------------------------------------------------
struct SideB {
    double h, hn, ht, hm, p, un, ut, m, b, taudir, fs, rho_sv, tau_sv;
};

DC_HD void zero_sideb(SideB& s) {
    s.h = s.hn = s.ht = s.hm = s.p = s.un = s.ut = s.m = s.b = s.taudir = s.fs = s.rho_sv = s.tau_sv = 0.0;
}

// riemann_solve reverse: wb adjoints of the 15 wave outputs; accumulates
// into Lb, Rb. With the rare-wave corrector (riemannsolvers_dclaw.f:
// 169-195, 365-386) it follows the forward's choice of the middle speed
// (s1m, s2m or their mean) and of the eigenvector system.
DC_HD bool riemann_solve_b(const dclaw_params& P, const Side& L, const Side& R, const Waves& wb, SideB& Lb,
                           SideB& Rb) {
    const double grav = P.grav;
    const double drytol = P.dry_tolerance;
    double wall1 = 1.0, wall2 = 1.0, wall3 = 1.0;
    bool wallprob = false;
    int pre = 0;  // 0: none, 1: R dry, 2: L dry
    double hL = L.h, hR = R.h, huL = L.hn, huR = R.hn, hvL = L.ht, hvR = R.ht;
    double hmL = L.hm, hmR = R.hm, pL = L.p, pR = R.p, bL = L.b, bR = R.b;
    double uL = L.un, uR = R.un, vL = L.ut, vR = R.ut, mL = L.m, mR = R.m;
    double rhoL_sv = L.rho_sv, tauL_sv = L.tau_sv, rhoR_sv = R.rho_sv, tauR_sv = R.tau_sv;
    if (hR <= drytol) {
        pre = 1;
        hR = 0.0; pR = 0.0; mR = mL;
        RType t = riemanntype(hL, hL, uL, -uL, drytol, grav);
        double hstartest = fmax2(hL, t.hm);
        if (hstartest + bL < bR) {
            wall2 = 0.0; wall3 = 0.0;
            wallprob = true;
            hR = hL; huR = -huL; hvR = hvL; hmR = hmL; bR = bL;
            uR = -uL; vR = vL; mR = mL; pR = pL;
            rhoR_sv = rhoL_sv; tauR_sv = tauL_sv;
        }
    } else if (hL <= drytol) {
        pre = 2;
        hL = 0.0; pL = 0.0; mL = mR;
        RType t = riemanntype(hR, hR, -uR, uR, drytol, grav);
        double hstartest = fmax2(hR, t.hm);
        if (hstartest + bR < bL) {
            wall1 = 0.0; wall2 = 0.0;
            wallprob = true;
            hL = hR; huL = -huR; hvL = hvR; hmL = hmR; mL = mR; bL = bR;
            uL = -uR; vL = vR; pL = pR;
            rhoL_sv = rhoR_sv; tauL_sv = tauR_sv;
        }
    }
    const double criticaltol = fmax2(drytol * grav, 1e-6);
    const double criticaltol_2 = sqrt(criticaltol);
    const double gz = grav;
    int rcase;
    double rhoL, rhoR, tauL0, tauR0;
    if (hL >= drytol && hR >= drytol) {
        rcase = 0;
        rhoL = rhoL_sv; tauL0 = tauL_sv; rhoR = rhoR_sv; tauR0 = tauR_sv;
    } else if (hL >= drytol) {
        rcase = 1;
        rhoL = rhoL_sv; tauL0 = tauL_sv; rhoR = rhoL_sv; tauR0 = 0.5 * tauL0;
    } else {
        rcase = 2;
        rhoL = rhoR_sv; rhoR = rhoR_sv; tauR0 = tauR_sv; tauL0 = 0.5 * tauR0;
    }
    double tauL = L.fs * tauL0;
    double tauR = R.fs * tauR0;
    double rho = 0.5 * (rhoL + rhoR);
    double gamma, gammaL, gammaR;
    if (P.src2method == -1) {
        gamma = P.rho_f / rho; gammaL = P.rho_f / rhoL; gammaR = P.rho_f / rhoR;
    } else {
        gamma = 0.25 * (P.rho_f + 3.0 * rho) / rho;
        gammaL = 0.25 * (P.rho_f + 3.0 * rhoL) / rhoL;
        gammaR = 0.25 * (P.rho_f + 3.0 * rhoR) / rhoR;
    }
    const double geps = gz;
    double sqhL = sqrt(hL), sqhR = sqrt(hR);
    double cL = sqrt(geps * hL), cR = sqrt(geps * hR);
    double sL = uL - cL, sR = uR + cR;
    double Du = sqhR + sqhL;
    double uhat = (sqhL * uL + sqhR * uR) / Du;
    double chat = sqrt(geps * 0.5 * (hR + hL));
    double sRoe1 = uhat - chat, sRoe2 = uhat + chat;
    double sE1 = fmin2(sL, sRoe1);
    double sE2 = fmax2(sR, sRoe2);
    double u = uhat;
    RType rt = riemanntype(hL, hR, uL, uR, drytol, geps);
    double sw1 = fmin2(sE1, rt.s2m);
    double sw3 = fmax2(sE2, rt.s1m);
    double Dd = sE2 - sE1;
    double Qh = (huL - huR + sE2 * hR - sE1 * hL) / Dd;
    double hstarHLL = fmax2(Qh, 0.0);
    // the middle speed: the mean of sw1, sw3 (rsel 0) or the corrector's s1m
    // (1), s2m (2) or their mean (3); the corrector's eigenvectors when rc
    double sw2 = 0.5 * (sw3 + sw1);
    int rsel = 0;
    bool rc = false;
    if (P.rarecorrectortest) {
        double sdelta = sw3 - sw1;
        double raremin = 0.5, raremax = 0.9;
        if (rt.rare1 && sE1 * rt.s1m < 0.0) raremin = 0.2;
        if (rt.rare2 && sE2 * rt.s2m < 0.0) raremin = 0.2;
        if (rt.rare1 || rt.rare2) {
            double sghm = sqrt(geps * rt.hm);
            double rare1st = 3.0 * (cL - sghm);
            double rare2st = 3.0 * (cR - sghm);
            if (fmax2(rare1st, rare2st) > raremin * sdelta && fmax2(rare1st, rare2st) < raremax * sdelta) {
                rc = true;
                if (rare1st > rare2st) { sw2 = rt.s1m; rsel = 1; }
                else if (rare2st > rare1st) { sw2 = rt.s2m; rsel = 2; }
                else { sw2 = 0.5 * (rt.s1m + rt.s2m); rsel = 3; }
            }
        }
        if (hstarHLL < fmin2(hL, hR) / 5.0) rc = false;
    }
    double delb = (bR - bL);
    double hbar = 0.5 * (hL + hR);
    double s1s2bar = 0.25 * sq(uL + uR) - gz * hbar;
    double s1s2tilde = fmax2(0.0, uL * uR) - gz * hbar;
    const double ct2 = sq(criticaltol);
    bool sonic = false;
    if (fabs(s1s2bar) <= criticaltol) sonic = true;
    else if (s1s2bar * s1s2tilde <= ct2) sonic = true;
    else if (s1s2bar * sE1 * sE2 <= ct2) sonic = true;
    else if (fmin2(fabs(sE1), fabs(sE2)) < criticaltol_2) sonic = true;
    else if (sE1 < criticaltol_2 && rt.s1m > -criticaltol_2) sonic = true;
    else if (sE2 > -criticaltol_2 && rt.s2m < criticaltol_2) sonic = true;
    else if ((uL + cL) * (uR + cR) < 0.0) sonic = true;
    else if ((uL - cL) * (uR - cR) < 0.0) sonic = true;
    double x0 = sonic ? -gz * hbar * delb : -gz * hbar * delb * s1s2tilde / s1s2bar;
    double nL = -hL * delb, nR = -hR * delb;
    double Y1 = gz * fmax2(nL, nR);
    double x1 = fmin2(x0, Y1);
    double Y2 = gz * fmin2(nL, nR);
    double x2 = fmax2(x1, Y2);
    bool u0 = fabs(u) <= 0.0;
    double source2dx = u0 ? -hbar * gz * delb : x2;
    double d0 = sonic ? -delb : delb * gz * hbar / s1s2bar;
    int dcase = 0;
    double X1 = 0.0, X2 = 0.0, d1 = d0, deldelh = d0;
    if (sE1 < -criticaltol && sE2 > criticaltol) {
        dcase = 1;
        X1 = hstarHLL * (sE2 - sE1) / sE2;
        d1 = fmin2(d0, X1);
        X2 = hstarHLL * (sE2 - sE1) / sE1;
        deldelh = fmax2(d1, X2);
    } else if (sE1 >= criticaltol) {
        dcase = 2;
        X1 = hstarHLL * (sE2 - sE1) / sE1;
        d1 = fmin2(d0, X1);
        X2 = -hL;
        deldelh = fmax2(d1, X2);
    } else if (sE2 <= -criticaltol) {
        dcase = 3;
        X1 = hR;
        d1 = fmin2(d0, X1);
        X2 = hstarHLL * (sE2 - sE1) / sE2;
        deldelh = fmax2(d1, X2);
    }
    double del0 = hR - hL - deldelh;
    double del1 = huR - huL;
    double del2a = hR * sq(uR) + 0.5 * 1.0 * gz * sq(hR) - (hL * sq(uL) + 0.5 * 1.0 * gz * sq(hL));
    double grg = gamma * rho * gz;
    double vnorm = sqrt(sq(uR) + sq(uL) + sq(vR) + sq(vL));
    bool is_static = false;
    int tcase = 0;  // 0: moving (tausource 0), 1: static, 2: sign-matched friction
    double tdR = R.taudir;
    double tA = 0.0, tB = 0.0, ts0 = 0.0;
    double xs = del2a - source2dx;
    if (vnorm > 0.0) {
        tcase = 0;
    } else {
        tA = tdR * tauR / rhoR;
        tB = tauL * tdR / rhoL;
        double fr = 0.5 * fabs(tA + tB);
        if (fr > fabs(xs)) {
            tcase = 1;
            del1 = 0.0; del0 = 0.0;
            is_static = true;
        } else {
            tcase = 2;
            ts0 = 0.5 * (tA + tB);
        }
    }
    double a = sw1, c = sw3, bb = sw2;
    double D = c - a;
    double beta1, beta2 = 0.0, beta3, D1 = 0.0, D2 = 0.0, D3 = 0.0;
    if (!rc) {
        beta1 = (c * del0 - del1) / D;
        beta3 = (del1 - a * del0) / D;
    } else {
        // the corrector's system needs del2 = del2a - source2dx - tausource
        double tsrc = 0.0;
        if (tcase == 1) tsrc = xs;
        else if (tcase == 2) tsrc = fsign(ts0, xs);
        if (wallprob) tsrc = 0.0;
        const double del2 = xs - tsrc;
        D1 = sq(a) - a * bb - a * c + bb * c;
        D2 = a * bb - a * c - sq(bb) + bb * c;
        D3 = a * bb - a * c - bb * c + sq(c);
        beta1 = (bb * c * del0 - (bb + c) * del1 + del2) / D1;
        beta2 = (-a * c * del0 + (a + c) * del1 - del2) / D2;
        beta3 = (a * bb * del0 - (a + bb) * del1 + del2) / D3;
    }
    double fw11 = beta1 * sw1;
    double fw13 = beta3 * sw3;
    double hustar = huL + fw11;
    double ui = 0.0;
    double Kd = -gamma * rho * gz;
    if (!is_static) ui = hustar / hstarHLL;

    // ---- reverse ----
    double sw1b = wb.s1 * wall1, sw2b = wb.s2 * wall2, sw3b = wb.s5 * wall3;
    double fw11b = wb.w1h * wall1, fw21b = wb.w1n * wall1, fw31b = wb.w1t * wall1, fw41b = wb.w1m * wall1,
           fw51b = wb.w1p * wall1;
    double fw12b = wb.w2h * wall2;  // fw12 = beta2 R(1,2): 0 without the corrector
    double fw22b = wb.w2n * wall2;
    double fw13b = wb.w5h * wall3, fw23b = wb.w5n * wall3, fw33b = wb.w5t * wall3, fw43b = wb.w5m * wall3,
           fw53b = wb.w5p * wall3;
    double fw32b, fw42b, fw52b;
    if (hustar <= 0.0) { fw32b = fw31b; fw42b = fw41b; fw52b = fw51b; }
    else { fw32b = fw33b; fw42b = fw43b; fw52b = fw53b; }
    // working-variable adjoints
    double hLb = 0, hRb = 0, huLb = 0, huRb = 0, hvLb = 0, hvRb = 0, hmLb = 0, hmRb = 0, pLb = 0, pRb = 0;
    double bLb = 0, bRb = 0, uLb = 0, uRb = 0, vLb = 0, vRb = 0, mLb = 0, mRb = 0;
    double gammab = 0, gammaLb = 0, gammaRb = 0, rhob = 0, rhoLb = 0, rhoRb = 0, tauLb = 0, tauRb = 0;
    double del0b = 0, del1b = 0, del2ab = 0, source2dxb = 0, grgb = 0, hstarb = 0;
    // fw52 = del4 - fw53 - fw51
    double del4b = fw52b;
    fw53b -= fw52b;
    fw51b -= fw52b;
    double hustarb = 0.0;
    if (!is_static) {
        double dh = hR - hL, dp = pR - pL;
        double uib = del4b * (Kd * dh + dp);
        gammab += del4b * (-rho * gz * ui * dh);
        rhob += del4b * (-gamma * gz * ui * dh);
        hRb += del4b * Kd * ui;
        hLb -= del4b * Kd * ui;
        grgb += del4b * del1;
        del1b += del4b * grg;
        pRb += del4b * ui;
        pLb -= del4b * ui;
        hustarb += uib / hstarHLL;
        hstarb -= uib * ui / hstarHLL;
    }
    huLb += hustarb;
    fw11b += hustarb;
    // fw53 = fw13 gammaR rhoR grav, fw51 = fw11 gammaL rhoL grav
    fw13b += fw53b * gammaR * rhoR * grav;
    gammaRb += fw53b * fw13 * rhoR * grav;
    rhoRb += fw53b * fw13 * gammaR * grav;
    fw11b += fw51b * gammaL * rhoL * grav;
    gammaLb += fw51b * fw11 * rhoL * grav;
    rhoLb += fw51b * fw11 * gammaL * grav;
    // fw32 = hvR uR - hvL uL - fw31 - fw33 (fw31 = fw11 vL, fw33 = fw13 vR)
    hvRb += fw32b * uR; uRb += fw32b * hvR; hvLb -= fw32b * uL; uLb -= fw32b * hvL;
    fw31b -= fw32b; fw33b -= fw32b;
    fw11b += fw31b * vL; vLb += fw31b * fw11; fw13b += fw33b * vR; vRb += fw33b * fw13;
    // fw42 = hmR uR - hmL uL - fw41 - fw43 (fw41 = fw11 mL, fw43 = fw13 mR)
    hmRb += fw42b * uR; uRb += fw42b * hmR; hmLb -= fw42b * uL; uLb -= fw42b * hmL;
    fw41b -= fw42b; fw43b -= fw42b;
    fw11b += fw41b * mL; mLb += fw41b * fw11; fw13b += fw43b * mR; mRb += fw43b * fw13;
    // fw11 = beta1 sw1, fw21 = beta1 sw1^2, fw22 = beta2, fw13 = beta3 sw3, fw23 = beta3 sw3^2
    double beta1b = fw11b * sw1 + fw21b * sq(sw1);
    sw1b += fw11b * beta1 + fw21b * beta1 * 2.0 * sw1;
    double beta2b;
    if (!rc) {
        beta2b = fw22b;
    } else {
        // fw12 = beta2 sw2, fw22 = beta2 sw2^2
        beta2b = fw12b * sw2 + fw22b * sq(sw2);
        sw2b += fw12b * beta2 + fw22b * beta2 * 2.0 * sw2;
    }
    double beta3b = fw13b * sw3 + fw23b * sq(sw3);
    sw3b += fw13b * beta3 + fw23b * beta3 * 2.0 * sw3;
    double ab_ = 0.0, cb_ = 0.0, bbb_ = 0.0, del2b = 0.0;
    if (!rc) {
        // beta1 = (c del0 - del1)/D, beta3 = (del1 - a del0)/D, beta2 = a c del0 - (a+c) del1 + del2
        cb_ += beta1b * (del0 - beta1) / D;
        ab_ += beta1b * beta1 / D;
        del0b += beta1b * c / D;
        del1b -= beta1b / D;
        ab_ += beta3b * (beta3 - del0) / D;
        cb_ -= beta3b * beta3 / D;
        del1b += beta3b / D;
        del0b -= beta3b * a / D;
        ab_ += beta2b * (c * del0 - del1);
        cb_ += beta2b * (a * del0 - del1);
        del0b += beta2b * a * c;
        del1b -= beta2b * (a + c);
        del2b += beta2b;
    } else {
        // beta_i = N_i / D_i of the corrector's system (riemannsolvers_dclaw.f:378-385)
        const double N1b = beta1b / D1, N2b = beta2b / D2, N3b = beta3b / D3;
        const double D1b = -beta1b * beta1 / D1, D2b = -beta2b * beta2 / D2, D3b = -beta3b * beta3 / D3;
        // N1 = bb c del0 - (bb + c) del1 + del2
        bbb_ += N1b * (c * del0 - del1);
        cb_ += N1b * (bb * del0 - del1);
        del0b += N1b * bb * c;
        del1b -= N1b * (bb + c);
        del2b += N1b;
        // N2 = -a c del0 + (a + c) del1 - del2
        ab_ += N2b * (-c * del0 + del1);
        cb_ += N2b * (-a * del0 + del1);
        del0b -= N2b * a * c;
        del1b += N2b * (a + c);
        del2b -= N2b;
        // N3 = a bb del0 - (a + bb) del1 + del2
        ab_ += N3b * (bb * del0 - del1);
        bbb_ += N3b * (a * del0 - del1);
        del0b += N3b * a * bb;
        del1b -= N3b * (a + bb);
        del2b += N3b;
        // D1 = a^2 - a bb - a c + bb c, D2 = a bb - a c - bb^2 + bb c, D3 = a bb - a c - bb c + c^2
        ab_ += D1b * (2.0 * a - bb - c) + D2b * (bb - c) + D3b * (bb - c);
        bbb_ += D1b * (c - a) + D2b * (a - 2.0 * bb + c) + D3b * (a - c);
        cb_ += D1b * (bb - a) + D2b * (bb - a) + D3b * (2.0 * c - a - bb);
    }
    sw1b += ab_;
    sw3b += cb_;
    sw2b += bbb_;
    // del2 = (del2a - source2dx) - tausource
    del2ab += del2b;
    source2dxb -= del2b;
    double tsb = wallprob ? 0.0 : -del2b;
    if (tcase == 1) {
        // tausource = del2a - source2dx; del0 = del1 = 0 afterwards
        del2ab += tsb;
        source2dxb -= tsb;
        del0b = 0.0;
        del1b = 0.0;
    } else if (tcase == 2) {
        double sx = signbit(xs) ? -1.0 : 1.0;
        double s0 = signbit(ts0) ? -1.0 : 1.0;
        double ts0b = tsb * sx * s0;
        double tAb = 0.5 * ts0b, tBb = 0.5 * ts0b;
        // tA = tdR tauR / rhoR, tB = tauL tdR / rhoL
        Rb.taudir += tAb * tauR / rhoR + tBb * tauL / rhoL;
        tauRb += tAb * tdR / rhoR;
        rhoRb -= tAb * tA / rhoR;
        tauLb += tBb * tdR / rhoL;
        rhoLb -= tBb * tB / rhoL;
    }
    // grg = gamma rho gz
    gammab += grgb * rho * gz;
    rhob += grgb * gamma * gz;
    // del2a
    hRb += del2ab * (sq(uR) + gz * hR);
    uRb += del2ab * 2.0 * hR * uR;
    hLb -= del2ab * (sq(uL) + gz * hL);
    uLb -= del2ab * 2.0 * hL * uL;
    // del1 = huR - huL, del0 = hR - hL - deldelh
    huRb += del1b;
    huLb -= del1b;
    hRb += del0b;
    hLb -= del0b;
    double deldelhb = -del0b;
    // deldelh clamps
    double d0b = 0.0, sE1b = 0.0, sE2b = 0.0, delbb = 0.0, hbarb = 0.0, s1s2barb = 0.0, s1s2tildeb = 0.0;
    if (dcase == 0) {
        d0b = deldelhb;
    } else {
        double d1b = 0.0, X1b = 0.0, X2b = 0.0;
        if (d1 > X2) d1b = deldelhb; else X2b = deldelhb;
        if (d0 < X1) d0b = d1b; else X1b = d1b;
        const double dS = sE2 - sE1;
        if (dcase == 1) {
            // X1 = hstar dS / sE2, X2 = hstar dS / sE1
            hstarb += X1b * dS / sE2;
            sE2b += X1b * hstarHLL / sE2 - X1b * X1 / sE2;
            sE1b -= X1b * hstarHLL / sE2;
            hstarb += X2b * dS / sE1;
            sE2b += X2b * hstarHLL / sE1;
            sE1b += -X2b * hstarHLL / sE1 - X2b * X2 / sE1;
        } else if (dcase == 2) {
            hstarb += X1b * dS / sE1;
            sE2b += X1b * hstarHLL / sE1;
            sE1b += -X1b * hstarHLL / sE1 - X1b * X1 / sE1;
            hLb -= X2b;
        } else {
            hRb += X1b;
            hstarb += X2b * dS / sE2;
            sE2b += X2b * hstarHLL / sE2 - X2b * X2 / sE2;
            sE1b -= X2b * hstarHLL / sE2;
        }
    }
    if (sonic) {
        delbb -= d0b;
    } else {
        delbb += d0b * gz * hbar / s1s2bar;
        hbarb += d0b * delb * gz / s1s2bar;
        s1s2barb -= d0b * d0 / s1s2bar;
    }
    // source2dx
    if (u0) {
        hbarb += source2dxb * (-gz * delb);
        delbb += source2dxb * (-hbar * gz);
    } else {
        double x2b = source2dxb;
        double x1b = 0.0, Y2b = 0.0, x0b = 0.0, Y1b = 0.0;
        if (x1 > Y2) x1b = x2b; else Y2b = x2b;
        if (nL < nR) { hLb += Y2b * gz * (-delb); delbb += Y2b * gz * (-hL); }
        else { hRb += Y2b * gz * (-delb); delbb += Y2b * gz * (-hR); }
        if (x0 < Y1) x0b = x1b; else Y1b = x1b;
        if (nL > nR) { hLb += Y1b * gz * (-delb); delbb += Y1b * gz * (-hL); }
        else { hRb += Y1b * gz * (-delb); delbb += Y1b * gz * (-hR); }
        if (sonic) {
            hbarb += x0b * (-gz) * delb;
            delbb += x0b * (-gz) * hbar;
        } else {
            hbarb += x0b * (-gz * delb * s1s2tilde) / s1s2bar;
            delbb += x0b * (-gz * hbar * s1s2tilde) / s1s2bar;
            s1s2tildeb += x0b * (-gz * hbar * delb) / s1s2bar;
            s1s2barb -= x0b * x0 / s1s2bar;
        }
    }
    // s1s2tilde, s1s2bar, hbar, delb
    if (!(0.0 > uL * uR)) {
        uLb += s1s2tildeb * uR;
        uRb += s1s2tildeb * uL;
    }
    hbarb -= s1s2tildeb * gz;
    uLb += s1s2barb * 0.5 * (uL + uR);
    uRb += s1s2barb * 0.5 * (uL + uR);
    hbarb -= s1s2barb * gz;
    hLb += 0.5 * hbarb;
    hRb += 0.5 * hbarb;
    bRb += delbb;
    bLb -= delbb;
    // hstarHLL = max(Qh, 0)
    if (Qh > 0.0) {
        double Qb = hstarb;
        huLb += Qb / Dd;
        huRb -= Qb / Dd;
        sE2b += Qb * hR / Dd - Qb * Qh / Dd;
        hRb += Qb * sE2 / Dd;
        sE1b += -Qb * hL / Dd + Qb * Qh / Dd;
        hLb -= Qb * sE1 / Dd;
    }
    // sw2, sw3, sw1
    double s1mb = 0.0, s2mb = 0.0;
    if (rsel == 0) {
        sw3b += 0.5 * sw2b;
        sw1b += 0.5 * sw2b;
    } else if (rsel == 1) {
        s1mb += sw2b;
    } else if (rsel == 2) {
        s2mb += sw2b;
    } else {
        s1mb += 0.5 * sw2b;
        s2mb += 0.5 * sw2b;
    }
    if (sE2 > rt.s1m) sE2b += sw3b; else s1mb += sw3b;
    if (sE1 < rt.s2m) sE1b += sw1b; else s2mb += sw1b;
    riemanntype_b(hL, hR, uL, uR, drytol, geps, 0.0, s1mb, s2mb, hLb, hRb, uLb, uRb);
    // sE1 = min(sL, sRoe1), sE2 = max(sR, sRoe2)
    double sLb = 0, sRb = 0, sRoe1b = 0, sRoe2b = 0;
    if (sL < sRoe1) sLb += sE1b; else sRoe1b += sE1b;
    if (sR > sRoe2) sRb += sE2b; else sRoe2b += sE2b;
    double uhatb = sRoe1b + sRoe2b;
    double chatb = -sRoe1b + sRoe2b;
    double tch = dsqrt_b(chat, chatb);
    hRb += tch * geps * 0.5;
    hLb += tch * geps * 0.5;
    double sqhLb = uhatb * (uL - uhat) / Du, sqhRb = uhatb * (uR - uhat) / Du;
    uLb += uhatb * sqhL / Du;
    uRb += uhatb * sqhR / Du;
    uLb += sLb;
    double cLb = -sLb;
    uRb += sRb;
    double cRb = sRb;
    hLb += geps * dsqrt_b(cL, cLb) + dsqrt_b(sqhL, sqhLb);
    hRb += geps * dsqrt_b(cR, cRb) + dsqrt_b(sqhR, sqhRb);
    // gammas
    if (P.src2method == -1) {
        rhob -= gammab * gamma / rho;
        rhoLb -= gammaLb * gammaL / rhoL;
        rhoRb -= gammaRb * gammaR / rhoR;
    } else {
        rhob -= gammab * 0.25 * P.rho_f / (rho * rho);
        rhoLb -= gammaLb * 0.25 * P.rho_f / (rhoL * rhoL);
        rhoRb -= gammaRb * 0.25 * P.rho_f / (rhoR * rhoR);
    }
    rhoLb += 0.5 * rhob;
    rhoRb += 0.5 * rhob;
    // tauL = L.fs tauL0, tauR = R.fs tauR0
    Lb.fs += tauLb * tauL0;
    Rb.fs += tauRb * tauR0;
    double tauL0b = tauLb * L.fs, tauR0b = tauRb * R.fs;
    double rhoLsvb = 0, tauLsvb = 0, rhoRsvb = 0, tauRsvb = 0;
    if (rcase == 0) {
        rhoLsvb += rhoLb; tauLsvb += tauL0b; rhoRsvb += rhoRb; tauRsvb += tauR0b;
    } else if (rcase == 1) {
        rhoLsvb += rhoLb + rhoRb; tauLsvb += tauL0b + 0.5 * tauR0b;
    } else {
        rhoRsvb += rhoLb + rhoRb; tauRsvb += tauR0b + 0.5 * tauL0b;
    }
    // working variables back to the sides
    auto to_L = [&](double h_, double hn_, double ht_, double hm_, double p_, double b_, double un_, double ut_,
                    double m_, double rs_, double ts_) {
        Lb.h += h_; Lb.hn += hn_; Lb.ht += ht_; Lb.hm += hm_; Lb.p += p_; Lb.b += b_;
        Lb.un += un_; Lb.ut += ut_; Lb.m += m_; Lb.rho_sv += rs_; Lb.tau_sv += ts_;
    };
    auto to_R = [&](double h_, double hn_, double ht_, double hm_, double p_, double b_, double un_, double ut_,
                    double m_, double rs_, double ts_) {
        Rb.h += h_; Rb.hn += hn_; Rb.ht += ht_; Rb.hm += hm_; Rb.p += p_; Rb.b += b_;
        Rb.un += un_; Rb.ut += ut_; Rb.m += m_; Rb.rho_sv += rs_; Rb.tau_sv += ts_;
    };
    if (pre == 0) {
        to_L(hLb, huLb, hvLb, hmLb, pLb, bLb, uLb, vLb, mLb, rhoLsvb, tauLsvb);
        to_R(hRb, huRb, hvRb, hmRb, pRb, bRb, uRb, vRb, mRb, rhoRsvb, tauRsvb);
    } else if (pre == 1) {
        to_L(hLb, huLb, hvLb, hmLb, pLb, bLb, uLb, vLb, mLb, rhoLsvb, tauLsvb);
        if (wallprob) to_L(hRb, -huRb, hvRb, hmRb, pRb, bRb, -uRb, vRb, mRb, rhoRsvb, tauRsvb);
        else {
            to_R(0.0, huRb, hvRb, hmRb, 0.0, bRb, uRb, vRb, 0.0, rhoRsvb, tauRsvb);
            Lb.m += mRb;
        }
    } else {
        to_R(hRb, huRb, hvRb, hmRb, pRb, bRb, uRb, vRb, mRb, rhoRsvb, tauRsvb);
        if (wallprob) to_R(hLb, -huLb, hvLb, hmLb, pLb, bLb, -uLb, vLb, mLb, rhoLsvb, tauLsvb);
        else {
            to_L(0.0, huLb, hvLb, hmLb, 0.0, bLb, uLb, vLb, 0.0, rhoLsvb, tauLsvb);
            Rb.m += mLb;
        }
    }
    return true;
}

// ---------------------------------------------------------------------------
// Adjoint of one cell's inputs: qB fields in q order (h, hu, hv, hm, p) plus
// its static-friction factor, friction direction and bed.
struct CellB {
    double q[5];
    double fs, taudir, b;
};

DC_HD void zero_cellb(CellB& c) {
    for (int k = 0; k < 5; ++k) c.q[k] = 0.0;
    c.fs = c.taudir = c.b = 0.0;
}

// load_side reverse (see load_side): Side adjoint -> cell adjoint, with
// setvars' partial derivatives read from the record (svrec_cell)
DC_HD void load_side_b_sv(const dclaw_params& P, const Work& W, const double* __restrict__ sv, size_t pi,
                          int comp_n, int comp_t, bool twice, const SideB& sb, CellB& cb, double* pbar) {
    cb.b += sb.b;
    cb.fs += sb.fs;
    cb.taudir += sb.taudir;
    double h = W.qB[pi];
    if (h <= P.dry_tolerance) return;
    double hn = W.qB[(size_t)comp_n * W.npad + pi];
    double ht = W.qB[(size_t)comp_t * W.npad + pi];
    double hm0 = W.qB[3 * W.npad + pi];
    double p0 = W.qB[4 * W.npad + pi];
    double hm1 = hm0, p1 = p0, m1;
    qfix_mp(P, h, hm1, p1, m1, P.grav);
    double un = hn / h, ut = ht / h;
    const double* r = sv + (size_t)(twice ? SV_N : 0) * W.npad + pi;
    const size_t np = W.npad;
    const double tb = sb.tau_sv;
    const int kn = comp_n == 1 ? SV_DU : SV_DV, kt = comp_n == 1 ? SV_DV : SV_DU;
    double hb = sb.h + tb * r[SV_DH * np];
    double unb = sb.un + tb * r[(size_t)kn * np];
    double utb = sb.ut + tb * r[(size_t)kt * np];
    double mb = sb.m + (tb * r[SV_DM * np] + sb.rho_sv * (P.rho_s - P.rho_f));
    double pb = sb.p + tb * r[SV_DP * np];
    pbar[PB_PHI] += tb * r[SV_DPHI * np];
    pbar[PB_MU] += tb * r[SV_DMU * np];
    double hnb = sb.hn + unb / h, htb = sb.ht + utb / h;
    hb -= unb * un / h + utb * ut / h;
    double hmb = sb.hm;
    if (twice) {
        qfix_mp_b(P, h, hm1, p1, P.grav, hb, hmb, pb, mb);
        mb = 0.0;
    }
    qfix_mp_b(P, h, hm0, p0, P.grav, hb, hmb, pb, mb);
    cb.q[0] += hb;
    cb.q[comp_n] += hnb;
    cb.q[comp_t] += htb;
    cb.q[3] += hmb;
    cb.q[4] += pb;
}

// setvars record of padded cell pi: for the rpn2 states A1 and A2, tau and
// its partial derivatives (the reverse of setvars for a unit tau adjoint)
DC_HD void svrec_cell(const dclaw_params& P, const Work& W, double* __restrict__ sv, size_t pi) {
    const size_t np = W.npad;
    const double h = W.qB[pi];
    if (h <= P.dry_tolerance) return;  // dry sides never read their record
    const double u = W.qB[np + pi] / h, v = W.qB[2 * np + pi] / h;
    double hm = W.qB[3 * np + pi], p = W.qB[4 * np + pi], m;
    for (int a = 0; a < 2; ++a) {
        qfix_mp(P, h, hm, p, m, P.grav);
        SetVars s = setvars<false>(P, P.phi, h, u, v, m, p, P.grav);
        SetVars ob{};
        ob.tau = 1.0;
        double phib = 0.0, hb = 0.0, ub = 0.0, vb = 0.0, mb = 0.0, pb = 0.0;
        double pl[NPB] = {0.0, 0.0, 0.0, 0.0};
        setvars_b<false>(P, P.phi, h, u, v, m, p, P.grav, ob, phib, hb, ub, vb, mb, pb, pl);
        double* o = sv + (size_t)(a * SV_N) * np + pi;
        o[SV_TAU * np] = s.tau;
        o[SV_DH * np] = hb;
        o[SV_DU * np] = ub;
        o[SV_DV * np] = vb;
        o[SV_DM * np] = mb;
        o[SV_DP * np] = pb;
        o[SV_DPHI * np] = phib;
        o[SV_DMU * np] = pl[PB_MU];
    }
}

// Stage C reverse: interface i of slice r; wb = adjoint of its 15 stored
// values (W_* order). Accumulates into the cell adjoints of L and R.
// Returns false when the interface has no adjoint form (rare-wave corrector).
template <int DIR>
DC_HD bool stage_riemann_b(const dclaw_params& P, const Geom& g, const Work& W, const double* __restrict__ sv,
                           int r, int i, const double* wbv, CellB& Lc, CellB& Rc, double* pbar) {
    size_t pL, pR;
    if (DIR == 0) { pL = pidx(g, i - 1, r); pR = pidx(g, i, r); }
    else { pL = pidx(g, r, i - 1); pR = pidx(g, r, i); }
    const int cn = DIR == 0 ? 1 : 2, ct = DIR == 0 ? 2 : 1;
    if (W.qB[pL] <= P.dry_tolerance && W.qB[pR] <= P.dry_tolerance) return true;
    Side R = load_side_sv(P, W, sv, pR, cn, ct, false, 1 + DIR);
    Side L = load_side_sv(P, W, sv, pL, cn, ct, i - 1 >= 0, 1 + DIR);
    Waves wb;
    wb.s1 = wbv[W_S1]; wb.s2 = wbv[W_S2]; wb.s5 = wbv[W_S5];
    wb.w1h = wbv[W_1H]; wb.w1n = wbv[W_1N]; wb.w1t = wbv[W_1T]; wb.w1m = wbv[W_1M]; wb.w1p = wbv[W_1P];
    wb.w2h = wbv[W_2H]; wb.w2n = wbv[W_2N];
    wb.w5h = wbv[W_5H]; wb.w5n = wbv[W_5N]; wb.w5t = wbv[W_5T]; wb.w5m = wbv[W_5M]; wb.w5p = wbv[W_5P];
    SideB Lb, Rb;
    zero_sideb(Lb);
    zero_sideb(Rb);
    if (!riemann_solve_b(P, L, R, wb, Lb, Rb)) return false;
    load_side_b_sv(P, W, sv, pR, cn, ct, false, Rb, Rc, pbar);
    load_side_b_sv(P, W, sv, pL, cn, ct, i - 1 >= 0, Lb, Lc, pbar);
    return true;
}

// ---------------------------------------------------------------------------
// derivative of the limiter function at r (same case split as limiter_phi)
DC_HD double limiter_dphi(int mth, double r) {
    switch (mth) {
        case 1: {
            double m = fmin2(1.0, r);
            if (0.0 > m) return 0.0;
            return (1.0 < r) ? 0.0 : 1.0;
        }
        case 2: {
            double i1 = fmin2(1.0, 2.0 * r);
            double A = fmax2(0.0, i1), B = fmin2(2.0, r);
            if (A > B) {
                if (0.0 > i1) return 0.0;
                return (1.0 < 2.0 * r) ? 0.0 : 2.0;
            }
            return (2.0 < r) ? 0.0 : 1.0;
        }
        case 3: return r > 0.0 ? 2.0 / sq(1.0 + r) : 0.0;
        case 4: {
            double c = (1.0 + r) / 2.0;
            double i1 = fmin2(c, 2.0);
            double i2 = fmin2(i1, 2.0 * r);
            if (0.0 > i2) return 0.0;
            if (i1 < 2.0 * r) return (c < 2.0) ? 0.5 : 0.0;
            return 2.0;
        }
        default: return 1.0;
    }
}

// limit_family reverse. Wi: unlimited wave. Wib: on entry adjoint of the
// limited wave, on return adjoint of the unlimited one. Wmb/Wpb +=.
DC_HD void limit_family_b(int mth, double s, const double Wm[5], const double Wi[5], const double Wp[5],
                          double Wib[5], double Wmb[5], double Wpb[5]) {
    double wnorm2 = 0.0, dotl = 0.0, dotr = 0.0;
    for (int m = 0; m < 5; ++m) {
        wnorm2 = wnorm2 + sq(Wi[m]);
        dotl = dotl + Wm[m] * Wi[m];
        dotr = dotr + Wi[m] * Wp[m];
    }
    if (wnorm2 == 0.0) return;
    double r = s > 0.0 ? dotl / wnorm2 : dotr / wnorm2;
    uint32_t code;
    double wl = limiter_phi(mth, r, code);
    double wlb = 0.0;
    for (int m = 0; m < 5; ++m) {
        wlb += Wib[m] * Wi[m];
        Wib[m] = wl * Wib[m];
    }
    double rb = wlb * limiter_dphi(mth, r);
    double dotb = rb / wnorm2;
    double wn2b = -rb * r / wnorm2;
    const double* Wu = s > 0.0 ? Wm : Wp;
    double* Wub = s > 0.0 ? Wmb : Wpb;
    for (int m = 0; m < 5; ++m) {
        Wib[m] += 2.0 * Wi[m] * wn2b + Wu[m] * dotb;
        Wub[m] += Wi[m] * dotb;
    }
}

// rpt2_split reverse. bmb/bpb: adjoints of bm/bp; accumulates adjoints of
// (h, hn, ht, hm) into xb[0..3] and of asdq into asdqb[0..4].
DC_HD void rpt2_split_b(const dclaw_params& P, double h, double hn, double ht, double hm, double b, double topo1,
                        double topo3, const double asdq[5], const double bmb[5], const double bpb[5], double xb[4],
                        double asdqb[5]) {
    if (h <= P.dry_tolerance) return;
    const double g = P.grav;
    double u = hn / h, v = ht / h, m = hm / h;
    double eta = h + b;
    double rho = m * P.rho_s + (1.0 - m) * P.rho_f;
    double gamma;
    if (P.src2method == -1) gamma = P.rho_f / rho;
    else gamma = 0.25 * (P.rho_f + 3.0 * rho) / rho;
    if (eta < fmin2(topo1, topo3)) return;
    double sgh = sqrt(g * h);
    double s1 = v - sgh, s2 = v, s3 = v + sgh;
    double d1 = asdq[0], d2 = asdq[1], d3 = asdq[2];
    double Dn = s3 - s1;
    double beta1 = (s3 * d1 - d3) / Dn;
    double beta2 = -u * d1 + d2;
    double beta3 = (d3 - s1 * d1) / Dn;
    double r5 = gamma * rho * g;
    double ub = 0, vb = 0, mb = 0, r5b = 0, s1b = 0, s2b = 0, s3b = 0, b1b = 0, b2b = 0, b3b = 0;
    auto wave = [&](double sk, double betak, double& skb, double& betakb) {
        const double* Tb = nullptr;
        if ((sk < 0.0) && (eta >= topo1)) Tb = bmb;
        else if ((sk > 0.0) && (eta >= topo3)) Tb = bpb;
        if (!Tb) return;
        double sbk = 1.0 * sk * betak;
        double sbkb = Tb[0] + Tb[1] * u + Tb[2] * sk + Tb[3] * m + Tb[4] * r5;
        ub += sbk * Tb[1];
        skb += sbk * Tb[2];
        mb += sbk * Tb[3];
        r5b += sbk * Tb[4];
        skb += sbkb * betak;
        betakb += sbkb * sk;
    };
    wave(s1, beta1, s1b, b1b);
    {
        const double* Tb = nullptr;
        if ((s2 < 0.0) && (eta >= topo1)) Tb = bmb;
        else if ((s2 > 0.0) && (eta >= topo3)) Tb = bpb;
        if (Tb) {
            s2b += Tb[1] * beta2;
            b2b += Tb[1] * s2;
        }
    }
    wave(s3, beta3, s3b, b3b);
    // betas
    s3b += b1b * (d1 - beta1) / Dn;
    s1b += b1b * beta1 / Dn;
    asdqb[0] += b1b * s3 / Dn;
    asdqb[2] -= b1b / Dn;
    ub -= b2b * d1;
    asdqb[0] -= b2b * u;
    asdqb[1] += b2b;
    s1b += b3b * (beta3 - d1) / Dn;
    s3b -= b3b * beta3 / Dn;
    asdqb[2] += b3b / Dn;
    asdqb[0] -= b3b * s1 / Dn;
    vb += s1b + s2b + s3b;
    double sghb = -s1b + s3b;
    double hb = g * dsqrt_b(sgh, sghb);
    double rhob = r5b * gamma * g;
    double gammab = r5b * rho * g;
    if (P.src2method == -1) rhob -= gammab * gamma / rho;
    else rhob -= gammab * 0.25 * P.rho_f / (rho * rho);
    mb += rhob * (P.rho_s - P.rho_f);
    xb[1] += ub / h;
    xb[2] += vb / h;
    xb[3] += mb / h;
    hb -= (ub * u + vb * v + mb * m) / h;
    xb[0] += hb;
}

// load_a2 reverse: adjoint of the A2 state (h, hn, ht, hm) of cell pi into
// its qB adjoint (q order)
DC_HD void load_a2_b(const dclaw_params& P, const Work& W, size_t pi, int cn, int ct, const double xb[4],
                     double qb[5]) {
    double h = W.qB[pi];
    if (h <= P.dry_tolerance) return;
    double hm0 = W.qB[3 * W.npad + pi], p0 = W.qB[4 * W.npad + pi];
    double hm1 = hm0, p1 = p0, m;
    qfix_mp(P, h, hm1, p1, m, P.grav);
    double hb = xb[0], hmb = xb[3], pb = 0.0;
    qfix_mp_b(P, h, hm1, p1, P.grav, hb, hmb, pb, 0.0);
    qfix_mp_b(P, h, hm0, p0, P.grav, hb, hmb, pb, 0.0);
    qb[0] += hb;
    qb[cn] += xb[1];
    qb[ct] += xb[2];
    qb[3] += hmb;
    qb[4] += pb;
}

// Adjoints produced by the reverse of one interface's flux stage: its own
// 15 stored values, the wave components (12, no speeds; W1, W2 h/n, W5) of
// the interfaces on its left and right (limiter), and the A2 states of
// cells i-1 and i (transverse splits).
struct FluxB {
    double self[NW];
    double left[12], right[12];
    double a2l[4], a2r[4];
};

DC_HD void waves_to_compact(int cn, int ct, const double W1[5], const double W2[5], const double W5[5],
                            double* o /*12*/) {
    o[0] = W1[0]; o[1] = W1[cn]; o[2] = W1[ct]; o[3] = W1[3]; o[4] = W1[4];
    o[5] = W2[0]; o[6] = W2[cn];
    o[7] = W5[0]; o[8] = W5[cn]; o[9] = W5[ct]; o[10] = W5[3]; o[11] = W5[4];
}

// Stage D reverse. fb[30]: adjoints of the interface's faddm, faddp, U1m,
// U1p, U2m, U2p (5 each, q order).
template <int DIR>
DC_HD void stage_flux_b(const dclaw_params& P, const Geom& g, const Work& W, int r, int i, double dtdx,
                        const double* fb, FluxB& o) {
    const double* wv = DIR == 0 ? W.wx : W.wy;
    const size_t nplane = DIR == 0 ? W.nxi : W.nyi;
    auto oidx = [&](int ii) -> size_t { return DIR == 0 ? xidx(g, r, ii) : yidx(g, ii, r); };
    auto cidx = [&](int ii) -> size_t { return DIR == 0 ? pidx(g, ii, r) : pidx(g, r, ii); };
    const int cn = DIR == 0 ? 1 : 2, ct = DIR == 0 ? 2 : 1;
    for (int k = 0; k < NW; ++k) o.self[k] = 0.0;
    for (int k = 0; k < 12; ++k) { o.left[k] = 0.0; o.right[k] = 0.0; }
    for (int k = 0; k < 4; ++k) { o.a2l[k] = 0.0; o.a2r[k] = 0.0; }

    double s[3], W1[5], W2[5], W5[5];
    expand_waves<DIR>(wv, nplane, oidx(i), s, W1, W2, W5);
    double amdq[5], apdq[5];
    for (int m = 0; m < 5; ++m) {
        double am = 0.0, ap = 0.0;
        if (s[0] < 0.0) am = am + W1[m]; else if (s[0] > 0.0) ap = ap + W1[m];
        if (s[1] < 0.0) am = am + W2[m]; else if (s[1] > 0.0) ap = ap + W2[m];
        if (s[2] < 0.0) am = am + W5[m]; else if (s[2] > 0.0) ap = ap + W5[m];
        amdq[m] = am;
        apdq[m] = ap;
    }
    double L1[5], L2[5], L5[5];  // limited waves
    for (int m = 0; m < 5; ++m) { L1[m] = W1[m]; L2[m] = W2[m]; L5[m] = W5[m]; }
    double sm[3], Wm1[5], Wm2[5], Wm5[5], sp[3], Wp1[5], Wp2[5], Wp5[5];
    bool lim = P.order != 1 && P.limiter != 0;
    bool wet4 = false;
    double cqxx[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    double c1 = 0.0, c2 = 0.0, c5 = 0.0;
    if (P.order != 1) {
        if (lim) {
            expand_waves<DIR>(wv, nplane, oidx(i - 1), sm, Wm1, Wm2, Wm5);
            expand_waves<DIR>(wv, nplane, oidx(i + 1), sp, Wp1, Wp2, Wp5);
            limit_family(P.limiter, 1, s[0], Wm1, L1, Wp1, nullptr);
            limit_family(P.limiter, 2, s[1], Wm2, L2, Wp2, nullptr);
            limit_family(P.limiter, 5, s[2], Wm5, L5, Wp5, nullptr);
        }
        double hl2 = W.qB[cidx(i - 2)], hl = W.qB[cidx(i - 1)], hr = W.qB[cidx(i)], hr2 = W.qB[cidx(i + 1)];
        wet4 = hl * hr * hl2 * hr2 > 0.0;
        if (wet4) {
            c1 = fsign(1.0, s[0]) * (1.0 - fabs(s[0]) * dtdx);
            c2 = fsign(1.0, s[1]) * (1.0 - fabs(s[1]) * dtdx);
            c5 = fsign(1.0, s[2]) * (1.0 - fabs(s[2]) * dtdx);
            for (int m = 0; m < 5; ++m) {
                double cq = 0.0;
                cq = cq + c1 * L1[m];
                cq = cq + c2 * L2[m];
                cq = cq + c5 * L5[m];
                cqxx[m] = cq;
            }
        }
    }
    // ---- reverse ----
    double amdqb[5], apdqb[5], cqxxb[5];
    for (int m = 0; m < 5; ++m) {
        amdqb[m] = fb[m];
        apdqb[m] = -fb[5 + m];
        cqxxb[m] = P.order != 1 ? 0.5 * fb[m] + 0.5 * fb[5 + m] : 0.0;
    }
    if (P.transverse_waves != 0) {
        const bool fold = P.order > 1 && P.transverse_waves == 2;
        const double half = 0.5 * dtdx;
        for (int imp = 1; imp <= 2; ++imp) {
            const int cc = imp == 1 ? i - 1 : i;
            const size_t pc = cidx(cc);
            double h, hn, ht, hm;
            load_a2(P, W, pc, cn, ct, h, hn, ht, hm);
            double topo1, topo3;
            if (DIR == 0) { topo1 = W.bP[pidx(g, cc, r - 1)]; topo3 = W.bP[pidx(g, cc, r + 1)]; }
            else { topo1 = W.bP[pidx(g, r - 1, cc)]; topo3 = W.bP[pidx(g, r + 1, cc)]; }
            const double* src = imp == 1 ? amdq : apdq;
            double asdq[5];
            for (int m = 0; m < 5; ++m) {
                double v = src[m];
                if (fold) v = imp == 1 ? v + cqxx[m] : v - cqxx[m];
                asdq[m] = v;
            }
            double asdq_s[5] = {asdq[0], asdq[cn], asdq[ct], asdq[3], asdq[4]};
            const int ob = imp == 1 ? 10 : 20;
            double bmb_q[5], bpb_q[5];
            for (int m = 0; m < 5; ++m) {
                bmb_q[m] = half * fb[ob + m];
                bpb_q[m] = half * fb[ob + 5 + m];
            }
            double bmb[5] = {bmb_q[0], bmb_q[cn], bmb_q[ct], bmb_q[3], bmb_q[4]};
            double bpb[5] = {bpb_q[0], bpb_q[cn], bpb_q[ct], bpb_q[3], bpb_q[4]};
            double asb_s[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
            double* xb = imp == 1 ? o.a2l : o.a2r;
            rpt2_split_b(P, h, hn, ht, hm, W.bP[pc], topo1, topo3, asdq_s, bmb, bpb, xb, asb_s);
            double asb[5];
            asb[0] = asb_s[0]; asb[cn] = asb_s[1]; asb[ct] = asb_s[2]; asb[3] = asb_s[3]; asb[4] = asb_s[4];
            for (int m = 0; m < 5; ++m) {
                if (imp == 1) { amdqb[m] += asb[m]; if (fold) cqxxb[m] += asb[m]; }
                else { apdqb[m] += asb[m]; if (fold) cqxxb[m] -= asb[m]; }
            }
        }
    }
    double L1b[5] = {0, 0, 0, 0, 0}, L2b[5] = {0, 0, 0, 0, 0}, L5b[5] = {0, 0, 0, 0, 0};
    double sb[3] = {0.0, 0.0, 0.0};
    if (wet4) {
        double c1b = 0.0, c2b = 0.0, c5b = 0.0;
        for (int m = 0; m < 5; ++m) {
            L1b[m] += c1 * cqxxb[m];
            L2b[m] += c2 * cqxxb[m];
            L5b[m] += c5 * cqxxb[m];
            c1b += cqxxb[m] * L1[m];
            c2b += cqxxb[m] * L2[m];
            c5b += cqxxb[m] * L5[m];
        }
        // c = sign(1, s) (1 - |s| dtdx): dc/ds = -dtdx for s != 0
        if (s[0] != 0.0) sb[0] -= c1b * dtdx;
        if (s[1] != 0.0) sb[1] -= c2b * dtdx;
        if (s[2] != 0.0) sb[2] -= c5b * dtdx;
    }
    double W1b[5], W2b[5], W5b[5];
    for (int m = 0; m < 5; ++m) { W1b[m] = L1b[m]; W2b[m] = L2b[m]; W5b[m] = L5b[m]; }
    if (lim) {
        double Wm1b[5] = {0, 0, 0, 0, 0}, Wm2b[5] = {0, 0, 0, 0, 0}, Wm5b[5] = {0, 0, 0, 0, 0};
        double Wp1b[5] = {0, 0, 0, 0, 0}, Wp2b[5] = {0, 0, 0, 0, 0}, Wp5b[5] = {0, 0, 0, 0, 0};
        limit_family_b(P.limiter, s[0], Wm1, W1, Wp1, W1b, Wm1b, Wp1b);
        limit_family_b(P.limiter, s[1], Wm2, W2, Wp2, W2b, Wm2b, Wp2b);
        limit_family_b(P.limiter, s[2], Wm5, W5, Wp5, W5b, Wm5b, Wp5b);
        waves_to_compact(cn, ct, Wm1b, Wm2b, Wm5b, o.left);
        waves_to_compact(cn, ct, Wp1b, Wp2b, Wp5b, o.right);
    }
    for (int m = 0; m < 5; ++m) {
        if (s[0] < 0.0) W1b[m] += amdqb[m]; else if (s[0] > 0.0) W1b[m] += apdqb[m];
        if (s[1] < 0.0) W2b[m] += amdqb[m]; else if (s[1] > 0.0) W2b[m] += apdqb[m];
        if (s[2] < 0.0) W5b[m] += amdqb[m]; else if (s[2] > 0.0) W5b[m] += apdqb[m];
    }
    o.self[W_S1] = sb[0]; o.self[W_S2] = sb[1]; o.self[W_S5] = sb[2];
    o.self[W_1H] = W1b[0]; o.self[W_1N] = W1b[cn]; o.self[W_1T] = W1b[ct]; o.self[W_1M] = W1b[3];
    o.self[W_1P] = W1b[4];
    o.self[W_2H] = W2b[0]; o.self[W_2N] = W2b[cn];
    o.self[W_5H] = W5b[0]; o.self[W_5N] = W5b[cn]; o.self[W_5T] = W5b[ct]; o.self[W_5M] = W5b[3];
    o.self[W_5P] = W5b[4];
}

// Adjoint of the 30 stored flux values of interface i of slice r from the
// adjoints lam of the updated interior states (5 planes mx*my, before src2),
// following stage_update's accumulation.
template <int DIR>
DC_HD void flux_bar(const Geom& g, const double* __restrict__ lam, int r, int i, double dt, double* fb) {
    const double dtdx = dt / g.dx, dtdy = dt / g.dy;
    const size_t plane = (size_t)g.mx * g.my;
    auto L = [&](int ci, int cj, int m) -> double {
        if (ci < 1 || ci > g.mx || cj < 1 || cj > g.my) return 0.0;
        return lam[(size_t)m * plane + (size_t)(cj - 1) * g.mx + (size_t)(ci - 1)];
    };
    for (int m = 0; m < 5; ++m) {
        if (DIR == 0) {
            fb[m] = -dtdx * L(i - 1, r, m);
            fb[5 + m] = dtdx * L(i, r, m);
            fb[10 + m] = dtdy * (L(i - 1, r - 1, m) - L(i - 1, r, m));
            fb[15 + m] = dtdy * (L(i - 1, r, m) - L(i - 1, r + 1, m));
            fb[20 + m] = dtdy * (L(i, r - 1, m) - L(i, r, m));
            fb[25 + m] = dtdy * (L(i, r, m) - L(i, r + 1, m));
        } else {
            fb[m] = -dtdy * L(r, i - 1, m);
            fb[5 + m] = dtdy * L(r, i, m);
            fb[10 + m] = dtdx * (L(r - 1, i - 1, m) - L(r, i - 1, m));
            fb[15 + m] = dtdx * (L(r, i - 1, m) - L(r + 1, i - 1, m));
            fb[20 + m] = dtdx * (L(r - 1, i, m) - L(r, i, m));
            fb[25 + m] = dtdx * (L(r, i, m) - L(r + 1, i, m));
        }
    }
}

// ---------------------------------------------------------------------------
// mp_update_relax reverse (src2method 0/1). Inputs (h, u, v, m, p, rhoh) as
// the forward received them; on entry hb..pb hold adjoints of the outputs
// (h, u, v, m, p), replaced by adjoints of the inputs; rhohb, phib, pbar +=.
DC_HD void mp_update_relax_b(const dclaw_params& P, double phi, double dt, double h, double u, double v, double m,
                             double p, double rhoh, double gz, double& hb, double& ub, double& vb, double& mb,
                             double& pb, double& rhohb, double& phib, double* pbar) {
    const double rs = P.rho_s, rf = P.rho_f;
    // ---- forward recompute ----
    SetVars sv = setvars<true>(P, phi, h, u, v, m, p, gz);
    double hu = h * u, hv = h * v, hm = h * m;
    double nrm = sqrt(sq(hu) + sq(hv));
    double vnorm = nrm / h;
    double pA = p - dt * 3.0 * vnorm * sv.tanpsi * sv.alphainv / h;
    double hB = h, huB = hu, hvB = hv, hmB = hm, pB = pA, uB, vB, mB;
    qfix(P, hB, huB, hvB, hmB, pB, uB, vB, mB, gz);
    double rho = rs * mB + (1.0 - mB) * rf;
    double z1 = 3.0 * sv.alphainv / (h * 2.0);
    double z2 = (rho - rf) * rf * gz / (4.0 * rho);
    double zeta = z1 + z2;
    double mumax = fmax2(P.mu, 1.0e-16);
    double krate = -zeta * 2.0 * sv.kperm / (h * mumax);
    double p_eq = rf * h * gz;
    double ek1 = em::d_exp(krate * dt);
    double pC = p_eq + (pB - p_eq) * ek1;
    double p_exc = pC - rf * gz * h;
    double h4 = h, m4 = mB, p4 = pC, rho4 = rho, pex4 = p_exc, hu4 = huB, hv4 = hvB, hm4 = hmB;
    qfix_cmass(P, h4, m4, p4, rho4, pex4, hu4, hv4, hm4, uB, vB, rhoh, gz);
    double D = -2.0 * (sv.kperm / (P.mu * h4)) * pex4;
    double krate2 = D * (rho4 - rf) / rhoh;
    double ek2 = em::d_exp(-dt * D * rf / (rhoh));
    double hm5 = hm4 * ek2;
    double h5, hu5, hv5, ek3 = 0.0;
    if (P.src2method == 0) {
        h5 = h4 + h4 * krate2 * dt;
        ek3 = em::d_exp(dt * krate2);
        hu5 = hu4 * ek3;
        hv5 = hv4 * ek3;
    } else {
        h5 = (rhoh - hm5 * (rs - rf)) / rf;
        hu5 = h5 * uB;
        hv5 = h5 * vB;
    }
    // ---- reverse ----
    // final qfix(h5, hu5, hv5, hm5, p4) -> (h, u, v, m, p)
    double h5b = hb, hu5b = 0.0, hv5b = 0.0, hm5b = 0.0, p4b = pb;
    qfix_b(P, h5, hu5, hv5, hm5, p4, gz, h5b, hu5b, hv5b, hm5b, p4b, ub, vb, mb);
    double h4b = 0.0, hu4b = 0.0, hv4b = 0.0, krate2b = 0.0, uBb = 0.0, vBb = 0.0;
    if (P.src2method == 0) {
        hu4b += hu5b * ek3;
        hv4b += hv5b * ek3;
        double ek3b = hu5b * hu4 + hv5b * hv4;
        krate2b += ek3b * ek3 * dt;
        h4b += h5b * (1.0 + krate2 * dt);
        krate2b += h5b * h4 * dt;
    } else {
        h5b += hu5b * uB + hv5b * vB;
        uBb += hu5b * h5;
        vBb += hv5b * h5;
        rhohb += h5b / rf;
        hm5b -= h5b * (rs - rf) / rf;
    }
    // hm5 = hm4 ek2, ek2 = exp(-dt D rf / rhoh)
    double hm4b = hm5b * ek2;
    double ek2b = hm5b * hm4;
    double argb = ek2b * ek2;
    double arg2 = -dt * D * rf / (rhoh);
    double Db = argb * (-dt * rf / rhoh);
    rhohb -= argb * arg2 / rhoh;
    // krate2 = D (rho4 - rf) / rhoh
    Db += krate2b * (rho4 - rf) / rhoh;
    double rho4b = krate2b * D / rhoh;
    rhohb -= krate2b * krate2 / rhoh;
    // D = -2 (kperm / (mu h4)) pex4
    double kpermb = Db * (-2.0 * pex4 / (P.mu * h4));
    double pex4b = Db * (-2.0 * (sv.kperm / (P.mu * h4)));
    h4b -= Db * D / h4;
    pbar[PB_MU] -= Db * D / P.mu;
    // qfix_cmass(m=mB, p_exc, u=uB, v=vB, rhoh) -> h4, m4, p4, rho4, pex4, hu4, hv4, hm4
    double mBb = 0.0;
    {
        double mb_io = 0.0, pexb_io = pex4b;
        // adjoint of output m4: none beyond qfix's final use (m is recomputed there)
        qfix_cmass_b(P, mB, p_exc, uB, vB, rhoh, gz, h4b, mb_io, p4b, rho4b, pexb_io, hu4b, hv4b, hm4b, uBb, vBb,
                     rhohb);
        mBb += mb_io;
        // p_exc = pC - rf gz h
        double pCb = pexb_io;
        double hb_loc = -pexb_io * rf * gz;
        // pC = p_eq + (pB - p_eq) ek1
        double p_eqb = pCb * (1.0 - ek1);
        double pBb = pCb * ek1;
        double ek1b = pCb * (pB - p_eq);
        double kb = ek1b * ek1 * dt;
        hb_loc += p_eqb * rf * gz;
        // krate = -zeta 2 kperm / (h mumax)
        double zetab = kb * (-2.0 * sv.kperm / (h * mumax));
        kpermb += kb * (-zeta * 2.0 / (h * mumax));
        hb_loc -= kb * krate / h;
        if (P.mu > 1.0e-16) pbar[PB_MU] -= kb * krate / mumax;
        // zeta = 3 alphainv / (2h) + (rho - rf) rf gz / (4 rho)
        double alphainvb = zetab * 3.0 / (h * 2.0);
        hb_loc -= zetab * z1 / h;
        // z2 = (rho - rf) rf gz / (4 rho): d/drho = rf gz / (4 rho) - z2 / rho
        double rhob = zetab * (rf * gz / (4.0 * rho) - z2 / rho);
        mBb += rhob * (rs - rf);
        // first qfix(h, hu, hv, hm, pA) -> (hB.., uB, vB, mB), hB = h
        double qhb = hb_loc, qhub = 0.0, qhvb = 0.0, qhmb = 0.0, qpb = pBb;
        qfix_b(P, h, hu, hv, hm, pA, gz, qhb, qhub, qhvb, qhmb, qpb, uBb, vBb, mBb);
        // pA = p - dt 3 vnorm tanpsi alphainv / h
        double pAb = qpb;
        double T = dt * 3.0 * vnorm * sv.tanpsi * sv.alphainv;
        double Tb = -pAb / h;
        double hbb = qhb + pAb * T / (h * h);
        double vnormb = Tb * dt * 3.0 * sv.tanpsi * sv.alphainv;
        double tanpsib = Tb * dt * 3.0 * vnorm * sv.alphainv;
        alphainvb += Tb * dt * 3.0 * vnorm * sv.tanpsi;
        // vnorm = nrm / h
        double nrmb = vnormb / h;
        hbb -= vnormb * vnorm / h;
        if (nrm > 0.0) {
            qhub += nrmb * hu / nrm;
            qhvb += nrmb * hv / nrm;
        }
        // hu = h u, hv = h v, hm = h m
        double u_b = qhub * h, v_b = qhvb * h, m_b = qhmb * h;
        hbb += qhub * u + qhvb * v + qhmb * m;
        double p_b = pAb;
        SetVars ob{};
        ob.kperm = kpermb;
        ob.alphainv = alphainvb;
        ob.tanpsi = tanpsib;
        setvars_b<true>(P, phi, h, u, v, m, p, gz, ob, phib, hbb, u_b, v_b, m_b, p_b, pbar);
        hb = hbb; ub = u_b; vb = v_b; mb = m_b; pb = p_b;
    }
}

// src2_cell reverse: q[5] the cell state before src2 (after the update);
// qb[5] on entry the adjoint of the output state, replaced by the adjoint of
// the input state. Always true.
DC_HD bool src2_cell_b(const dclaw_params& P, double phi, double dt, const double q[5], double qb[5], double& phib,
                       double* pbar) {
    const double rs = P.rho_s, rf = P.rho_f;
    double h = q[0];
    if (h <= P.dry_tolerance) {
        for (int k = 0; k < 5; ++k) qb[k] = 0.0;
        return true;
    }
    double hu0 = q[1], hv0 = q[2], hm0 = q[3], p0 = q[4];
    double rhoh = hm0 * rs + (h - hm0) * rf;
    if (hm0 < 0.0) return true;  // identity
    const double gz = P.grav;
    double h1 = h, hu1 = hu0, hv1 = hv0, hm1 = hm0, p1 = p0, u1, v1, m1;
    qfix(P, h1, hu1, hv1, hm1, p1, u1, v1, m1, gz);
    SetVars sv = setvars<false>(P, phi, h1, u1, v1, m1, p1, gz);
    double hvnorm0 = sqrt(sq(hu1) + sq(hv1));
    double vnorm = hvnorm0 / h1;
    double u2 = u1, v2 = v1;
    double a = 0.0, vn1 = 0.0, ex = 0.0, vn2 = 0.0, hvnorm = 0.0, hu2 = 0.0, hv2 = 0.0, earg = 0.0;
    bool moving = hvnorm0 > 0.0;
    if (moving) {
        a = vnorm - dt * sv.tau / rhoh;
        vn1 = fmax2(0.0, a);
        earg = -(1.0 - m1) * 2.0 * P.mu * dt / (h1 * rhoh);
        ex = em::d_exp(earg);
        vn2 = vn1 * ex;
        hvnorm = h1 * vn2;
        hu2 = hvnorm * hu1 / hvnorm0 + 0.0 * h1 * dt;
        hv2 = hvnorm * hv1 / hvnorm0;
        u2 = hu2 / h1;
        v2 = hv2 / h1;
    }
    double h3 = h1, u3 = u2, v3 = v2, m3 = m1, p3 = p1;
    if (P.src2method != -1) mp_update_relax(P, phi, dt, h3, u3, v3, m3, p3, rhoh, gz);
    // ---- reverse ----
    if (h3 <= P.dry_tolerance) {
        for (int k = 0; k < 5; ++k) qb[k] = 0.0;
        return true;
    }
    // outputs (h3, h3 u3, h3 v3, h3 m3, p3), or Manning's update of them
    // (src2.f90:271-289): hu, hv divided by 1 + dt gamma, gamma =
    // |(hu, hv)| g cm^2 / h^(7/3), cm constant or (dd_manning) a tanh ramp
    // in h, then qfix
    double h3b, u3b, v3b, m3b, p3b;
    if (P.friction_forcing && P.manning_coefficient > 0.0 && h3 <= P.friction_depth) {
        const double hM = h3, huM = h3 * u3, hvM = h3 * v3, hmM = h3 * m3, pM = p3;
        double cm = P.manning_coefficient, th = 0.0;
        if (P.dd_manning) {
            th = em::d_tanh(300.0 * (hM - 0.05));
            cm = P.manning_max + (P.manning_coefficient - P.manning_max) * 0.5 * (1.0 + th);
        }
        const double N = sqrt(sq(huM) + sq(hvM));
        const double gamma = N * (gz * sq(cm)) / (em::d_pow_7_3(hM));
        const double D = 1.0 + dt * gamma;
        const double hu5 = huM / D, hv5 = hvM / D;
        // qfix(hM, hu5, hv5, hmM, pM) -> the outputs
        double hb = qb[0], hu5b = qb[1], hv5b = qb[2], hmMb = qb[3], pMb = qb[4];
        qfix_b(P, hM, hu5, hv5, hmM, pM, gz, hb, hu5b, hv5b, hmMb, pMb, 0.0, 0.0, 0.0);
        // hu5 = huM / D, hv5 = hvM / D
        double huMb = hu5b / D, hvMb = hv5b / D;
        const double Db = -(hu5b * hu5 + hv5b * hv5) / D;
        const double gammab = Db * dt;
        // gamma = N g cm^2 h^(-7/3)
        if (N > 0.0) {
            const double Nb = gammab * gamma / N;
            huMb += Nb * huM / N;
            hvMb += Nb * hvM / N;
            hb -= gammab * gamma * (7.0 / 3.0) / hM;
            if (P.dd_manning) {
                const double cmb = gammab * 2.0 * gamma / cm;
                hb += cmb * (P.manning_coefficient - P.manning_max) * 0.5 * 300.0 * (1.0 - th * th);
            }
        }
        // (hM, huM, hvM, hmM, pM) = (h3, h3 u3, h3 v3, h3 m3, p3)
        h3b = hb + huMb * u3 + hvMb * v3 + hmMb * m3;
        u3b = huMb * h3;
        v3b = hvMb * h3;
        m3b = hmMb * h3;
        p3b = pMb;
    } else {
        h3b = qb[0] + qb[1] * u3 + qb[2] * v3 + qb[3] * m3;
        u3b = qb[1] * h3;
        v3b = qb[2] * h3;
        m3b = qb[3] * h3;
        p3b = qb[4];
    }
    double rhohb = 0.0;
    double h1b, u2b, v2b, m1b, p1b;
    if (P.src2method != -1) {
        double hb_ = h3b, ub_ = u3b, vb_ = v3b, mb_ = m3b, pb_ = p3b;
        mp_update_relax_b(P, phi, dt, h1, u2, v2, m1, p1, rhoh, gz, hb_, ub_, vb_, mb_, pb_, rhohb, phib, pbar);
        h1b = hb_; u2b = ub_; v2b = vb_; m1b = mb_; p1b = pb_;
    } else {
        h1b = h3b; u2b = u3b; v2b = v3b; m1b = m3b; p1b = p3b;
    }
    double hu1b = 0.0, hv1b = 0.0, u1b = 0.0, v1b = 0.0, taub = 0.0;
    if (moving) {
        // u2 = hu2 / h1, v2 = hv2 / h1
        double hu2b = u2b / h1, hv2b = v2b / h1;
        h1b -= (u2b * u2 + v2b * v2) / h1;
        // hu2 = hvnorm hu1 / hvnorm0, hv2 = hvnorm hv1 / hvnorm0
        double hvnormb = (hu2b * hu1 + hv2b * hv1) / hvnorm0;
        hu1b += hu2b * hvnorm / hvnorm0;
        hv1b += hv2b * hvnorm / hvnorm0;
        double hvnorm0b = -(hu2b * hu2 + hv2b * hv2) / hvnorm0;
        // hvnorm = h1 vn2
        h1b += hvnormb * vn2;
        double vn2b = hvnormb * h1;
        // vn2 = vn1 ex, ex = exp(earg)
        double vn1b = vn2b * ex;
        double eargb = vn2b * vn1 * ex;
        // earg = -(1 - m1) 2 mu dt / (h1 rhoh)
        m1b += eargb * 2.0 * P.mu * dt / (h1 * rhoh);
        pbar[PB_MU] += eargb * earg / P.mu;
        h1b -= eargb * earg / h1;
        rhohb -= eargb * earg / rhoh;
        // vn1 = max(0, a), a = vnorm - dt tau / rhoh
        double ab = (0.0 > a) ? 0.0 : vn1b;
        double vnormb = ab;
        taub -= ab * dt / rhoh;
        rhohb += ab * dt * sv.tau / (rhoh * rhoh);
        // vnorm = hvnorm0 / h1
        hvnorm0b += vnormb / h1;
        h1b -= vnormb * vnorm / h1;
        hu1b += hvnorm0b * hu1 / hvnorm0;
        hv1b += hvnorm0b * hv1 / hvnorm0;
    } else {
        u1b += u2b;
        v1b += v2b;
    }
    // setvars(phi, h1, u1, v1, m1, p1) -> tau
    {
        SetVars ob{};
        ob.tau = taub;
        setvars_b<false>(P, phi, h1, u1, v1, m1, p1, gz, ob, phib, h1b, u1b, v1b, m1b, p1b, pbar);
    }
    // qfix(h, hu0, hv0, hm0, p0) -> (h1, hu1, hv1, hm1 (unused), p1, u1, v1, m1)
    double qh = h1b, qhu = hu1b, qhv = hv1b, qhm = 0.0, qp = p1b;
    qfix_b(P, h, hu0, hv0, hm0, p0, gz, qh, qhu, qhv, qhm, qp, u1b, v1b, m1b);
    // rhoh = hm0 rs + (h - hm0) rf
    qh += rhohb * rf;
    qhm += rhohb * (rs - rf);
    qb[0] = qh; qb[1] = qhu; qb[2] = qhv; qb[3] = qhm; qb[4] = qp;
    return true;
}

// ---------------------------------------------------------------------------
// Stage B reverse on cell (i, j): tdb = adjoints of (fs, taudir_x,
// taudir_y). Accumulates the cell's qB adjoint into qb[5] and the adjoints of
// the neighbours' depths into nb[4] (left, right, bottom, top).
// bedb[5] += adjoints of the beds of the cell and of its neighbours L, R,
// B, T (eta = h + b enters the driving forces)
DC_HD void stage_taudir_b(const dclaw_params& P, const Geom& g, const Work& W, int i, int j, const double tdb[3],
                          double qb[5], double nb[4], double* pbar, double bedb[5]) {
    if (i < 0 || j < 0 || i > g.mx + 1 || j > g.my + 1) return;
    const size_t pi = pidx(g, i, j);
    const double dry = P.dry_tolerance;
    const double gz = P.grav;
    const double* qh = W.qB;
    double h = qh[pi];
    double hu0 = W.qB[W.npad + pi], hv0 = W.qB[2 * W.npad + pi];
    double hm0 = W.qB[3 * W.npad + pi], p0 = W.qB[4 * W.npad + pi];
    const size_t pL = pidx(g, i - 1, j), pR = pidx(g, i + 1, j), pB = pidx(g, i, j - 1), pT = pidx(g, i, j + 1);
    double hL = qh[pL], hR = qh[pR], hB = qh[pB], hT = qh[pT];
    double b = W.bP[pi];
    double eta0 = h + b;
    double etaL0 = hL + W.bP[pL], etaL = etaL0;
    bool mL = false, mR = false, mB = false, mT = false;  // neighbour eta replaced by eta0
    if (hL < dry && !(etaL0 < eta0)) { etaL = eta0; mL = true; }
    double etaR0 = hR + W.bP[pR], etaR = etaR0;
    if (hR < dry && !(etaR0 < eta0)) { etaR = eta0; mR = true; }
    double etaB0 = hB + W.bP[pB], etaB = etaB0;
    if (hB < dry && !(etaB0 < eta0)) { etaB = eta0; mB = true; }
    double etaT0 = hT + W.bP[pT], etaT = etaT0;
    if (hT < dry && !(etaT0 < eta0)) { etaT = eta0; mT = true; }
    // eta chain when the centre is dry: eta = min(etaL, eta0); eta = min(etaB, eta)
    int esrc = 0;  // 0: eta0, 1: etaL, 2: etaB
    double eta = eta0;
    if (h < dry) {
        double e1 = fmin2(etaL, eta0);
        int s1 = (etaL < eta0) ? 1 : 0;
        double e2 = fmin2(etaB, e1);
        esrc = (etaB < e1) ? 2 : s1;
        eta = e2;
    }
    if ((h + hL + hB + hR + hT) < dry) return;
    double hh = h, hu = hu0, hv = hv0, hm = hm0, p = p0, u, v, m;
    qfix(P, hh, hu, hv, hm, p, u, v, m, gz);
    SetVars sv = setvars<false>(P, P.phi, hh, u, v, m, p, gz);
    const double dx = g.dx, dy = g.dy;
    const double sint = 0.0;
    double FxL = -gz * 0.5 * (hh + hL) * (eta - etaL) / (dx) + gz * 0.5 * (hh + hL) * sint;
    double FyL = -gz * 0.5 * (hh + hB) * (eta - etaB) / (dy);
    double FxR = -gz * 0.5 * (hh + hR) * (etaR - eta) / (dx) + gz * 0.5 * (hh + hR) * sint;
    double FyR = -gz * 0.5 * (hh + hT) * (etaT - eta) / (dy);
    int fxs = 0, fys = 0;  // 0: zero, 1: FxL, 2: FxR
    double Fx = 0.0, Fy = 0.0;
    if (FxL * FxR > 0.0) { fxs = fabs(FxL) < fabs(FxR) ? 1 : 2; Fx = fsign(fmin2(fabs(FxL), fabs(FxR)), FxL); }
    if (FyL * FyR > 0.0) { fys = fabs(FyL) < fabs(FyR) ? 1 : 2; Fy = fsign(fmin2(fabs(FyL), fabs(FyR)), FyL); }
    double hvnorm = sqrt(sq(hu) + sq(hv));
    // ---- reverse ----
    double hub = 0.0, hvb = 0.0, Fxb = 0.0, Fyb = 0.0, FxLb = 0.0, FyLb = 0.0, rhob = 0.0, taub = 0.0;
    if (hvnorm > 0.0) {
        double otx = -dx * hu / hvnorm, oty = -dy * hv / hvnorm;
        double hvnormb = 0.0;
        hub += tdb[1] * (-dx) / hvnorm;
        hvnormb -= tdb[1] * otx / hvnorm;
        hvb += tdb[2] * (-dy) / hvnorm;
        hvnormb -= tdb[2] * oty / hvnorm;
        double A = fmax2(0.0, Fx * hu), B = fmax2(0.0, Fy * hv);
        double dot = fmin2(A, B);
        if (dot > 0.0) {
            double Fproj = dot / hvnorm;
            double T = fmax2(sv.tau, 1.0e-16);
            double inner = Fproj * sv.rho / T;
            if (!(1.0 < inner)) {
                double innerb = tdb[0];
                double Fprojb = innerb * sv.rho / T;
                rhob += innerb * Fproj / T;
                if (sv.tau > 1.0e-16) taub -= innerb * inner / T;
                double dotb = Fprojb / hvnorm;
                hvnormb -= Fprojb * Fproj / hvnorm;
                if (A < B) {
                    if (!(0.0 > Fx * hu)) { Fxb += dotb * hu; hub += dotb * Fx; }
                } else {
                    if (!(0.0 > Fy * hv)) { Fyb += dotb * hv; hvb += dotb * Fy; }
                }
            }
        }
        hub += hvnormb * hu / hvnorm;
        hvb += hvnormb * hv / hvnorm;
    } else {
        double nx2 = sq(FxL) + sq(Fy);
        if (nx2 > 0.0) {
            double n = sqrt(nx2), n3 = n * nx2;
            FxLb += tdb[1] * (-dx * sq(Fy) / n3);
            Fyb += tdb[1] * (dx * FxL * Fy / n3);
        }
        double ny2 = sq(Fx) + sq(FyL);
        if (ny2 > 0.0) {
            double n = sqrt(ny2), n3 = n * ny2;
            FyLb += tdb[2] * (-dy * sq(Fx) / n3);
            Fxb += tdb[2] * (dy * FyL * Fx / n3);
        }
    }
    double FxRb = 0.0, FyRb = 0.0;
    if (fxs == 1) FxLb += Fxb; else if (fxs == 2) FxRb += Fxb;
    if (fys == 1) FyLb += Fyb; else if (fys == 2) FyRb += Fyb;
    // F = -gz 0.5 (h + hN) (e1 - e2) / d
    double hhb = 0.0, etab = 0.0, etaLb = 0.0, etaRb = 0.0, etaBb = 0.0, etaTb = 0.0;
    double hLb = 0.0, hRb = 0.0, hBb = 0.0, hTb = 0.0;
    {
        double k = -gz * 0.5 / dx;
        double sb_ = FxLb * k * (eta - etaL);
        hhb += sb_; hLb += sb_;
        double eb = FxLb * k * (hh + hL);
        etab += eb; etaLb -= eb;
        sb_ = FxRb * k * (etaR - eta);
        hhb += sb_; hRb += sb_;
        eb = FxRb * k * (hh + hR);
        etaRb += eb; etab -= eb;
        double ky = -gz * 0.5 / dy;
        sb_ = FyLb * ky * (eta - etaB);
        hhb += sb_; hBb += sb_;
        eb = FyLb * ky * (hh + hB);
        etab += eb; etaBb -= eb;
        sb_ = FyRb * ky * (etaT - eta);
        hhb += sb_; hTb += sb_;
        eb = FyRb * ky * (hh + hT);
        etaTb += eb; etab -= eb;
    }
    // eta source
    double eta0b = 0.0;
    if (esrc == 0) eta0b += etab; else if (esrc == 1) etaLb += etab; else etaBb += etab;
    auto nbeta = [&](bool mm, double eb, double& hNb, double& bNb) {
        if (mm) eta0b += eb;   // etaN replaced by eta0
        else { hNb += eb; bNb += eb; }  // etaN0 = hN + bN
    };
    nbeta(mL, etaLb, hLb, bedb[1]);
    nbeta(mR, etaRb, hRb, bedb[2]);
    nbeta(mB, etaBb, hBb, bedb[3]);
    nbeta(mT, etaTb, hTb, bedb[4]);
    double h_b = eta0b;  // eta0 = h + b
    bedb[0] += eta0b;
    // setvars and qfix
    double phib = 0.0, ub = 0.0, vb = 0.0, mb = 0.0, pb = 0.0;
    SetVars ob{};
    ob.rho = rhob;
    ob.tau = taub;
    setvars_b<false>(P, P.phi, hh, u, v, m, p, gz, ob, phib, hhb, ub, vb, mb, pb, pbar);
    pbar[PB_PHI] += phib;
    double qhb = hhb, qhub = hub, qhvb = hvb, qhmb = 0.0, qpb = pb;
    qfix_b(P, h, hu0, hv0, hm0, p0, gz, qhb, qhub, qhvb, qhmb, qpb, ub, vb, mb);
    qb[0] += qhb + h_b;
    qb[1] += qhub;
    qb[2] += qhvb;
    qb[3] += qhmb;
    qb[4] += qpb;
    nb[0] += hLb; nb[1] += hRb; nb[2] += hBb; nb[3] += hTb;
}

// Stage A reverse on padded cell (i, j): qb = adjoint of its qB state;
// returns in sb the adjoint of its source interior cell's q (source frame,
// momentum flips undone) and the source cell in (si, sj).
DC_HD void stage_b4_b(const dclaw_params& P, const Geom& g, const double* __restrict__ q_in, int i, int j,
                      const double qb[5], double sb[5], int& si_out, int& sj_out) {
    const int mx = g.mx, my = g.my;
    int si = i, sj = j;
    bool flip_u = false, flip_v = false;
    if (i < 1) {
        if (P.bc_lower[0] == DCLAW_BC_WALL) { si = 1 - i; flip_u = true; } else si = 1;
    } else if (i > mx) {
        if (P.bc_upper[0] == DCLAW_BC_WALL) { si = 2 * mx + 1 - i; flip_u = true; } else si = mx;
    }
    if (j < 1) {
        if (P.bc_lower[1] == DCLAW_BC_WALL) { sj = 1 - j; flip_v = true; } else sj = 1;
    } else if (j > my) {
        if (P.bc_upper[1] == DCLAW_BC_WALL) { sj = 2 * my + 1 - j; flip_v = true; } else sj = my;
    }
    si_out = si;
    sj_out = sj;
    const size_t plane = (size_t)mx * my;
    const size_t c = (size_t)(sj - 1) * mx + (size_t)(si - 1);
    double h = q_in[c], hu = q_in[plane + c], hv = q_in[2 * plane + c], hm = q_in[3 * plane + c],
           p = q_in[4 * plane + c];
    if (flip_u) hu = -hu;
    if (flip_v) hv = -hv;
    double h1 = h, hu1 = hu, hv1 = hv, hm1 = hm, p1 = p, u, v, m;
    qfix(P, h1, hu1, hv1, hm1, p1, u, v, m, P.grav);
    double hb = qb[0], hub = qb[1], hvb = qb[2], hmb = qb[3], pb = qb[4];
    if (h1 > 0.0) {
        double nrm = sqrt((sq(hu1) + sq(hv1)));
        double s = nrm / h1;
        if (s > P.speed_limit) {
            double sr = P.speed_limit / s;
            double srb = hub * hu1 + hvb * hv1;
            hub = hub * sr;
            hvb = hvb * sr;
            double s_b = -srb * sr / s;
            double nrmb = s_b / h1;
            hb -= s_b * s / h1;
            hub += nrmb * hu1 / nrm;
            hvb += nrmb * hv1 / nrm;
        }
    }
    qfix_b(P, h, hu, hv, hm, p, P.grav, hb, hub, hvb, hmb, pb, 0.0, 0.0, 0.0);
    if (flip_u) hub = -hub;
    if (flip_v) hvb = -hvb;
    sb[0] = hb; sb[1] = hub; sb[2] = hvb; sb[3] = hmb; sb[4] = pb;
}

}  // namespace dclaw

// ===========================================================================
// The adjoint of one whole step, as per-item stages over the staged forward
// intermediates (Work, recomputed from the step's input state):
//
//   R  adj_item_svrec    padded cell     setvars records of the rpn2 states
//                                        (after the forward stages A, B)
//   E  adj_item_src2     interior cell   src2 and the update: adjoint of the
//                                        updated state (lamq)
//   D  adj_item_flux     interface       flux differencing, 2nd-order
//                                        correction, limiter, transverse splits
//   C  adj_item_riemann  interface       the augmented solver and rpn2
//   B  adj_item_taudir   padded cell     calc_taudir
//   A  adj_item_b4       padded cell     qfix, speed limit, ghost mapping
//   G  adj_item_gather   interior cell   sums the ghost copies of each cell
//
// Every stage writes only its own item's slots and reads the previous
// stages' slots (gathers, no atomics), so each is one data-parallel launch.
namespace dclaw {

constexpr int NFB = 47;  // FluxB: self 15, left 12, right 12, a2l 4, a2r 4
constexpr int NCB = 16;  // CellB of both sides: q[5], fs, taudir; then the beds of L and R
constexpr int NTD = 14;  // taudir reverse: qb[5], neighbour depths[4], beds of the cell and L, R, B, T
constexpr int NQSB = 6;  // per padded cell: its source cell's q adjoint (5), its bed's adjoint
// the planes that need zeros in inactive blocks (all but the bed planes)
constexpr int NCB_Q = 14, NTD_Q = 9, NQSB_Q = 5;

struct AdjWork {
    double* lamq;  // 5 interior planes
    double* xfb;   // NFB x-interface planes
    double* yfb;   // NFB y-interface planes
    double* xcb;   // NCB x-interface planes
    double* ycb;   // NCB y-interface planes
    double* tdq;   // NTD padded planes
    double* qsb;   // NQSB padded planes
    double* sv;    // NSV padded planes: setvars records (svrec_cell)
    // activity of ACT_TILE x ACT_TILE blocks of padded cells (nullable: all
    // active): nonzero when a cell within ACT_REACH of the block is wet in
    // the step's b4step2 state. Every reverse item whose cell lies in an
    // inactive block has only dry cells within ACT_REACH: its outputs are
    // zeros (dry-dry solves and dry cells have no adjoint form, a wave of
    // zero norm takes no part in the limiter) or values no item reads, so
    // with the reverse planes zeroed beforehand it can be skipped.
    const uint32_t* act;
    int act_nx;    // blocks per row of padded cells
    // the beds' adjoints are wanted: the bed planes are written (solver
    // sides, calc_taudir) and summed (adj_item_b4, adj_item_gather_bed).
    // They are not zeroed in inactive blocks: their readers take only items
    // of active blocks (the others' bed adjoints are zeros).
    bool bed = false;
};

constexpr int ACT_TILE = 16, ACT_REACH = 4;

// whether the reverse items at padded cell (i, j) (interfaces: the cell on
// their high side) may contribute
DC_HD bool adj_active(const AdjWork& A, int i, int j) {
    if (!A.act) return true;
    return A.act[((j + 1) / ACT_TILE) * A.act_nx + (i + 1) / ACT_TILE] != 0u;
}

// padded cell (i, j), i in -1..mx+2, j in -1..my+2: setvars records
DC_HD void adj_item_svrec(const dclaw_params& P, const Geom& g, const Work& W, const AdjWork& A, int i, int j) {
    svrec_cell(P, W, A.sv, pidx(g, i, j));
}

DC_HD void adj_item_src2(const dclaw_params& P, const Geom& g, const Work& W, const AdjWork& A,
                         const double* __restrict__ lam_out, int i, int j, double dt, double* pbar) {
    double qn[5];
    stage_update(g, W, i, j, dt, qn, nullptr);
    const size_t plane = (size_t)g.mx * g.my;
    const size_t c = (size_t)(j - 1) * g.mx + (size_t)(i - 1);
    double qb[5];
    for (int m = 0; m < 5; ++m) qb[m] = lam_out[(size_t)m * plane + c];
    double phib = 0.0;
    src2_cell_b(P, P.phi, dt, qn, qb, phib, pbar);
    pbar[PB_PHI] += phib;
    for (int m = 0; m < 5; ++m) A.lamq[(size_t)m * plane + c] = qb[m];
}

template <int DIR>
DC_HD void adj_item_flux(const dclaw_params& P, const Geom& g, const Work& W, const AdjWork& A, int r, int i,
                         double dt) {
    double fb[30];
    flux_bar<DIR>(g, A.lamq, r, i, dt, fb);
    FluxB o;
    const double dtdx = DIR == 0 ? dt / g.dx : dt / g.dy;
    stage_flux_b<DIR>(P, g, W, r, i, dtdx, fb, o);
    double* dst = DIR == 0 ? A.xfb : A.yfb;
    const size_t np = DIR == 0 ? W.nxi : W.nyi;
    const size_t oi = DIR == 0 ? xidx(g, r, i) : yidx(g, i, r);
    for (int k = 0; k < NW; ++k) dst[(size_t)k * np + oi] = o.self[k];
    for (int k = 0; k < 12; ++k) dst[(size_t)(15 + k) * np + oi] = o.left[k];
    for (int k = 0; k < 12; ++k) dst[(size_t)(27 + k) * np + oi] = o.right[k];
    for (int k = 0; k < 4; ++k) dst[(size_t)(39 + k) * np + oi] = o.a2l[k];
    for (int k = 0; k < 4; ++k) dst[(size_t)(43 + k) * np + oi] = o.a2r[k];
}

template <int DIR>
DC_HD bool adj_item_riemann(const dclaw_params& P, const Geom& g, const Work& W, const AdjWork& A, int r, int i,
                            double* pbar) {
    const int n = DIR == 0 ? g.mx : g.my;
    const double* src = DIR == 0 ? A.xfb : A.yfb;
    const size_t np = DIR == 0 ? W.nxi : W.nyi;
    auto at = [&](int ii) -> size_t { return DIR == 0 ? xidx(g, r, ii) : yidx(g, ii, r); };
    double wb[NW];
    for (int k = 0; k < NW; ++k) wb[k] = 0.0;
    if (i >= 1 && i <= n + 1)
        for (int k = 0; k < NW; ++k) wb[k] += src[(size_t)k * np + at(i)];
    if (i + 1 >= 1 && i + 1 <= n + 1)
        for (int k = 0; k < 12; ++k) wb[3 + k] += src[(size_t)(15 + k) * np + at(i + 1)];
    if (i - 1 >= 1 && i - 1 <= n + 1)
        for (int k = 0; k < 12; ++k) wb[3 + k] += src[(size_t)(27 + k) * np + at(i - 1)];
    CellB Lc, Rc;
    zero_cellb(Lc);
    zero_cellb(Rc);
    bool ok = stage_riemann_b<DIR>(P, g, W, A.sv, r, i, wb, Lc, Rc, pbar);
    double* dst = DIR == 0 ? A.xcb : A.ycb;
    const size_t oi = at(i);
    for (int k = 0; k < 5; ++k) {
        dst[(size_t)k * np + oi] = Lc.q[k];
        dst[(size_t)(7 + k) * np + oi] = Rc.q[k];
    }
    dst[(size_t)5 * np + oi] = Lc.fs;
    dst[(size_t)6 * np + oi] = Lc.taudir;
    dst[(size_t)12 * np + oi] = Rc.fs;
    dst[(size_t)13 * np + oi] = Rc.taudir;
    if (A.bed) {
        dst[(size_t)14 * np + oi] = Lc.b;
        dst[(size_t)15 * np + oi] = Rc.b;
    }
    return ok;
}

// padded cell (i, j), i in -1..mx+2, j in -1..my+2
DC_HD void adj_item_taudir(const dclaw_params& P, const Geom& g, const Work& W, const AdjWork& A, int i, int j,
                           double* pbar) {
    double tdb[3] = {0.0, 0.0, 0.0};
    const size_t nx = W.nxi, ny = W.nyi;
    if (j >= 0 && j <= g.my + 1) {
        if (i + 1 >= 0 && i + 1 <= g.mx + 2) {
            const size_t o = xidx(g, j, i + 1);
            tdb[0] += A.xcb[5 * nx + o];
            tdb[1] += A.xcb[6 * nx + o];
        }
        if (i >= 0 && i <= g.mx + 2) {
            const size_t o = xidx(g, j, i);
            tdb[0] += A.xcb[12 * nx + o];
            tdb[1] += A.xcb[13 * nx + o];
        }
    }
    if (i >= 0 && i <= g.mx + 1) {
        if (j + 1 >= 0 && j + 1 <= g.my + 2) {
            const size_t o = yidx(g, j + 1, i);
            tdb[0] += A.ycb[5 * ny + o];
            tdb[2] += A.ycb[6 * ny + o];
        }
        if (j >= 0 && j <= g.my + 2) {
            const size_t o = yidx(g, j, i);
            tdb[0] += A.ycb[12 * ny + o];
            tdb[2] += A.ycb[13 * ny + o];
        }
    }
    double qb[5] = {0.0, 0.0, 0.0, 0.0, 0.0}, nb[4] = {0.0, 0.0, 0.0, 0.0};
    double bedb[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    stage_taudir_b(P, g, W, i, j, tdb, qb, nb, pbar, bedb);
    const size_t pi = pidx(g, i, j);
    for (int k = 0; k < 5; ++k) A.tdq[(size_t)k * W.npad + pi] = qb[k];
    for (int k = 0; k < 4; ++k) A.tdq[(size_t)(5 + k) * W.npad + pi] = nb[k];
    if (A.bed)
        for (int k = 0; k < 5; ++k) A.tdq[(size_t)(9 + k) * W.npad + pi] = bedb[k];
}

DC_HD void adj_item_b4(const dclaw_params& P, const Geom& g, const Work& W, const AdjWork& A,
                       const double* __restrict__ q_in, int i, int j) {
    double qb[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    const size_t nx = W.nxi, ny = W.nyi, np = W.npad;
    const int mx = g.mx, my = g.my;
    if (i >= 1 && i <= mx && j >= 1 && j <= my) {
        const size_t plane = (size_t)mx * my, c = (size_t)(j - 1) * mx + (size_t)(i - 1);
        for (int m = 0; m < 5; ++m) qb[m] += A.lamq[(size_t)m * plane + c];
    }
    // solver sides and transverse-split states
    double a2x[4] = {0.0, 0.0, 0.0, 0.0}, a2y[4] = {0.0, 0.0, 0.0, 0.0};
    if (j >= 0 && j <= my + 1) {
        if (i + 1 >= 0 && i + 1 <= mx + 2) {
            const size_t o = xidx(g, j, i + 1);
            for (int m = 0; m < 5; ++m) qb[m] += A.xcb[(size_t)m * nx + o];
            if (i + 1 >= 1 && i + 1 <= mx + 1)
                for (int k = 0; k < 4; ++k) a2x[k] += A.xfb[(size_t)(39 + k) * nx + o];
        }
        if (i >= 0 && i <= mx + 2) {
            const size_t o = xidx(g, j, i);
            for (int m = 0; m < 5; ++m) qb[m] += A.xcb[(size_t)(7 + m) * nx + o];
            if (i >= 1 && i <= mx + 1)
                for (int k = 0; k < 4; ++k) a2x[k] += A.xfb[(size_t)(43 + k) * nx + o];
        }
    }
    if (i >= 0 && i <= mx + 1) {
        if (j + 1 >= 0 && j + 1 <= my + 2) {
            const size_t o = yidx(g, j + 1, i);
            for (int m = 0; m < 5; ++m) qb[m] += A.ycb[(size_t)m * ny + o];
            if (j + 1 >= 1 && j + 1 <= my + 1)
                for (int k = 0; k < 4; ++k) a2y[k] += A.yfb[(size_t)(39 + k) * ny + o];
        }
        if (j >= 0 && j <= my + 2) {
            const size_t o = yidx(g, j, i);
            for (int m = 0; m < 5; ++m) qb[m] += A.ycb[(size_t)(7 + m) * ny + o];
            if (j >= 1 && j <= my + 1)
                for (int k = 0; k < 4; ++k) a2y[k] += A.yfb[(size_t)(43 + k) * ny + o];
        }
    }
    const size_t pi = pidx(g, i, j);
    load_a2_b(P, W, pi, 1, 2, a2x, qb);
    load_a2_b(P, W, pi, 2, 1, a2y, qb);
    // calc_taudir: the cell's own stencil and its neighbours' stencils
    for (int k = 0; k < 5; ++k) qb[k] += A.tdq[(size_t)k * np + pi];
    if (i - 1 >= -1) qb[0] += A.tdq[(size_t)6 * np + pidx(g, i - 1, j)];
    if (i + 1 <= mx + 2) qb[0] += A.tdq[(size_t)5 * np + pidx(g, i + 1, j)];
    if (j - 1 >= -1) qb[0] += A.tdq[(size_t)8 * np + pidx(g, i, j - 1)];
    if (j + 1 <= my + 2) qb[0] += A.tdq[(size_t)7 * np + pidx(g, i, j + 1)];
    double sb[5];
    int si, sj;
    stage_b4_b(P, g, q_in, i, j, qb, sb, si, sj);
    for (int k = 0; k < 5; ++k) A.qsb[(size_t)k * np + pi] = sb[k];
    if (!A.bed) return;
    // the cell's bed: the solver sides it takes (x and y), its own
    // calc_taudir stencil and its neighbours' (items of active blocks only:
    // the others' bed adjoints are zeros and their planes are not zeroed)
    double bb = 0.0;
    if (j >= 0 && j <= my + 1) {
        if (i + 1 >= 0 && i + 1 <= mx + 2 && adj_active(A, i + 1, j)) bb += A.xcb[(size_t)14 * nx + xidx(g, j, i + 1)];
        if (i >= 0 && i <= mx + 2 && adj_active(A, i, j)) bb += A.xcb[(size_t)15 * nx + xidx(g, j, i)];
    }
    if (i >= 0 && i <= mx + 1) {
        if (j + 1 >= 0 && j + 1 <= my + 2 && adj_active(A, i, j + 1)) bb += A.ycb[(size_t)14 * ny + yidx(g, j + 1, i)];
        if (j >= 0 && j <= my + 2 && adj_active(A, i, j)) bb += A.ycb[(size_t)15 * ny + yidx(g, j, i)];
    }
    if (adj_active(A, i, j)) bb += A.tdq[(size_t)9 * np + pi];
    if (i + 1 <= mx + 2 && adj_active(A, i + 1, j)) bb += A.tdq[(size_t)10 * np + pidx(g, i + 1, j)];
    if (i - 1 >= -1 && adj_active(A, i - 1, j)) bb += A.tdq[(size_t)11 * np + pidx(g, i - 1, j)];
    if (j + 1 <= my + 2 && adj_active(A, i, j + 1)) bb += A.tdq[(size_t)12 * np + pidx(g, i, j + 1)];
    if (j - 1 >= -1 && adj_active(A, i, j - 1)) bb += A.tdq[(size_t)13 * np + pidx(g, i, j - 1)];
    A.qsb[(size_t)5 * np + pi] = bb;
}

// interior source index of padded coordinate x (bc2amr mapping)
DC_HD int bc_source(int x, int n, int lo, int hi) {
    if (x < 1) return lo == DCLAW_BC_WALL ? 1 - x : 1;
    if (x > n) return hi == DCLAW_BC_WALL ? 2 * n + 1 - x : n;
    return x;
}

DC_HD void adj_item_gather(const dclaw_params& P, const Geom& g, const AdjWork& A, const Work& W,
                           double* __restrict__ lam_in, int i, int j) {
    const int mx = g.mx, my = g.my;
    int ci[5], cj[5], ni = 0, nj = 0;
    const int candx[5] = {i, -1, 0, mx + 1, mx + 2};
    const int candy[5] = {j, -1, 0, my + 1, my + 2};
    for (int k = 0; k < 5; ++k) {
        if (k > 0 && candx[k] >= 1 && candx[k] <= mx) continue;
        if (bc_source(candx[k], mx, P.bc_lower[0], P.bc_upper[0]) == i) ci[ni++] = candx[k];
    }
    for (int k = 0; k < 5; ++k) {
        if (k > 0 && candy[k] >= 1 && candy[k] <= my) continue;
        if (bc_source(candy[k], my, P.bc_lower[1], P.bc_upper[1]) == j) cj[nj++] = candy[k];
    }
    const size_t plane = (size_t)mx * my, c = (size_t)(j - 1) * mx + (size_t)(i - 1);
    for (int m = 0; m < 5; ++m) {
        double s = 0.0;
        for (int b = 0; b < nj; ++b)
            for (int a = 0; a < ni; ++a) s += A.qsb[(size_t)m * W.npad + pidx(g, ci[a], cj[b])];
        lam_in[(size_t)m * plane + c] = s;
    }
}

// interior cell (i, j): bbar += the adjoint of its bed, summed over the
// padded cells whose bed is a copy of it (the ghost bed is the nearest
// interior cell's, whatever the boundary condition)
DC_HD void adj_item_gather_bed(const Geom& g, const AdjWork& A, const Work& W, double* __restrict__ bbar, int i,
                               int j) {
    const int mx = g.mx, my = g.my;
    int ci[3], cj[3], ni = 1, nj = 1;
    ci[0] = i;
    cj[0] = j;
    if (i == 1) { ci[ni++] = -1; ci[ni++] = 0; }
    if (i == mx) { ci[ni++] = mx + 1; ci[ni++] = mx + 2; }
    if (j == 1) { cj[nj++] = -1; cj[nj++] = 0; }
    if (j == my) { cj[nj++] = my + 1; cj[nj++] = my + 2; }
    double s = 0.0;
    for (int b = 0; b < nj; ++b)
        for (int a = 0; a < ni; ++a)
            if (adj_active(A, ci[a], cj[b])) s += A.qsb[(size_t)5 * W.npad + pidx(g, ci[a], cj[b])];
    bbar[(size_t)(j - 1) * mx + (size_t)(i - 1)] += s;
}

}  // namespace dclaw
