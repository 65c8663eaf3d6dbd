// physics.cuh -- pointwise D-Claw closures and interface solvers, FP64, sm_100a.
//
// Device restatement of the reference's pointwise physics. Every expression
// keeps the operand order of the Fortran (left-to-right, as gfortran -O
// evaluates it) and the library is compiled with --fmad=false, so additions
// and products round exactly as on the host; sqrt and division are IEEE
// correctly rounded on the GPU as on x86-64. The elementary functions (exp,
// atan, tan, tanh, h^(7/3)) are the project's own deterministic versions in
// elementary.cuh, so the device returns the same bits as a host build.
//
// Reference map (paths in the youryugi/dclaw tree):
//   qfix          src/2d/dig/digclaw_module.f90:285-345
//   qfix_cmass    src/2d/dig/digclaw_module.f90:353-387
//   setvars       src/2d/dig/digclaw_module.f90:394-491
//   riemanntype   src/2d/dig/riemannsolvers_dclaw.f:526-637
//   riemann_solve src/2d/dig/riemannsolvers_dclaw.f:3-521 with the wall /
//                 inundation set-up of src/2d/dig/rpn2_dclaw.f:124-272
//   rpt2_split    src/2d/dig/rpt2_dclaw.f:78-263
//   src2_cell     src/2d/dig/src2.f90:100-300 + mp_update.f90:710-789
//   mp_update_fe4quad  src/2d/dig/mp_update.f90:38-707 (src2method 2)
//
// The hchi (segregation) and bdif (bed change) components are identically
// zero for the accepted configurations; their contributions are the exact
// zeros the reference adds, so they are not carried.
#pragma once
#include <stdint.h>
#include <math.h>
#include "../../include/dclaw_b200.h"

#if defined(__CUDACC__)
#define DC_HD __host__ __device__ __forceinline__
#else
// host build of the same stage code (used only by the CPU emulation test)
#define DC_HD inline
#endif

#include "elementary.cuh"

// Large device routines can be compiled out of line (-DDCLAW_OUTLINE_BIG)
// to shrink the tile kernel's code; inline is the default.
#if defined(__CUDACC__) && defined(DCLAW_OUTLINE_BIG)
#define DC_BIG __host__ __device__ __noinline__
#else
#define DC_BIG DC_HD
#endif

namespace dclaw {

// branch bits recorded per interface (same meaning as the oracle's)
constexpr uint32_t BR_DRY = 1u << 0, BR_WALL = 1u << 1, BR_SONIC = 1u << 2, BR_STATIC = 1u << 3,
                   BR_WET4 = 1u << 4, BR_REVERT_L = 1u << 5, BR_RPT1 = 1u << 6, BR_RPT2 = 1u << 7;
DC_HD constexpr uint32_t br_lim(int mw, uint32_t code) { return code << (8 + 3 * (mw - 1)); }
DC_HD constexpr uint32_t br_up(int mw) { return 1u << (23 + (mw - 1)); }

DC_HD double sq(double x) { return x * x; }
// Fortran MAX/MIN of two reals, SIGN(a,b)
DC_HD double fmax2(double a, double b) { return a > b ? a : b; }
DC_HD double fmin2(double a, double b) { return a < b ? a : b; }
DC_HD double fsign(double a, double b) { return copysign(fabs(a), b); }

// ---------------------------------------------------------------------------
// Cell state after qfix: conserved (h, hu, hv, hm, p) plus primitives.
struct Prim {
    double h, hu, hv, hm, p;  // hu/hv in the caller's (normal, tangential) order
    double u, v, m;
};

// qfix on (h, hu, hv, hm, p); chi = hchi/h = 0 is not carried.
DC_HD void qfix(const dclaw_params& P, double& h, double& hu, double& hv, double& hm,
                                     double& p, double& u, double& v, double& m, double gz) {
    if (h <= P.dry_tolerance) {
        h = 0.0; hu = 0.0; hv = 0.0; hm = 0.0; p = 0.0;
        u = 0.0; v = 0.0; m = 0.0;
        return;
    }
    u = hu / h;
    v = hv / h;
    m = hm / h;
    m = fmax2(m, 0.0);
    m = fmin2(m, 1.0);
    hm = h * m;
    double rho = P.rho_s * m + (1.0 - m) * P.rho_f;
    double pmax = rho * gz * h;
    p = fmax2(0.0, p);
    p = fmin2(pmax, p);
}

// qfix for a cell whose (h, hu, hv) are known and wet or zero; only the
// fields qfix changes are recomputed (hm, p, m). u, v are the same
// quotients every application produces, so callers compute them once.
DC_HD void qfix_mp(const dclaw_params& P, double h, double& hm, double& p, double& m,
                                        double gz) {
    m = hm / h;
    m = fmax2(m, 0.0);
    m = fmin2(m, 1.0);
    hm = h * m;
    double rho = P.rho_s * m + (1.0 - m) * P.rho_f;
    double pmax = rho * gz * h;
    p = fmax2(0.0, p);
    p = fmin2(pmax, p);
}

DC_HD void qfix_cmass(const dclaw_params& P, double& h, double& m, double& p, double& rho,
                                           double& p_exc, double& hu, double& hv, double& hm, double u,
                                           double v, double rhoh, double gz) {
    m = fmax2(m, 0.0);
    m = fmin2(m, 1.0);
    rho = m * (P.rho_s - P.rho_f) + P.rho_f;
    h = rhoh / rho;
    double p_exc_max = rhoh * gz - P.rho_f * h * gz;
    double p_exc_min = 0.0 - P.rho_f * h * gz;
    p_exc = fmax2(p_exc_min, p_exc);
    p_exc = fmin2(p_exc_max, p_exc);
    p = P.rho_f * gz * h + p_exc;
    hu = h * u;
    hv = h * v;
    hm = h * m;
}

struct SetVars {
    double rho, kperm, alphainv, m_eq, tanpsi, tau;
};

// setvars. `phi` is the basal friction angle, chi the species fraction
// (read only with segregation = 1: kperm times 10^(delta_kr_order 2 (chi -
// 1/2)), digclaw_module.f90:418-431; kr_chi = 1 otherwise).
template <bool NEED_ALL>
DC_BIG SetVars setvars(const dclaw_params& P, double phi, double h, double u, double v,
                                           double m, double p, double gz, double chi = 0.0) {
    SetVars o;
    o.rho = m * (P.rho_s - P.rho_f) + P.rho_f;
    double kr_chi = 1.0;
    if (NEED_ALL && P.segregation == 1) kr_chi = em::d_pow(10.0, P.delta_kr_order * 2.0 * (chi - 0.5));
    if (NEED_ALL) o.kperm = kr_chi * P.kref * em::d_exp(-(m - P.mref) / (0.04));
    else o.kperm = 0.0;
    double sig_eff = fmax2(0.0, o.rho * gz * h - p);
    double sig_0 = 0.0;
    if (P.alphamethod == 0) sig_0 = P.sigma_0;
    else if (P.alphamethod == 1) sig_0 = 0.50 * P.alpha_c * P.rho_f * (P.rho_s - P.rho_f) * gz * h / o.rho;
    o.alphainv = m * (sig_eff + sig_0) / P.alpha_c;
    double vnorm = sqrt(sq(u) + sq(v));
    double shear;
    if (h > P.dry_tolerance) shear = 2.0 * vnorm / h;
    else shear = 0.0;
    double Nden = P.rho_s * sq(shear * P.delta) + sig_eff;
    double Nnum = P.mu * shear;
    if (Nnum <= 0.0) o.m_eq = P.m_crit;
    else o.m_eq = P.m_crit * (sqrt(Nden) / (sqrt(Nden) + sqrt(Nnum)));
    o.tanpsi = P.c1 * (m - o.m_eq);
    double psi = em::d_atan(P.c1 * (m - o.m_eq));
    double tau = sig_eff * em::d_tan(phi + psi);
    o.tau = tau * 0.5 * (1.0 + em::d_tanh(100.0 * (m - 0.1)));
    return o;
}

// ---------------------------------------------------------------------------
struct RType {
    double hm, s1m, s2m;
    bool rare1, rare2;
};

// riemanntype with maxiter = 1
DC_HD RType riemanntype(double hL, double hR, double uL, double uR, double drytol, double g) {
    RType o;
    double h_min = fmin2(hR, hL);
    double h_max = fmax2(hR, hL);
    double delu = uR - uL;
    if (h_min <= drytol) {
        o.hm = 0.0;
        o.s1m = uR + uL - 2.0 * sqrt(g * hR) + 2.0 * sqrt(g * hL);
        o.s2m = o.s1m;
        if (hL <= 0.0) { o.rare2 = true; o.rare1 = false; }
        else { o.rare1 = true; o.rare2 = false; }
    } else {
        double F_min = delu + 2.0 * (sqrt(g * h_min) - sqrt(g * h_max));
        double F_max = delu + (h_max - h_min) * (sqrt(.5 * g * (h_max + h_min) / (h_max * h_min)));
        if (F_min > 0.0) {
            double hm = (1.0 / (16.0 * g)) * sq(fmax2(0.0, -delu + 2.0 * (sqrt(g * hL) + sqrt(g * hR))));
            o.hm = hm;
            double sghm = sqrt(g * hm);
            o.s1m = uL + 2.0 * sqrt(g * hL) - 3.0 * sghm;
            o.s2m = uR - 2.0 * sqrt(g * hR) + 3.0 * sghm;
            o.rare1 = true;
            o.rare2 = true;
        } else if (F_max <= 0.0) {
            double h0 = h_max;
            double gL = sqrt(.5 * g * (1.0 / h0 + 1.0 / hL));
            double gR = sqrt(.5 * g * (1.0 / h0 + 1.0 / hR));
            double F0 = delu + (h0 - hL) * gL + (h0 - hR) * gR;
            double dfdh = gL - g * (h0 - hL) / (4.0 * (sq(h0)) * gL) + gR - g * (h0 - hR) / (4.0 * (sq(h0)) * gR);
            double slope = 2.0 * sqrt(h0) * dfdh;
            h0 = sq(sqrt(h0) - F0 / slope);
            double hm = h0;
            o.hm = hm;
            double u1m = uL - (hm - hL) * sqrt((.5 * g) * (1.0 / hm + 1.0 / hL));
            double u2m = uR + (hm - hR) * sqrt((.5 * g) * (1.0 / hm + 1.0 / hR));
            double sghm = sqrt(g * hm);
            o.s1m = u1m - sghm;
            o.s2m = u2m + sghm;
            o.rare1 = false;
            o.rare2 = false;
        } else {
            double h0 = h_min;
            double F0 = delu + 2.0 * (sqrt(g * h0) - sqrt(g * h_max))
                        + (h0 - h_min) * sqrt(.5 * g * (1.0 / h0 + 1.0 / h_min));
            double slope = (F_max - F0) / (h_max - h_min);
            h0 = h0 - F0 / slope;
            double hm = h0;
            o.hm = hm;
            double sghm = sqrt(g * hm);
            if (hL > hR) {
                double a = uL + 2.0 * sqrt(g * hL);
                o.s1m = a - 3.0 * sghm;
                o.s2m = a - sghm;
                o.rare1 = true;
                o.rare2 = false;
            } else {
                double a = uR - 2.0 * sqrt(g * hR);
                o.s2m = a + 3.0 * sghm;
                o.s1m = a + sghm;
                o.rare2 = true;
                o.rare1 = false;
            }
        }
    }
    return o;
}

// Result of one interface solve in compact form. In the reference's five
// clawpack waves: wave 1 = (w1h, w1n, w1t, w1m, w1p) speed s1; wave 2 =
// (w2h, w2n, 0, 0, 0) speed s2; waves 3 and 4 are exact zero vectors after
// the middle-wave merge (delta_huvm_revert); wave 5 = (w5h, ...) speed s5.
// "n" is the normal momentum component, "t" the tangential one.
struct Waves {
    double s1, s2, s5;
    double w1h, w1n, w1t, w1m, w1p;
    double w2h, w2n;
    double w5h, w5n, w5t, w5m, w5p;
};

DC_HD void zero_waves(Waves& w) {
    w.s1 = w.s2 = w.s5 = 0.0;
    w.w1h = w.w1n = w.w1t = w.w1m = w.w1p = 0.0;
    w.w2h = w.w2n = 0.0;
    w.w5h = w.w5n = w.w5t = w.w5m = w.w5p = 0.0;
}

// Side state handed to the solver (after the two rpn2 qfix passes).
struct Side {
    double h, hn, ht, hm, p;  // conserved, normal/tangential momentum
    double un, ut, m;         // primitives from the last qfix
    double b, taudir, fs;     // bed, static-friction direction and factor of safety
    // setvars outputs for this state (rho, tau), valid when h >= drytol
    double rho_sv, tau_sv;
    double chi;               // species fraction; read only for the species waves
};

// The species (hchi) components of the waves, for the full-state step:
// waves 1 and 5 after the middle-wave merge (wave 2's is merged too).
struct ChiWaves {
    double w1c, w5c;
};

// riemann_dig2_aug_sswave_ez with the wall / inundation preprocessing of
// rpn2 (the dry-dry skip is done by the caller). bed_normal = 0: theta = 0.
// L and R carry setvars (rho, tau) of their states; the mirrored ghost of a
// wall problem has the same closures as its source because setvars depends
// on the velocity only through u^2 + v^2. With cw, the species waves are
// computed too from L.chi, R.chi (riemannsolvers_dclaw.f:463-468, merged at
// :495-510; the dry side takes the wet side's chi, rpn2_dclaw.f:197,226).
DC_BIG Waves riemann_solve(const dclaw_params& P, Side L, Side R, uint32_t* br, ChiWaves* cw = nullptr) {
    const double grav = P.grav;
    const double drytol = P.dry_tolerance;
    double wall1 = 1.0, wall2 = 1.0, wall3 = 1.0;
    bool wallprob = false;
    double hL = L.h, hR = R.h, huL = L.hn, huR = R.hn, hvL = L.ht, hvR = R.ht;
    double hmL = L.hm, hmR = R.hm, pL = L.p, pR = R.p, bL = L.b, bR = R.b;
    double uL = L.un, uR = R.un, vL = L.ut, vR = R.ut, mL = L.m, mR = R.m;
    double rhoL_sv = L.rho_sv, tauL_sv = L.tau_sv, rhoR_sv = R.rho_sv, tauR_sv = R.tau_sv;
    double chiL = 0.0, chiR = 0.0;
    if (cw) {
        chiL = L.chi;
        chiR = R.chi;
    }
    if (hR <= drytol) {
        hR = 0.0;
        pR = 0.0;
        mR = mL;
        chiR = chiL;
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
        hL = 0.0;
        pL = 0.0;
        mL = mR;
        chiL = chiR;
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
    if (wallprob && br) *br |= BR_WALL;

    // ---- riemann_dig2_aug_sswave_ez ----
    const double criticaltol = fmax2(drytol * grav, 1e-6);
    const double criticaltol_2 = sqrt(criticaltol);
    const double gz = grav;  // cos(0) = 1
    double rhoL, rhoR, tauL, tauR;
    if (hL >= drytol && hR >= drytol) {
        rhoL = rhoL_sv; tauL = tauL_sv;
        rhoR = rhoR_sv; tauR = tauR_sv;
    } else if (hL >= drytol) {
        rhoL = rhoL_sv; tauL = tauL_sv;
        rhoR = rhoL_sv;
        tauR = 0.5 * tauL;
    } else {
        rhoL = rhoR_sv;
        rhoR = rhoR_sv; tauR = tauR_sv;
        tauL = 0.5 * tauR;
    }
    tauL = L.fs * tauL;
    tauR = R.fs * tauR;
    double rho = 0.5 * (rhoL + rhoR);
    double gamma, gammaL, gammaR;
    if (P.src2method == -1) {
        gamma = P.rho_f / rho;
        gammaL = P.rho_f / rhoL;
        gammaR = P.rho_f / rhoR;
    } else {
        gamma = 0.25 * (P.rho_f + 3.0 * rho) / rho;
        gammaL = 0.25 * (P.rho_f + 3.0 * rhoL) / rhoL;
        gammaR = 0.25 * (P.rho_f + 3.0 * rhoR) / rhoR;
    }
    // kappa = 1: eps = 1 + 0*gamma = 1, geps = gz
    const double geps = gz;

    double sqhL = sqrt(hL), sqhR = sqrt(hR);
    double cL = sqrt(geps * hL), cR = sqrt(geps * hR);
    double sL = uL - cL;
    double sR = uR + cR;
    double uhat = (sqhL * uL + sqhR * uR) / (sqhR + sqhL);
    double chat = sqrt(geps * 0.5 * (hR + hL));
    double sRoe1 = uhat - chat;
    double sRoe2 = uhat + chat;
    double sE1 = fmin2(sL, sRoe1);
    double sE2 = fmax2(sR, sRoe2);
    double sw1 = sE1, sw3 = sE2;
    double u = uhat;

    RType rt = riemanntype(hL, hR, uL, uR, drytol, geps);
    sw1 = fmin2(sw1, rt.s2m);
    sw3 = fmax2(sw3, rt.s1m);
    double sw2 = 0.5 * (sw3 + sw1);

    double hstarHLL = fmax2((huL - huR + sE2 * hR - sE1 * hL) / (sE2 - sE1), 0.0);
    bool rarecorrector = false;
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
                rarecorrector = true;
                if (rare1st > rare2st) sw2 = rt.s1m;
                else if (rare2st > rare1st) sw2 = rt.s2m;
                else sw2 = 0.5 * (rt.s1m + rt.s2m);
            }
        }
        if (hstarHLL < fmin2(hL, hR) / 5.0) rarecorrector = false;
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
    if (sonic && br) *br |= BR_SONIC;

    double source2dx;
    if (sonic) source2dx = -gz * hbar * delb;
    else source2dx = -gz * hbar * delb * s1s2tilde / s1s2bar;
    source2dx = fmin2(source2dx, gz * fmax2(-hL * delb, -hR * delb));
    source2dx = fmax2(source2dx, gz * fmin2(-hL * delb, -hR * delb));
    if (fabs(u) <= 0.0) source2dx = -hbar * gz * delb;

    double deldelh;
    if (sonic) deldelh = -delb;
    else deldelh = delb * gz * hbar / s1s2bar;
    if (sE1 < -criticaltol && sE2 > criticaltol) {
        deldelh = fmin2(deldelh, hstarHLL * (sE2 - sE1) / sE2);
        deldelh = fmax2(deldelh, hstarHLL * (sE2 - sE1) / sE1);
    } else if (sE1 >= criticaltol) {
        deldelh = fmin2(deldelh, hstarHLL * (sE2 - sE1) / sE1);
        deldelh = fmax2(deldelh, -hL);
    } else if (sE2 <= -criticaltol) {
        deldelh = fmin2(deldelh, hR);
        deldelh = fmax2(deldelh, hstarHLL * (sE2 - sE1) / sE2);
    }

    double del0 = hR - hL - deldelh;
    double del1 = huR - huL;
    // kappa = 1: the (1-kappa) pressure term adds an exact zero
    double del2 = hR * sq(uR) + 0.5 * 1.0 * gz * sq(hR) - (hL * sq(uL) + 0.5 * 1.0 * gz * sq(hL));
    double grg = gamma * rho * gz;
    double del4 = -gamma * rho * gz * u * (hR - hL) + grg * del1 + u * (pR - pL);

    double vnorm = sqrt(sq(uR) + sq(uL) + sq(vR) + sq(vL));
    bool is_static = false;
    double tausource;
    if (vnorm > 0.0) {
        tausource = 0.0;
    } else {
        double tdR = R.taudir;
        double fr = 0.5 * fabs(tdR * tauR / rhoR + tauL * tdR / rhoL);
        if (fr > fabs(del2 - source2dx)) {
            tausource = del2 - source2dx;
            del1 = 0.0; del0 = 0.0; del4 = 0.0;
            is_static = true;
        } else {
            tausource = 0.5 * ((tdR * tauR / rhoR) + (tauL * tdR / rhoL));
            tausource = fsign(tausource, del2 - source2dx);
        }
    }
    if (is_static && br) *br |= BR_STATIC;
    if (wallprob) tausource = 0.0;
    del2 = del2 - source2dx - tausource;

    double a = sw1, bb = sw2, c = sw3;
    double beta1, beta2, beta3;
    double R12, R22;  // r2 = (R(0,2), R(1,2), R(2,2))
    if (!rarecorrector) {
        beta1 = (c * del0 - del1) / (c - a);
        beta2 = a * c * del0 - (a + c) * del1 + del2;
        beta3 = (del1 - a * del0) / (c - a);
        R12 = 0.0; R22 = 1.0;
    } else {
        beta1 = (bb * c * del0 - (bb + c) * del1 + del2) / (sq(a) - a * bb - a * c + bb * c);
        beta2 = (-a * c * del0 + (a + c) * del1 - del2) / (a * bb - a * c - sq(bb) + bb * c);
        beta3 = (a * bb * del0 - (a + bb) * del1 + del2) / (a * bb - a * c - bb * c + sq(c));
        R12 = sw2; R22 = sq(sw2);
    }
    Waves w;
    w.s1 = sw1; w.s2 = sw2; w.s5 = sw3;
    double fw11 = beta1 * sw1, fw21 = beta1 * sq(sw1);
    double fw12 = beta2 * R12, fw22 = beta2 * R22;
    double fw13 = beta3 * sw3, fw23 = beta3 * sq(sw3);

    double fw41 = fw11 * mL;
    double fw43 = fw13 * mR;
    double fw42 = hmR * uR - hmL * uL - fw41 - fw43;
    double fw31 = fw11 * vL;
    double fw33 = fw13 * vR;
    double fw32 = hvR * uR - hvL * uL - fw31 - fw33;
    double fw51 = fw11 * gammaL * rhoL * grav * 1.0;
    double fw53 = fw13 * gammaR * rhoR * grav * 1.0;
    double fw52;

    double fw61 = 0.0, fw63 = 0.0, fw62 = 0.0;
    if (cw) {
        const double alpha_seg = 1.0 - P.beta_seg;
        const double seg_L = chiL * hL * uL * (1.0 + (1.0 - alpha_seg) * (1.0 - chiL));
        const double seg_R = chiR * hR * uR * (1.0 + (1.0 - alpha_seg) * (1.0 - chiR));
        fw61 = fw11 * chiL * (1.0 + (1.0 - alpha_seg) * (1.0 - chiL));
        fw63 = fw13 * chiR * (1.0 + (1.0 - alpha_seg) * (1.0 - chiR));
        fw62 = seg_R - seg_L - fw61 - fw63;
    }
    double hustar_interface = huL + fw11;
    if (!is_static) {
        double u_interface = hustar_interface / hstarHLL;
        del4 = -gamma * rho * gz * u_interface * (hR - hL) + grg * del1 + u_interface * (pR - pL);
    }
    fw52 = del4 - fw53 - fw51;
    if (cw) {
        if (hustar_interface <= 0.0) fw61 = fw61 + fw62;
        else fw63 = fw63 + fw62;
    }
    if (hustar_interface <= 0.0) {
        if (br) *br |= BR_REVERT_L;
        fw31 = fw31 + fw32;
        fw41 = fw41 + fw42;
        fw51 = fw51 + fw52;
    } else {
        fw33 = fw33 + fw32;
        fw43 = fw43 + fw42;
        fw53 = fw53 + fw52;
    }
    // wall masking of the three solver waves
    w.s1 = w.s1 * wall1; w.s2 = w.s2 * wall2; w.s5 = w.s5 * wall3;
    w.w1h = fw11 * wall1; w.w1n = fw21 * wall1; w.w1t = fw31 * wall1; w.w1m = fw41 * wall1; w.w1p = fw51 * wall1;
    w.w2h = fw12 * wall2; w.w2n = fw22 * wall2;
    w.w5h = fw13 * wall3; w.w5n = fw23 * wall3; w.w5t = fw33 * wall3; w.w5m = fw43 * wall3; w.w5p = fw53 * wall3;
    if (cw) {
        cw->w1c = fw61 * wall1;
        cw->w5c = fw63 * wall3;
    }
    return w;
}

// ---------------------------------------------------------------------------
// rpt2 for one fluctuation. cell = the imp cell (A2 state: h, hn, ht, hm),
// b = its bed, topo1/topo3 = bed of the neighbours below/above in the
// transverse direction. asdq in (h, n, t, hm, p). Outputs bm/bp in the same
// order. Returns false when the split is skipped. With bmp6 (the
// full-state step) the species component is split too: bmp6[0], bmp6[1]
// receive its B-, B+ parts, with r(6, 1) = r(6, 3) = chi = hchi / h
// (rpt2_dclaw.f:104,208-215,244-258); b is then the bed less the bed change.
// The cell part of rpt2_split: the primitives and eigenvalues of the
// Jacobian of the cell the fluctuation splits in. ok is false where the
// reference returns zero waves (a dry cell, or eta below both transverse
// neighbours' beds). One cell part serves every fluctuation split there.
struct Rpt2Cell {
    bool ok;
    double u, m, chi, eta, r5, s1, s2, s3, s31;
};

DC_HD Rpt2Cell rpt2_cell(const dclaw_params& P, double h, double hn, double ht, double hm, double b, double topo1,
                         double topo3, double hchi = 0.0, bool with_chi = false) {
    Rpt2Cell c;
    c.ok = false;
    c.u = c.m = c.chi = c.eta = c.r5 = c.s1 = c.s2 = c.s3 = c.s31 = 0.0;
    if (h <= P.dry_tolerance) return c;
    const double g = P.grav;
    c.u = hn / h;
    double v = ht / h;
    c.m = hm / h;
    if (with_chi) c.chi = hchi / h;
    c.eta = h + b;
    double rho = c.m * P.rho_s + (1.0 - c.m) * P.rho_f;
    double gamma;
    if (P.src2method == -1) gamma = P.rho_f / rho;
    else gamma = 0.25 * (P.rho_f + 3.0 * rho) / rho;
    if (c.eta < fmin2(topo1, topo3)) return c;
    c.ok = true;
    double sgh = sqrt(g * h);
    c.s1 = v - sgh;
    c.s2 = v;
    c.s3 = v + sgh;
    c.s31 = c.s3 - c.s1;
    c.r5 = gamma * rho * g;
    return c;
}

// The fluctuation part of rpt2_split: asdq split into bm/bp with the cell
// part c (bmp6: the species row, with_chi in rpt2_cell).
DC_HD bool rpt2_apply(const Rpt2Cell& c, double topo1, double topo3, const double asdq[5], double bm[5],
                      double bp[5], double* bmp6 = nullptr) {
    for (int k = 0; k < 5; ++k) { bm[k] = 0.0; bp[k] = 0.0; }
    if (bmp6) { bmp6[0] = 0.0; bmp6[1] = 0.0; }
    if (!c.ok) return false;
    const double u = c.u, m = c.m, chi = c.chi, eta = c.eta, r5 = c.r5, s1 = c.s1, s2 = c.s2, s3 = c.s3;
    double delf1 = asdq[0], delf2 = asdq[1], delf3 = asdq[2];
    double beta1 = (s3 * delf1 - delf3) / c.s31;
    double beta2 = -u * delf1 + delf2;
    double beta3 = (delf3 - s1 * delf1) / c.s31;
    // wave 1: r = (1, u, s1, m, r5, chi)
    {
        double sb = 1.0 * s1 * beta1;
        if ((s1 < 0.0) && (eta >= topo1)) {
            bm[0] = bm[0] + sb * 1.0; bm[1] = bm[1] + sb * u; bm[2] = bm[2] + sb * s1;
            bm[3] = bm[3] + sb * m; bm[4] = bm[4] + sb * r5;
            if (bmp6) bmp6[0] = bmp6[0] + sb * chi;
        } else if ((s1 > 0.0) && (eta >= topo3)) {
            bp[0] = bp[0] + sb * 1.0; bp[1] = bp[1] + sb * u; bp[2] = bp[2] + sb * s1;
            bp[3] = bp[3] + sb * m; bp[4] = bp[4] + sb * r5;
            if (bmp6) bmp6[1] = bmp6[1] + sb * chi;
        }
    }
    // wave 2: r = (0, 1, 0, 0, 0): only the normal-momentum component is nonzero
    {
        double sb = 1.0 * s2 * beta2;
        if ((s2 < 0.0) && (eta >= topo1)) bm[1] = bm[1] + sb * 1.0;
        else if ((s2 > 0.0) && (eta >= topo3)) bp[1] = bp[1] + sb * 1.0;
    }
    // wave 3: r = (1, u, s3, m, r5, chi)
    {
        double sb = 1.0 * s3 * beta3;
        if ((s3 < 0.0) && (eta >= topo1)) {
            bm[0] = bm[0] + sb * 1.0; bm[1] = bm[1] + sb * u; bm[2] = bm[2] + sb * s3;
            bm[3] = bm[3] + sb * m; bm[4] = bm[4] + sb * r5;
            if (bmp6) bmp6[0] = bmp6[0] + sb * chi;
        } else if ((s3 > 0.0) && (eta >= topo3)) {
            bp[0] = bp[0] + sb * 1.0; bp[1] = bp[1] + sb * u; bp[2] = bp[2] + sb * s3;
            bp[3] = bp[3] + sb * m; bp[4] = bp[4] + sb * r5;
            if (bmp6) bmp6[1] = bmp6[1] + sb * chi;
        }
    }
    return true;
}

DC_BIG bool rpt2_split(const dclaw_params& P, double h, double hn, double ht, double hm,
                                          double b, double topo1, double topo3, const double asdq[5],
                                          double bm[5], double bp[5], double hchi = 0.0,
                                          double* bmp6 = nullptr) {
    const Rpt2Cell c = rpt2_cell(P, h, hn, ht, hm, b, topo1, topo3, hchi, bmp6 != nullptr);
    return rpt2_apply(c, topo1, topo3, asdq, bm, bp, bmp6);
}

// ---------------------------------------------------------------------------
// mp_update_relax_Dclaw4 for src2method 0/1
DC_HD void mp_update_relax(const dclaw_params& P, double phi, double dt, double& h,
                                                double& u, double& v, double& m, double& p, double rhoh,
                                                double gz) {
    SetVars sv = setvars<true>(P, phi, h, u, v, m, p, gz);
    double hu = h * u, hv = h * v, hm = h * m;
    double vnorm = sqrt(sq(hu) + sq(hv)) / h;
    p = p - dt * 3.0 * vnorm * sv.tanpsi * sv.alphainv / h;
    qfix(P, h, hu, hv, hm, p, u, v, m, gz);
    double rho = P.rho_s * m + (1.0 - m) * P.rho_f;
    if (h <= P.dry_tolerance) rho = 0.0;
    double zeta = 3.0 * sv.alphainv / (h * 2.0) + (rho - P.rho_f) * P.rho_f * gz / (4.0 * rho);
    double krate = -zeta * 2.0 * sv.kperm / (h * fmax2(P.mu, 1.0e-16));
    double p_eq = P.rho_f * h * gz;
    p = p_eq + (p - p_eq) * em::d_exp(krate * dt);
    double p_exc = p - P.rho_f * gz * h;
    qfix_cmass(P, h, m, p, rho, p_exc, hu, hv, hm, u, v, rhoh, gz);
    double D = -2.0 * (sv.kperm / (P.mu * h)) * p_exc;
    krate = D * (rho - P.rho_f) / rhoh;
    hm = hm * em::d_exp(-dt * D * P.rho_f / (rhoh));
    if (P.src2method == 0) {
        h = h + h * krate * dt;
        double e = em::d_exp(dt * krate);
        hu = hu * e;
        hv = hv * e;
        qfix(P, h, hu, hv, hm, p, u, v, m, gz);
    } else {
        h = (rhoh - hm * (P.rho_s - P.rho_f)) / P.rho_f;
        hu = h * u;
        hv = h * v;
        qfix(P, h, hu, hv, hm, p, u, v, m, gz);
    }
}

// mp_update_FE_4quad (mp_update.f90:38-707), src2method 2: one substep of
// the quadrant-wise explicit integration of (m, p_exc) on the rho h = const
// manifold; returns the time the substep covered. Where the reference reads
// dtm unassigned (branch vnorm == 0 or m == m_eq, mp_update.f90:225-249),
// dtm = dtr, the whole remaining time.
DC_BIG double mp_update_fe4quad(const dclaw_params& P, double phi, double dtr, double& h, double u, double v,
                                double& m, double& p, double rhoh, double gz, double chi = 0.0) {
    const double rs = P.rho_s, rf = P.rho_f, mu = P.mu;
    const double vnorm = sqrt(sq(u) + sq(v));
    SetVars sv = setvars<true>(P, phi, h, u, v, m, p, gz, chi);
    const double h0 = h, m_0 = m;
    const double rho0 = m_0 * (rs - rf) + rf;
    const double p_eq0 = rf * gz * h0;
    const double p_exc0 = p - p_eq0;
    const double km0 = ((2.0 * sv.kperm * (rho0 * rho0)) / (mu * (rhoh * rhoh)));
    const double c_d0 = -3.0 * vnorm * (sv.alphainv * rho0 / (rhoh)) * sv.tanpsi;
    double kp0 = (sv.kperm / (h0 * mu)) * (3.0 * sv.alphainv * rho0 / rhoh - 1.5 * rf * gz * h0 * (rho0 - rf) / rhoh);
    kp0 = fmax2(kp0, 1.0e-3);
    double rho, p_exc, hu, hv, hm;
    if (m == 0.0) {
        p_exc = p_exc0 * em::d_exp(-kp0 * dtr);
        qfix_cmass(P, h, m, p, rho, p_exc, hu, hv, hm, u, v, rhoh, gz);
        return dtr;
    }
    const double m_eq = sv.m_eq;
    if ((fabs(p_exc0 / (rf * gz * h0)) < 1.0e-12) && (fabs(m - m_eq) < 1.0e-12)) return dtr;
    if ((vnorm == 0.0) || (m == m_eq)) {
        const double dtm = dtr;
        p_exc = p_exc0 * em::d_exp(-kp0 * dtm);
        if (!((m == m_eq) && (m < 0.3))) m = m_0 * em::d_exp(km0 * p_exc * dtm);
        qfix_cmass(P, h, m, p, rho, p_exc, hu, hv, hm, u, v, rhoh, gz);
        return dtm;
    }
    // critical point (m_c, p_eq_c) by fixed-point iteration
    double m_c = P.m_crit;
    double rho_c = m_c * (rs - rf) + rf;
    double h_c = rhoh / rho_c;
    double p_eq_c = rf * gz * h_c;
    const double shear = 2.0 * vnorm / h0;
    int iter;
    double normc = 0.0;
    for (iter = 1; iter <= 100; ++iter) {
        const double m_c0 = m_c, p_eq_c0 = p_eq_c;
        rho_c = m_c * (rs - rf) + rf;
        h_c = rhoh / rho_c;
        p_eq_c = rf * gz * h_c;
        const double sig_c = fmax2(rhoh * gz - p_eq_c, 0.0);
        const double Nd = rs * sq(shear * P.delta) + sig_c;
        const double Nn = mu * shear;
        m_c = P.m_crit * (sqrt(Nd) / (sqrt(Nd) + sqrt(Nn)));
        normc = sq(1.0e2 * (m_c - m_c0)) + sq(1.0e-3 * (p_eq_c - p_eq_c0));
        if (normc < 1.0e-16) break;
    }
    if ((iter >= 100) && (normc > 1.0)) m_c = P.m_crit;
    rho_c = m_c * (rs - rf) + rf;
    h_c = rhoh / rho_c;
    p_eq_c = rf * gz * h_c;
    int quad0 = 0;
    if ((m < m_c) && (p >= p_eq_c)) quad0 = 1;
    else if ((m >= m_c) && (p > p_eq_c)) quad0 = 2;
    else if ((m > m_c) && (p <= p_eq_c)) quad0 = 3;
    else if ((m <= m_c) && (p < p_eq_c)) quad0 = 4;
    if (quad0 == 0) return 0.0;
    // p_exc(t) = (1/kp0) ((kp0 p_exc0 - c_d0) e^{-kp0 t} + c_d0)
    auto pexc_at = [&](double t) { return (1.0 / kp0) * ((kp0 * p_exc0 - c_d0) * em::d_exp(-kp0 * t) + c_d0); };
    double dtm, dtp, dts, p_exc_ave;
    if (quad0 == 1) {
        if (p_exc0 < -1.0e-3 * rhoh * gz) {  // region 1A
            if (c_d0 > 0.0) dtp = -(1.0 / kp0) * em::d_log(c_d0 / (c_d0 - kp0 * p_exc0));
            else dtp = dtr;
            dtm = em::d_log(0.98) / (kp0 * p_exc0);
            dts = fmin2(fmin2(dtr, dtp), dtm);
            dts = fmax2(dts, 0.0);
            p_exc = pexc_at(dts);
            m = m_0 * em::d_exp(dts * km0 * p_exc);
        } else if ((-kp0 * p_exc0 + c_d0) > 0.0) {  // region 1B
            if ((c_d0 / kp0) > (rhoh * gz - p_eq_c))
                dtp = fmin2(dtr, -(1.0 / kp0) * em::d_log((-kp0 * rhoh * gz + kp0 * p_eq_c + c_d0) / (-kp0 * p_exc0 + c_d0)));
            else
                dtp = dtr;
            p_exc = pexc_at(dtp);
            p_exc_ave = 0.5 * (p_exc + p_exc0);
            if (p_exc_ave <= 0.0) dtm = dtr;
            else if ((km0 * p_exc_ave * m_0) < 1.0e-99) dtm = dtp;
            else dtm = fmin2(dtp, (m_eq - m_0) / (km0 * p_exc_ave * m_0));
            m = m_0 + km0 * m_0 * p_exc_ave * dtm;
            dts = dtm;
        } else if (c_d0 > 0.0) {  // region 1C, left of m_eq
            dtp = dtr;
            if ((km0 * p_exc0 * m_0) > 1.0e-99) dtm = (m_c - m_0) / (km0 * p_exc0 * m_0);
            else dtm = dtp;
            dts = fmin2(dtm, dtp);
            dts = fmax2(dts, 0.0);
            m = m_0 + km0 * m_0 * p_exc0 * dts;
            p_exc = pexc_at(dts);
        } else {  // region 1C, right of m_eq
            dts = dtr;
            dtp = dtr;
            if ((km0 * p_exc0 * m_0) > 1.0e-99) dts = fmin2(dtr, (m_c - m_0) / (km0 * p_exc0 * m_0));
            if ((kp0 * p_exc0 - c_d0) != 0.0) {
                if ((-kp0 * p_eq0 - c_d0) / (kp0 * p_exc0 - c_d0) > 1.0e-99)
                    dtp = fmin2(dtr, -(1.0 / kp0) * em::d_log((c_d0) / (c_d0 - kp0 * p_exc0)));
            }
            dts = fmin2(dts, dtp);
            dts = fmax2(dts, 0.0);
            m = m_0 + km0 * m_0 * p_exc0 * dts;
            p_exc = pexc_at(dts);
        }
    } else if (quad0 == 2) {
        dtp = dtr;
        if ((c_d0 - kp0 * (p_eq_c - p_eq0)) / (c_d0 - kp0 * p_exc0) > 1.0e-99)
            dtp = fmin2(dtr, -(1.0 / kp0) * em::d_log((c_d0 - kp0 * (p_eq_c - p_eq0)) / (c_d0 - kp0 * p_exc0)));
        dtm = dtp;
        if (km0 * p_exc0 * m_0 > 1.0e-99) dtm = fmin2(dtp, (fmin2(1.0 - m_0, 0.02) / (km0 * p_exc0 * m_0)));
        dts = fmin2(dtp, dtm);
        p_exc = pexc_at(dts);
        m = m_0 + km0 * m_0 * p_exc * dts;
    } else if (quad0 == 3) {
        if (p_exc0 > 1.0e-3 * rhoh * gz) {  // region 3A
            dtp = dtr;
            if ((c_d0 / (-kp0 * p_exc0 + c_d0)) > 1.0e-99)
                dtp = fmin2(dtr, -(1.0 / kp0) * em::d_log(c_d0 / (c_d0 - kp0 * p_exc0)));
            dtm = dtp;
            if ((km0 * p_exc0 * m_0) > 1.0e-99) dtm = fmin2(dtp, (fmin2(1.0 - m_0, 0.02)) / (km0 * p_exc0 * m_0));
            p_exc = pexc_at(dtp);
            m = m_0 + km0 * m_0 * 0.5 * (p_exc0 + p_exc) * dtm;
            dts = dtp;
        } else if ((-kp0 * p_exc0 + c_d0) < 0.0) {  // region 3B
            dtp = dtr;
            if (c_d0 / kp0 < -p_eq0) {
                if (((c_d0 + kp0 * p_eq0) / (-kp0 * p_exc0 + c_d0)) > 1.0e-99)
                    dtp = fmin2(dtr, -(1.0 / kp0) * em::d_log((c_d0 + kp0 * p_eq0) / (-kp0 * p_exc0 + c_d0)));
            }
            p_exc = pexc_at(dtp);
            p_exc_ave = 0.5 * (p_exc + p_exc0);
            if (p_exc_ave > 0.0) {
                dtm = fmin2(dtr, (0.02) / (km0 * p_exc_ave * m_0));
            } else {
                const double m_lower = m_eq + fmax2(0.0, (1.0 / 3.0) * kp0 * h0 * (-p_exc_ave) / (vnorm * sv.alphainv));
                dtm = fmin2(dtr, (m_lower - m_0) / (km0 * p_exc_ave * m_0));
            }
            m = m_0 + km0 * m_0 * p_exc_ave * dtm;
            dts = dtm;
        } else if (c_d0 < 0.0) {  // region 3C, between the p-nullcline and m_eq
            dtp = dtr;
            dtm = dtr;
            if (-(km0 * p_exc0 * m_0) > 1.0e-99) dtm = (m_c - m_0) / (km0 * p_exc0 * m_0);
            dts = fmin2(dtp, dtm);
            dts = fmax2(dts, 0.0);
            p_exc = pexc_at(dts);
            m = m_0 + km0 * m_0 * p_exc0 * dts;
        } else {  // region 3C, left of m_eq
            dtm = dtr;
            dtp = dtr;
            if ((km0 * p_exc0 * m_0) > 1.0e-99) dtm = (m_c - m_0) / (km0 * p_exc0 * m_0);
            if ((-c_d0 / (kp0 * p_exc0 - c_d0)) > 1.0e-99) dtp = -(1.0 / kp0) * em::d_log(c_d0 / (c_d0 - kp0 * p_exc0));
            dts = fmin2(dtp, dtm);
            dts = fmax2(dts, 0.0);
            p_exc = pexc_at(dts);
            m = m_0 + km0 * m_0 * p_exc0 * dts;
        }
    } else {  // quad0 == 4
        dtp = dtr;
        if ((c_d0 - kp0 * (p_eq_c - p_eq0)) / (c_d0 - kp0 * p_exc0) > 1.0e-99)
            dtp = fmin2(dtr, -(1.0 / kp0) * em::d_log((c_d0 - kp0 * (p_eq_c - p_eq0)) / (c_d0 - kp0 * p_exc0)));
        dtm = em::d_log(0.98) / (kp0 * p_exc0);
        dts = fmin2(dtr, fmin2(dtp, dtm));
        p_exc = pexc_at(dts);
        m = m_0 * em::d_exp(dts * km0 * 0.5 * (p_exc0 + p_exc));
        dts = dtp;  // the reference reports dtp as the time covered
    }
    qfix_cmass(P, h, m, p, rho, p_exc, hu, hv, hm, u, v, rhoh, gz);
    return dts;
}

// src2 on one interior cell (in place on the 5 conserved fields)
DC_BIG void src2_cell(const dclaw_params& P, double phi, double dt, double& qh, double& qhu,
                                          double& qhv, double& qhm, double& qp) {
    double h = qh;
    if (h <= P.dry_tolerance) {
        qh = 0.0; qhu = 0.0; qhv = 0.0; qhm = 0.0; qp = 0.0;
        return;
    }
    double hu = qhu, hv = qhv, hm = qhm, p = qp;
    double rhoh = hm * P.rho_s + (h - hm) * P.rho_f;
    if (hm < 0.0) return;
    const double gz = P.grav;
    const double gx = 0.0;
    double u, v, m;
    qfix(P, h, hu, hv, hm, p, u, v, m, gz);
    SetVars sv = setvars<false>(P, phi, h, u, v, m, p, gz);
    double hvnorm0 = sqrt(sq(hu) + sq(hv));
    double vnorm = hvnorm0 / h;
    if (hvnorm0 > 0.0) {
        vnorm = fmax2(0.0, vnorm - dt * sv.tau / rhoh);
        vnorm = vnorm * em::d_exp(-(1.0 - m) * 2.0 * P.mu * dt / (h * rhoh));
        double hvnorm = h * vnorm;
        hu = hvnorm * hu / hvnorm0 + gx * h * dt;
        hv = hvnorm * hv / hvnorm0;
        u = hu / h;
        v = hv / h;
    }
    if (P.src2method == -1) {
        hu = h * u; hv = h * v; hm = h * m;
    } else if (P.src2method == 2) {
        // src2.f90:206-229: substeps until dt is covered, at most 100
        double dtremaining = dt;
        int itercount = 0;
        while (dtremaining > 1.0e-99) {
            const double dtk = mp_update_fe4quad(P, phi, dtremaining, h, u, v, m, p, rhoh, gz);
            dtremaining = dtremaining - dtk;
            itercount = itercount + 1;
            if (dtk == 0.0) break;
            if (h < P.dry_tolerance) break;
            if (itercount >= 100) break;
        }
        hu = h * u; hv = h * v; hm = h * m;
        qfix(P, h, hu, hv, hm, p, u, v, m, gz);
    } else {
        mp_update_relax(P, phi, dt, h, u, v, m, p, rhoh, gz);
        hu = h * u; hv = h * v; hm = h * m;
    }
    if (h <= P.dry_tolerance) {
        qh = 0.0; qhu = 0.0; qhv = 0.0; qhm = 0.0; qp = 0.0;
        return;
    }
    if (P.friction_forcing && P.manning_coefficient > 0.0) {
        if (h <= P.friction_depth) {
            double cm = P.manning_coefficient;
            if (P.dd_manning)
                cm = P.manning_max + (P.manning_coefficient - P.manning_max) * 0.5 * (1.0 + em::d_tanh(300.0 * (h - 0.05)));
            double beta = 1.0;
            double gamma = beta * sqrt(sq(hu) + sq(hv)) * (gz * sq(cm)) / (em::d_pow_7_3(h));
            double dgamma = 1.0 + dt * gamma;
            hu = hu / dgamma;
            hv = hv / dgamma;
            qfix(P, h, hu, hv, hm, p, u, v, m, gz);
        }
    }
    qh = h; qhu = hu; qhv = hv; qhm = hm; qp = p;
}

}  // namespace dclaw
