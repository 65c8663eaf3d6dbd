// stages.cuh -- the per-cell / per-interface stages of one uniform-patch step.
//
// The step of the reference (GeoClaw stepgrid driving src/2d/dig/b4step2.f90,
// flux2fw.f via step2, src/2d/dig/src2.f90) is split into five data-parallel
// stages. Each stage is a DC_HD function of one work item so that the CUDA
// kernels (kernels.cu) and a host emulation used only by the CPU tests run
// identical arithmetic.
//
//   A  stage_b4        cell   ghost fill (bc2amr) + qfix + speed limit
//   B  stage_taudir    cell   calc_taudir (fsphi, taudir_x, taudir_y)
//   C  stage_riemann   iface  the two rpn2 qfix passes + augmented solver
//   D  stage_flux      iface  wave limiter, 2nd-order correction, A-/+dq,
//                             transverse splits (rpt2 imp=1,2)
//   E  stage_finalize  cell   flux accumulation in step2's order, the
//                             flux-differencing update, src2
//
// The reference mutates the 1-D slice copy inside rpn2: at interface i the
// right cell has been through qfix once and the left cell twice (the first
// cell of a slice only once). qfix is not bitwise idempotent
// (hm = h * (hm/h)), so stage C applies it exactly that many times.
#pragma once
#include "physics.cuh"

namespace dclaw {

constexpr int NW = 15;   // stored doubles per interface solve
constexpr int NF = 30;   // stored doubles per interface flux: faddm[5] faddp[5] U1m U1p U2m U2p
enum { W_S1 = 0, W_S2, W_S5, W_1H, W_1N, W_1T, W_1M, W_1P, W_2H, W_2N, W_5H, W_5N, W_5T, W_5M, W_5P };

struct Geom {
    int mx, my;
    int PX, PY;      // padded extents mx+4, my+4
    double dx, dy;
};

// Workspace views. Padded planes are PX*PY; x-interface planes are
// (my+2) rows x (mx+3) interfaces (rows 0..my+1, interfaces 0..mx+2);
// y-interface planes are (my+3) interfaces x (mx+2) columns.
struct Work {
    double* qB;   // 5 padded planes: state after b4step2
    double* bP;   // padded bed
    double* td;   // 3 padded planes: fsphi, taudir_x, taudir_y
    double* wx;   // NW x-interface planes
    double* wy;   // NW y-interface planes
    double* fx;   // NF x-interface planes
    double* fy;   // NF y-interface planes
    size_t npad, nxi, nyi;
};

DC_HD size_t pidx(const Geom& g, int i, int j) { return (size_t)(j + 1) * g.PX + (size_t)(i + 1); }
DC_HD size_t xidx(const Geom& g, int r, int i) { return (size_t)r * (g.mx + 3) + (size_t)i; }
DC_HD size_t yidx(const Geom& g, int k, int c) { return (size_t)k * (g.mx + 2) + (size_t)c; }

// ---------------------------------------------------------------------------
// Stage A. Cell (i, j), i in -1..mx+2, j in -1..my+2. q_in is the interior
// state (5 planes mx*my). Ghost cells come from the boundary conditions
// (bc2amr restated: wall = mirror with negated normal momentum, extrap =
// nearest interior copy; x sides first, then y sides incl. corners), the
// ghost bed is the nearest interior bed (setaux.f90:155-184).
// Returns true when the source cell holds a NaN.
DC_HD bool stage_b4(const dclaw_params& P, const Geom& g, const double* __restrict__ q_in,
                    const double* __restrict__ b_in, const Work& W, int i, int j) {
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
    const size_t plane = (size_t)mx * my;
    const size_t c = (size_t)(sj - 1) * mx + (size_t)(si - 1);
    double h = q_in[c], hu = q_in[plane + c], hv = q_in[2 * plane + c], hm = q_in[3 * plane + c],
           p = q_in[4 * plane + c];
    bool nan = (h != h) || (hu != hu) || (hv != hv) || (hm != hm) || (p != p);
    if (flip_u) hu = -hu;
    if (flip_v) hv = -hv;
    double u, v, m;
    qfix(P, h, hu, hv, hm, p, u, v, m, P.grav);
    // speed limit (b4step2.f90:74-100)
    if (h > 0.0) {
        double s = sqrt((sq(hu) + sq(hv))) / h;
        if (s > P.speed_limit) {
            double sratio = P.speed_limit / s;
            hu = hu * sratio;
            hv = hv * sratio;
        }
    }
    const size_t pi = pidx(g, i, j);
    W.qB[pi] = h;
    W.qB[W.npad + pi] = hu;
    W.qB[2 * W.npad + pi] = hv;
    W.qB[3 * W.npad + pi] = hm;
    W.qB[4 * W.npad + pi] = p;
    int bi = i < 1 ? 1 : (i > mx ? mx : i);
    int bj = j < 1 ? 1 : (j > my ? my : j);
    W.bP[pi] = b_in[(size_t)(bj - 1) * mx + (size_t)(bi - 1)];
    return nan;
}

// ---------------------------------------------------------------------------
// Stage B. calc_taudir on cell (i, j) of the padded patch. Cells of the outer
// ghost ring keep fsphi = taudir = 0 (setaux zeroes them, calc_taudir covers
// only 2-mbc..m+mbc-1).
// qB: the b4step2 state's padded planes (h, hu, hv, hm, pb first), td the
// three output planes, bed(pi) the bed of padded cell pi (the bed less the
// bed change on the full state: digclaw_module.f90:555-613).
template <typename Bed>
DC_HD void taudir_cell(const dclaw_params& P, const Geom& g, const double* __restrict__ qB, size_t npad,
                       double* td, Bed bed, int i, int j) {
    const size_t pi = pidx(g, i, j);
    double* fs = td;
    double* tx = td + npad;
    double* ty = td + 2 * npad;
    if (i < 0 || j < 0 || i > g.mx + 1 || j > g.my + 1) {
        fs[pi] = 0.0; tx[pi] = 0.0; ty[pi] = 0.0;
        return;
    }
    const double dry = P.dry_tolerance;
    const double gz = P.grav;
    const double* qh = qB;
    // the qB state is already admissible: qfix leaves h of every cell as is
    double h = qh[pi];
    double hu = qB[npad + pi], hv = qB[2 * npad + pi];
    double hm = qB[3 * npad + pi], p = qB[4 * npad + pi];
    const size_t pL = pidx(g, i - 1, j), pR = pidx(g, i + 1, j), pB = pidx(g, i, j - 1), pT = pidx(g, i, j + 1);
    double hL = qh[pL], hR = qh[pR], hB = qh[pB], hT = qh[pT];
    double b = bed(pi);
    double eta = h + b;
    double etaL = hL + bed(pL);
    if (hL < dry) etaL = fmin2(etaL, eta);
    double etaR = hR + bed(pR);
    if (hR < dry) etaR = fmin2(etaR, eta);
    double etaB = hB + bed(pB);
    if (hB < dry) etaB = fmin2(etaB, eta);
    double etaT = hT + bed(pT);
    if (hT < dry) etaT = fmin2(etaT, eta);
    if (h < dry) {
        eta = fmin2(etaL, eta);
        eta = fmin2(etaB, eta);
    }
    if ((h + hL + hB + hR + hT) < dry) {
        fs[pi] = 0.0; tx[pi] = 0.0; ty[pi] = 0.0;
        return;
    }
    double u, v, m;
    qfix(P, h, hu, hv, hm, p, u, v, m, gz);
    SetVars sv = setvars<false>(P, P.phi, h, u, v, m, p, gz);
    const double dx = g.dx, dy = g.dy;
    const double sint = 0.0;  // sin(theta), theta = 0
    double FxL = -gz * 0.5 * (h + hL) * (eta - etaL) / (dx) + gz * 0.5 * (h + hL) * sint;
    double FyL = -gz * 0.5 * (h + hB) * (eta - etaB) / (dy);
    double FxR = -gz * 0.5 * (h + hR) * (etaR - eta) / (dx) + gz * 0.5 * (h + hR) * sint;
    double FyR = -gz * 0.5 * (h + hT) * (etaT - eta) / (dy);
    double Fx, Fy;
    if (FxL * FxR > 0.0) Fx = fsign(fmin2(fabs(FxL), fabs(FxR)), FxL);
    else Fx = 0.0;
    if (FyL * FyR > 0.0) Fy = fsign(fmin2(fabs(FyL), fabs(FyR)), FyL);
    else Fy = 0.0;
    double hvnorm = sqrt(sq(hu) + sq(hv));
    double ofs, otx, oty;
    if (hvnorm > 0.0) {
        otx = -dx * hu / hvnorm;
        oty = -dy * hv / hvnorm;
        double dot = fmin2(fmax2(0.0, Fx * hu), fmax2(0.0, Fy * hv));
        if (dot > 0.0) {
            double Fproj = dot / hvnorm;
            ofs = fmin2(1.0, Fproj * sv.rho / fmax2(sv.tau, 1.0e-16));
        } else {
            ofs = 0.0;
        }
    } else {
        if ((sq(FxL) + sq(Fy)) > 0.0) otx = -dx * FxL / sqrt(sq(FxL) + sq(Fy));
        else otx = dx * 1.0;
        if ((sq(Fx) + sq(FyL)) > 0.0) oty = -dy * FyL / sqrt(sq(Fx) + sq(FyL));
        else oty = dy * 1.0;
        if ((sq(oty) + sq(otx)) > 0.0) ofs = 1.0;
        else ofs = 0.0;
    }
    fs[pi] = ofs; tx[pi] = otx; ty[pi] = oty;
}

DC_HD void stage_taudir(const dclaw_params& P, const Geom& g, const Work& W, int i, int j) {
    const double* bP = W.bP;
    taudir_cell(P, g, W.qB, W.npad, W.td, [bP](size_t q) { return bP[q]; }, i, j);
}

// ---------------------------------------------------------------------------
// Side state for the solver: qfix once (A1) or twice (A2) from the qB state.
// comp_n / comp_t: q component index (1 = hu, 2 = hv) of the normal and
// tangential momentum.
DC_HD Side load_side(const dclaw_params& P, const Work& W, size_t pi, int comp_n, int comp_t, bool twice,
                     int taudir_plane) {
    Side s;
    double h = W.qB[pi];
    s.b = W.bP[pi];
    s.fs = W.td[pi];
    s.taudir = W.td[(size_t)taudir_plane * W.npad + pi];
    if (h <= P.dry_tolerance) {
        s.h = 0.0; s.hn = 0.0; s.ht = 0.0; s.hm = 0.0; s.p = 0.0;
        s.un = 0.0; s.ut = 0.0; s.m = 0.0;
        s.rho_sv = 0.0; s.tau_sv = 0.0;
        return s;
    }
    double hn = W.qB[(size_t)comp_n * W.npad + pi];
    double ht = W.qB[(size_t)comp_t * W.npad + pi];
    double hm = W.qB[3 * W.npad + pi];
    double p = W.qB[4 * W.npad + pi];
    double m;
    qfix_mp(P, h, hm, p, m, P.grav);
    if (twice) qfix_mp(P, h, hm, p, m, P.grav);
    s.h = h; s.hn = hn; s.ht = ht; s.hm = hm; s.p = p; s.m = m;
    s.un = hn / h;
    s.ut = ht / h;
    SetVars sv = setvars<false>(P, P.phi, h, s.un, s.ut, m, p, P.grav);
    s.rho_sv = sv.rho;
    s.tau_sv = sv.tau;
    return s;
}

// Per-cell setvars records of the two rpn2 states (A1: qfix once, A2:
// twice) of a wet padded cell, SV_N planes per state (padded layout): tau and
// its partial derivatives in (h, u, v, m, p, phi, mu), u = hu/h, v = hv/h.
// setvars reads the velocity only through u^2 + v^2, so the record serves
// both sweep directions. Written by the adjoint's record stage.
constexpr int SV_N = 8;
constexpr int NSV = 2 * SV_N;
enum { SV_TAU = 0, SV_DH, SV_DU, SV_DV, SV_DM, SV_DP, SV_DPHI, SV_DMU };

// load_side with tau read from the record instead of recomputed (same bits)
DC_HD Side load_side_sv(const dclaw_params& P, const Work& W, const double* __restrict__ sv, size_t pi,
                        int comp_n, int comp_t, bool twice, int taudir_plane) {
    Side s;
    double h = W.qB[pi];
    s.b = W.bP[pi];
    s.fs = W.td[pi];
    s.taudir = W.td[(size_t)taudir_plane * W.npad + pi];
    if (h <= P.dry_tolerance) {
        s.h = 0.0; s.hn = 0.0; s.ht = 0.0; s.hm = 0.0; s.p = 0.0;
        s.un = 0.0; s.ut = 0.0; s.m = 0.0;
        s.rho_sv = 0.0; s.tau_sv = 0.0;
        return s;
    }
    double hn = W.qB[(size_t)comp_n * W.npad + pi];
    double ht = W.qB[(size_t)comp_t * W.npad + pi];
    double hm = W.qB[3 * W.npad + pi];
    double p = W.qB[4 * W.npad + pi];
    double m;
    qfix_mp(P, h, hm, p, m, P.grav);
    if (twice) qfix_mp(P, h, hm, p, m, P.grav);
    s.h = h; s.hn = hn; s.ht = ht; s.hm = hm; s.p = p; s.m = m;
    s.un = hn / h;
    s.ut = ht / h;
    s.rho_sv = m * (P.rho_s - P.rho_f) + P.rho_f;
    s.tau_sv = sv[(size_t)((twice ? SV_N : 0) + SV_TAU) * W.npad + pi];
    return s;
}

// Stage C. Interface `i` (0..n+2) of slice `r` (x: row 0..my+1; y: column
// 0..mx+1). Writes the compact waves; returns max |s| over the waves for the
// Courant number and ORs branch bits into *br (nullable). sv (nullable):
// setvars records to read tau from instead of recomputing it.
template <int DIR>
DC_HD double stage_riemann(const dclaw_params& P, const Geom& g, const Work& W, int r, int i, uint32_t* br,
                           const double* __restrict__ sv = nullptr) {
    size_t pL, pR, oi;
    double* wv;
    size_t nplane;
    if (DIR == 0) {
        pL = pidx(g, i - 1, r); pR = pidx(g, i, r);
        oi = xidx(g, r, i); wv = W.wx; nplane = W.nxi;
    } else {
        pL = pidx(g, r, i - 1); pR = pidx(g, r, i);
        oi = yidx(g, i, r); wv = W.wy; nplane = W.nyi;
    }
    const int cn = DIR == 0 ? 1 : 2, ct = DIR == 0 ? 2 : 1;
    Waves w;
    if (W.qB[pL] <= P.dry_tolerance && W.qB[pR] <= P.dry_tolerance) {
        zero_waves(w);
        if (br) *br |= BR_DRY;
    } else {
        Side R = sv ? load_side_sv(P, W, sv, pR, cn, ct, false, 1 + DIR) : load_side(P, W, pR, cn, ct, false, 1 + DIR);
        Side L = sv ? load_side_sv(P, W, sv, pL, cn, ct, i - 1 >= 0, 1 + DIR)
                    : load_side(P, W, pL, cn, ct, i - 1 >= 0, 1 + DIR);
        w = riemann_solve(P, L, R, br);
    }
    const double vals[NW] = {w.s1, w.s2, w.s5, w.w1h, w.w1n, w.w1t, w.w1m, w.w1p,
                             w.w2h, w.w2n, w.w5h, w.w5n, w.w5t, w.w5m, w.w5p};
    for (int k = 0; k < NW; ++k) wv[(size_t)k * nplane + oi] = vals[k];
    return fmax2(fmax2(fabs(w.s1), fabs(w.s2)), fabs(w.s5));
}

// ---------------------------------------------------------------------------
// wave limiter for one family at interface i (Clawpack inlinelimiter
// restated, LeVeque 2002 sec. 6.9/6.12); W* in q-component order.
DC_HD double limiter_phi(int mth, double r, uint32_t& code) {
    double wl;
    switch (mth) {
        case 1: wl = fmax2(0.0, fmin2(1.0, r)); code = wl == 0.0 ? 1u : 2u; break;
        case 2: wl = fmax2(fmax2(0.0, fmin2(1.0, 2.0 * r)), fmin2(2.0, r)); code = wl == 0.0 ? 1u : 2u; break;
        case 3: wl = (r + fabs(r)) / (1.0 + fabs(r)); code = wl == 0.0 ? 1u : 2u; break;
        case 4: {
            double c = (1.0 + r) / 2.0;
            wl = fmax2(0.0, fmin2(fmin2(c, 2.0), 2.0 * r));
            code = wl == 0.0 ? 1u : (wl == c ? 2u : (wl == 2.0 ? 3u : 4u));
            break;
        }
        default: wl = r; code = 2u; break;
    }
    return wl;
}

template <int N = 5>
DC_HD void limit_family(int mth, int mw, double s, const double* Wm, double* Wi, const double* Wp,
                        uint32_t* br) {
    double wnorm2 = 0.0, dotl = 0.0, dotr = 0.0;
    for (int m = 0; m < N; ++m) {
        wnorm2 = wnorm2 + sq(Wi[m]);
        dotl = dotl + Wm[m] * Wi[m];
        dotr = dotr + Wi[m] * Wp[m];
    }
    if (wnorm2 == 0.0) return;
    double r;
    if (s > 0.0) {
        r = dotl / wnorm2;
        if (br) *br |= br_up(mw);
    } else {
        r = dotr / wnorm2;
    }
    uint32_t code;
    double wl = limiter_phi(mth, r, code);
    if (br) *br |= br_lim(mw, code);
    for (int m = 0; m < N; ++m) Wi[m] = wl * Wi[m];
}

// expand the compact waves at one interface into q-ordered 5-vectors
template <int DIR>
DC_HD void expand_waves(const double* wv, size_t nplane, size_t oi, double s[3], double W1[5], double W2[5],
                        double W5[5]) {
    double v[NW];
    for (int k = 0; k < NW; ++k) v[k] = wv[(size_t)k * nplane + oi];
    s[0] = v[W_S1]; s[1] = v[W_S2]; s[2] = v[W_S5];
    const int cn = DIR == 0 ? 1 : 2, ct = DIR == 0 ? 2 : 1;
    W1[0] = v[W_1H]; W1[cn] = v[W_1N]; W1[ct] = v[W_1T]; W1[3] = v[W_1M]; W1[4] = v[W_1P];
    W2[0] = v[W_2H]; W2[cn] = v[W_2N]; W2[ct] = 0.0; W2[3] = 0.0; W2[4] = 0.0;
    W5[0] = v[W_5H]; W5[cn] = v[W_5N]; W5[ct] = v[W_5T]; W5[3] = v[W_5M]; W5[4] = v[W_5P];
}

// A2 state (qfix applied twice) of a cell, in (h, n, t, hm) order
DC_HD void load_a2(const dclaw_params& P, const Work& W, size_t pi, int cn, int ct, double& h, double& hn,
                   double& ht, double& hm) {
    h = W.qB[pi];
    if (h <= P.dry_tolerance) { h = 0.0; hn = 0.0; ht = 0.0; hm = 0.0; return; }
    hn = W.qB[(size_t)cn * W.npad + pi];
    ht = W.qB[(size_t)ct * W.npad + pi];
    hm = W.qB[3 * W.npad + pi];
    double p = W.qB[4 * W.npad + pi], m;
    qfix_mp(P, h, hm, p, m, P.grav);
    qfix_mp(P, h, hm, p, m, P.grav);
}

// Stage D. Interface i (1..n+1) of slice r. dtdx = dt/dx (x) or dt/dy (y).
template <int DIR>
DC_HD void stage_flux(const dclaw_params& P, const Geom& g, const Work& W, int r, int i, double dtdx,
                      uint32_t* br) {
    const double* wv = DIR == 0 ? W.wx : W.wy;
    double* fo = DIR == 0 ? W.fx : W.fy;
    const size_t nplane = DIR == 0 ? W.nxi : W.nyi;
    auto oidx = [&](int ii) -> size_t { return DIR == 0 ? xidx(g, r, ii) : yidx(g, ii, r); };
    auto cidx = [&](int ii) -> size_t { return DIR == 0 ? pidx(g, ii, r) : pidx(g, r, ii); };
    const int cn = DIR == 0 ? 1 : 2, ct = DIR == 0 ? 2 : 1;
    const size_t oi = oidx(i);

    double s[3], W1[5], W2[5], W5[5];
    expand_waves<DIR>(wv, nplane, oi, s, W1, W2, W5);
    // fluctuations from the unlimited waves, family order 1..5
    double amdq[5], apdq[5];
    for (int m = 0; m < 5; ++m) {
        double am = 0.0, ap = 0.0;
        if (s[0] < 0.0) am = am + W1[m]; else if (s[0] > 0.0) ap = ap + W1[m];
        if (s[1] < 0.0) am = am + W2[m]; else if (s[1] > 0.0) ap = ap + W2[m];
        if (s[2] < 0.0) am = am + W5[m]; else if (s[2] > 0.0) ap = ap + W5[m];
        amdq[m] = am;
        apdq[m] = ap;
    }
    double faddm[5], faddp[5], cqxx[5];
    for (int m = 0; m < 5; ++m) {
        faddm[m] = 0.0 + amdq[m];
        faddp[m] = 0.0 - apdq[m];
        cqxx[m] = 0.0;
    }
    if (P.order != 1) {
        if (P.limiter != 0) {
            double sm[3], Wm1[5], Wm2[5], Wm5[5], sp[3], Wp1[5], Wp2[5], Wp5[5];
            expand_waves<DIR>(wv, nplane, oidx(i - 1), sm, Wm1, Wm2, Wm5);
            expand_waves<DIR>(wv, nplane, oidx(i + 1), sp, Wp1, Wp2, Wp5);
            limit_family(P.limiter, 1, s[0], Wm1, W1, Wp1, br);
            limit_family(P.limiter, 2, s[1], Wm2, W2, Wp2, br);
            limit_family(P.limiter, 5, s[2], Wm5, W5, Wp5, br);
        }
        double hl2 = W.qB[cidx(i - 2)], hl = W.qB[cidx(i - 1)], hr = W.qB[cidx(i)], hr2 = W.qB[cidx(i + 1)];
        bool wet4 = hl * hr * hl2 * hr2 > 0.0;
        if (wet4) {
            if (br) *br |= BR_WET4;
            const double c1 = fsign(1.0, s[0]) * (1.0 - fabs(s[0]) * dtdx);
            const double c2 = fsign(1.0, s[1]) * (1.0 - fabs(s[1]) * dtdx);
            const double c5 = fsign(1.0, s[2]) * (1.0 - fabs(s[2]) * dtdx);
            for (int m = 0; m < 5; ++m) {
                double cq = 0.0;
                cq = cq + c1 * W1[m];
                cq = cq + c2 * W2[m];
                cq = cq + c5 * W5[m];
                cqxx[m] = cq;
            }
        }
        for (int m = 0; m < 5; ++m) {
            faddm[m] = faddm[m] + 0.5 * cqxx[m];
            faddp[m] = faddp[m] + 0.5 * cqxx[m];
        }
    }
    double U1m[5], U1p[5], U2m[5], U2p[5];
    for (int m = 0; m < 5; ++m) { U1m[m] = 0.0; U1p[m] = 0.0; U2m[m] = 0.0; U2p[m] = 0.0; }
    if (P.transverse_waves != 0) {
        if (P.order > 1 && P.transverse_waves == 2) {
            for (int m = 0; m < 5; ++m) {
                amdq[m] = amdq[m] + cqxx[m];
                apdq[m] = apdq[m] - cqxx[m];
            }
        }
        const double half = 0.5 * dtdx;
        // imp = 1: left-going fluctuation split with the left cell (i-1)
        for (int imp = 1; imp <= 2; ++imp) {
            const int cc = imp == 1 ? i - 1 : i;
            const size_t pc = cidx(cc);
            double h, hn, ht, hm;
            load_a2(P, W, pc, cn, ct, h, hn, ht, hm);
            double topo1, topo3;
            if (DIR == 0) { topo1 = W.bP[pidx(g, cc, r - 1)]; topo3 = W.bP[pidx(g, cc, r + 1)]; }
            else { topo1 = W.bP[pidx(g, r - 1, cc)]; topo3 = W.bP[pidx(g, r + 1, cc)]; }
            double asdq[5], bm[5], bp[5];
            const double* src = imp == 1 ? amdq : apdq;
            asdq[0] = src[0]; asdq[1] = src[cn]; asdq[2] = src[ct]; asdq[3] = src[3]; asdq[4] = src[4];
            bool done = rpt2_split(P, h, hn, ht, hm, W.bP[pc], topo1, topo3, asdq, bm, bp);
            if (done && br) *br |= (imp == 1 ? BR_RPT1 : BR_RPT2);
            // back to q order
            double bmq[5] = {bm[0], 0.0, 0.0, bm[3], bm[4]}, bpq[5] = {bp[0], 0.0, 0.0, bp[3], bp[4]};
            bmq[cn] = bm[1]; bmq[ct] = bm[2];
            bpq[cn] = bp[1]; bpq[ct] = bp[2];
            double* Um = imp == 1 ? U1m : U2m;
            double* Up = imp == 1 ? U1p : U2p;
            for (int m = 0; m < 5; ++m) {
                Um[m] = half * bmq[m];
                Up[m] = half * bpq[m];
            }
        }
    }
    for (int m = 0; m < 5; ++m) {
        fo[(size_t)(0 + m) * nplane + oi] = faddm[m];
        fo[(size_t)(5 + m) * nplane + oi] = faddp[m];
        fo[(size_t)(10 + m) * nplane + oi] = U1m[m];
        fo[(size_t)(15 + m) * nplane + oi] = U1p[m];
        fo[(size_t)(20 + m) * nplane + oi] = U2m[m];
        fo[(size_t)(25 + m) * nplane + oi] = U2p[m];
    }
}

// ---------------------------------------------------------------------------
// Stage E. Interior cell (i, j): accumulate fm, fp, gm, gp in the order the
// reference's step2 adds them (x-sweep row j-1, row j, then y-sweep column
// i-1, column i) and apply stepgrid's flux-differencing update to the qB
// state. qn receives the updated state; fl (nullable, 4 x 5 values)
// receives fm(i+1,j), fp(i,j), gm(i,j+1), gp(i,j). Returns true on NaN.
DC_HD bool stage_update(const Geom& g, const Work& W, int i, int j, double dt, double qn[5], double* fl) {
    const double dtdx = dt / g.dx, dtdy = dt / g.dy;
    const double* fx = W.fx;
    const double* fy = W.fy;
    const size_t nx = W.nxi, ny = W.nyi;
    const size_t pc = pidx(g, i, j);
    for (int m = 0; m < 5; ++m) {
        // transverse increments of the y-sweeps into x-fluxes: column c, cell j
        auto G1y = [&](int c) -> double {
            return (0.0 - fy[(size_t)(10 + m) * ny + yidx(g, j + 1, c)]) - fy[(size_t)(20 + m) * ny + yidx(g, j, c)];
        };
        auto G2y = [&](int c) -> double {
            return (0.0 - fy[(size_t)(15 + m) * ny + yidx(g, j + 1, c)]) - fy[(size_t)(25 + m) * ny + yidx(g, j, c)];
        };
        // transverse increments of the x-sweeps into y-fluxes: row rr, cell i
        auto G1x = [&](int rr) -> double {
            return (0.0 - fx[(size_t)(10 + m) * nx + xidx(g, rr, i + 1)]) - fx[(size_t)(20 + m) * nx + xidx(g, rr, i)];
        };
        auto G2x = [&](int rr) -> double {
            return (0.0 - fx[(size_t)(15 + m) * nx + xidx(g, rr, i + 1)]) - fx[(size_t)(25 + m) * nx + xidx(g, rr, i)];
        };
        double fm = ((0.0 + fx[(size_t)(0 + m) * nx + xidx(g, j, i + 1)]) + G2y(i)) + G1y(i + 1);
        double fp = ((0.0 + fx[(size_t)(5 + m) * nx + xidx(g, j, i)]) + G2y(i - 1)) + G1y(i);
        double gm = ((0.0 + G2x(j)) + G1x(j + 1)) + fy[(size_t)(0 + m) * ny + yidx(g, j + 1, i)];
        double gp = ((0.0 + G2x(j - 1)) + G1x(j)) + fy[(size_t)(5 + m) * ny + yidx(g, j, i)];
        double q = W.qB[(size_t)m * W.npad + pc];
        qn[m] = q - dtdx * (fm - fp) - dtdy * (gm - gp);
        if (fl) { fl[m] = fm; fl[5 + m] = fp; fl[10 + m] = gm; fl[15 + m] = gp; }
    }
    return (qn[0] != qn[0]) || (qn[1] != qn[1]) || (qn[2] != qn[2]) || (qn[3] != qn[3]) || (qn[4] != qn[4]);
}

// Stage E of the fused step: update + src2, written to q_out (interior layout).
DC_HD bool stage_finalize(const dclaw_params& P, const Geom& g, const Work& W, double* __restrict__ q_out,
                          int i, int j, double dt) {
    double qn[5];
    bool nan = stage_update(g, W, i, j, dt, qn, nullptr);
    src2_cell(P, P.phi, dt, qn[0], qn[1], qn[2], qn[3], qn[4]);
    const size_t plane = (size_t)g.mx * g.my;
    const size_t c = (size_t)(j - 1) * g.mx + (size_t)(i - 1);
    for (int m = 0; m < 5; ++m) q_out[(size_t)m * plane + c] = qn[m];
    return nan;
}

// tick rule (tick.f:490-526; stepgrid dtnew = dt*cfl_desired/cflgrid)
DC_HD double tick_next_dt(const dclaw_params& P, double dt, double cfl) {
    double dtnew = cfl > 0.0 ? dt * P.cfl_desired / cfl : 1.0e300;
    return fmin2(dtnew, P.dt_max);
}

}  // namespace dclaw
