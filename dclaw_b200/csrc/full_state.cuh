// full_state.cuh -- the uniform-patch step on the reference's whole state,
// for segregation and entrainment.
//
// The reference carries q(7) = (h, hu, hv, hm, pb, hchi, bdif) in every run
// (digclaw_module.f90:96-102). With segregation = 0 and entrainment = 0, hchi
// and bdif stay exactly zero and the five-field step (stages.cuh, tile.cuh)
// gives the same bits without them. The stages below keep both:
//   hchi  h times the species fraction chi: clipped by qfix
//         (digclaw_module.f90:321-335), carried by the species waves of the
//         solver (riemannsolvers_dclaw.f:463-468) and by rpt2
//         (rpt2_dclaw.f:195-258), and through src2's updates; with
//         segregation = 1 it scales the permeability in setvars
//         (digclaw_module.f90:418-431)
//   bdif  the bed eroded by entrainment: the bed the step sees is aux(1) -
//         bdif in calc_taudir, rpn2 and rpt2's surface (digclaw_module.f90:
//         555-613, rpn2_dclaw.f:181-182, rpt2_dclaw.f:105,115); no wave
//         carries it, b4step2 clips it at 0 (b4step2.f90:62), and src2's
//         entrainment raises it (src2.f90:252-262, entrainment.f90:27-100)
// The staged form: one launch per stage over the padded patch or its
// interfaces (kernels.cu: k_full_*), the same structure as the five-field
// patch calls, with the stored waves and fluxes widened by the species
// component.
#pragma once
#include "workspace.cuh"

namespace dclaw {

enum { F_H = 0, F_HU, F_HV, F_HM, F_PB, F_HCHI, F_BDIF, NQF };
constexpr int NWF = NW + 2;               // + species components of waves 1 and 5
enum { W_1C = NW, W_5C = NW + 1 };
constexpr int NQC = 6;                    // components the waves carry (all but bdif)
constexpr int NFF = 6 * NQC;              // faddm faddp U1m U1p U2m U2p, 6 each

struct WorkF {
    double* qB;   // NQF padded planes: state after b4step2
    double* bP;   // padded bed, aux(1)
    double* td;   // 3 padded planes: fsphi, taudir_x, taudir_y
    double* wx;   // NWF x-interface planes
    double* wy;   // NWF y-interface planes
    double* fx;   // NFF x-interface planes
    double* fy;   // NFF y-interface planes
    size_t npad, nxi, nyi;
    // the bed the step sees: aux(1) - bdif
    DC_HD double beff(size_t pi) const { return bP[pi] - qB[(size_t)F_BDIF * npad + pi]; }
};

struct FullLayout {
    size_t npad, nxi, nyi;
    size_t off_qB, off_bP, off_td, off_wx, off_wy, off_fx, off_fy, total;
};

WS_HD FullLayout full_layout(int mx, int my) {
    FullLayout L;
    L.npad = (size_t)(mx + 4) * (my + 4);
    L.nxi = (size_t)(mx + 3) * (my + 2);
    L.nyi = (size_t)(my + 3) * (mx + 2);
    size_t o = 0;
    L.off_qB = o; o += align256((size_t)NQF * L.npad * 8);
    L.off_bP = o; o += align256(L.npad * 8);
    L.off_td = o; o += align256(3 * L.npad * 8);
    L.off_wx = o; o += align256((size_t)NWF * L.nxi * 8);
    L.off_wy = o; o += align256((size_t)NWF * L.nyi * 8);
    L.off_fx = o; o += align256((size_t)NFF * L.nxi * 8);
    L.off_fy = o; o += align256((size_t)NFF * L.nyi * 8);
    L.total = o;
    return L;
}

WS_HD WorkF make_work_full(void* base, const FullLayout& L) {
    char* b = (char*)base;
    WorkF W;
    W.qB = (double*)(b + L.off_qB);
    W.bP = (double*)(b + L.off_bP);
    W.td = (double*)(b + L.off_td);
    W.wx = (double*)(b + L.off_wx);
    W.wy = (double*)(b + L.off_wy);
    W.fx = (double*)(b + L.off_fx);
    W.fy = (double*)(b + L.off_fy);
    W.npad = L.npad;
    W.nxi = L.nxi;
    W.nyi = L.nyi;
    return W;
}

// qfix with the species fraction (digclaw_module.f90:285-345)
DC_HD void qfix_chi(const dclaw_params& P, double& h, double& hu, double& hv, double& hm, double& p, double& hchi,
                    double& u, double& v, double& m, double& chi, double gz) {
    if (h <= P.dry_tolerance) {
        h = 0.0; hu = 0.0; hv = 0.0; hm = 0.0; p = 0.0; hchi = 0.0;
        u = 0.0; v = 0.0; m = 0.0; chi = 0.0;
        return;
    }
    u = hu / h;
    v = hv / h;
    m = hm / h;
    chi = hchi / h;
    m = fmax2(m, 0.0);
    m = fmin2(m, 1.0);
    hm = h * m;
    chi = fmax2(chi, 0.0);
    chi = fmin2(chi, 1.0);
    hchi = h * chi;
    double rho = P.rho_s * m + (1.0 - m) * P.rho_f;
    double pmax = rho * gz * h;
    p = fmax2(0.0, p);
    p = fmin2(pmax, p);
}

// qfix's species part on a wet cell whose (h, hu, hv) it leaves as they are
DC_HD void qfix_c(double h, double& hchi, double& chi) {
    chi = hchi / h;
    chi = fmax2(chi, 0.0);
    chi = fmin2(chi, 1.0);
    hchi = h * chi;
}

// ---------------------------------------------------------------------------
// Stage A. Padded cell (i, j): ghost fill (hchi and bdif copied as they are),
// qfix, bdif >= 0, speed limit (b4step2.f90:56-100).
DC_HD bool full_b4(const dclaw_params& P, const Geom& g, const double* __restrict__ q_in,
                   const double* __restrict__ b_in, const WorkF& W, int i, int j) {
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
    double q[NQF];
    bool nan = false;
    for (int f = 0; f < NQF; ++f) {
        q[f] = q_in[(size_t)f * plane + c];
        nan = nan || (q[f] != q[f]);
    }
    if (flip_u) q[F_HU] = -q[F_HU];
    if (flip_v) q[F_HV] = -q[F_HV];
    double u, v, m, chi;
    qfix_chi(P, q[F_H], q[F_HU], q[F_HV], q[F_HM], q[F_PB], q[F_HCHI], u, v, m, chi, P.grav);
    q[F_BDIF] = fmax2(q[F_BDIF], 0.0);
    if (q[F_H] > 0.0) {
        double s = sqrt((sq(q[F_HU]) + sq(q[F_HV]))) / q[F_H];
        if (s > P.speed_limit) {
            double sratio = P.speed_limit / s;
            q[F_HU] = q[F_HU] * sratio;
            q[F_HV] = q[F_HV] * sratio;
        }
    }
    const size_t pi = pidx(g, i, j);
    for (int f = 0; f < NQF; ++f) W.qB[(size_t)f * W.npad + pi] = q[f];
    int bi = i < 1 ? 1 : (i > mx ? mx : i);
    int bj = j < 1 ? 1 : (j > my ? my : j);
    W.bP[pi] = b_in[(size_t)(bj - 1) * mx + (size_t)(bi - 1)];
    return nan;
}

// Stage B. calc_taudir on the bed less the bed change
DC_HD void full_taudir(const dclaw_params& P, const Geom& g, const WorkF& W, int i, int j) {
    const WorkF w = W;
    taudir_cell(P, g, W.qB, W.npad, W.td, [w](size_t q) { return w.beff(q); }, i, j);
}

// solver side after one or two rpn2 qfix passes, with chi (load_side)
DC_HD Side full_load_side(const dclaw_params& P, const WorkF& W, size_t pi, int comp_n, int comp_t, bool twice,
                          int taudir_plane) {
    Side s;
    double h = W.qB[pi];
    s.b = W.beff(pi);
    s.fs = W.td[pi];
    s.taudir = W.td[(size_t)taudir_plane * W.npad + pi];
    if (h <= P.dry_tolerance) {
        s.h = 0.0; s.hn = 0.0; s.ht = 0.0; s.hm = 0.0; s.p = 0.0;
        s.un = 0.0; s.ut = 0.0; s.m = 0.0;
        s.rho_sv = 0.0; s.tau_sv = 0.0; s.chi = 0.0;
        return s;
    }
    double hn = W.qB[(size_t)comp_n * W.npad + pi];
    double ht = W.qB[(size_t)comp_t * W.npad + pi];
    double hm = W.qB[(size_t)F_HM * W.npad + pi];
    double p = W.qB[(size_t)F_PB * W.npad + pi];
    double hchi = W.qB[(size_t)F_HCHI * W.npad + pi];
    double m, chi;
    qfix_mp(P, h, hm, p, m, P.grav);
    qfix_c(h, hchi, chi);
    if (twice) {
        qfix_mp(P, h, hm, p, m, P.grav);
        qfix_c(h, hchi, chi);
    }
    s.h = h; s.hn = hn; s.ht = ht; s.hm = hm; s.p = p; s.m = m; s.chi = chi;
    s.un = hn / h;
    s.ut = ht / h;
    SetVars sv = setvars<false>(P, P.phi, h, s.un, s.ut, m, p, P.grav);
    s.rho_sv = sv.rho;
    s.tau_sv = sv.tau;
    return s;
}

// Stage C. Interface i of slice r (stage_riemann with the species waves)
template <int DIR>
DC_HD double full_riemann(const dclaw_params& P, const Geom& g, const WorkF& W, int r, int i, uint32_t* br) {
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
    ChiWaves cw{0.0, 0.0};
    if (W.qB[pL] <= P.dry_tolerance && W.qB[pR] <= P.dry_tolerance) {
        zero_waves(w);
        if (br) *br |= BR_DRY;
    } else {
        Side R = full_load_side(P, W, pR, cn, ct, false, 1 + DIR);
        Side L = full_load_side(P, W, pL, cn, ct, i - 1 >= 0, 1 + DIR);
        w = riemann_solve(P, L, R, br, &cw);
    }
    const double vals[NWF] = {w.s1, w.s2, w.s5, w.w1h, w.w1n, w.w1t, w.w1m, w.w1p,
                              w.w2h, w.w2n, w.w5h, w.w5n, w.w5t, w.w5m, w.w5p, cw.w1c, cw.w5c};
    for (int k = 0; k < NWF; ++k) wv[(size_t)k * nplane + oi] = vals[k];
    return fmax2(fmax2(fabs(w.s1), fabs(w.s2)), fabs(w.s5));
}

// the stored waves at one interface as q-ordered 6-vectors (bdif has none)
template <int DIR>
DC_HD void full_expand_waves(const double* wv, size_t nplane, size_t oi, double s[3], double W1[NQC],
                             double W2[NQC], double W5[NQC]) {
    double v[NWF];
    for (int k = 0; k < NWF; ++k) v[k] = wv[(size_t)k * nplane + oi];
    s[0] = v[W_S1]; s[1] = v[W_S2]; s[2] = v[W_S5];
    const int cn = DIR == 0 ? 1 : 2, ct = DIR == 0 ? 2 : 1;
    W1[0] = v[W_1H]; W1[cn] = v[W_1N]; W1[ct] = v[W_1T]; W1[3] = v[W_1M]; W1[4] = v[W_1P]; W1[5] = v[W_1C];
    W2[0] = v[W_2H]; W2[cn] = v[W_2N]; W2[ct] = 0.0; W2[3] = 0.0; W2[4] = 0.0; W2[5] = 0.0;
    W5[0] = v[W_5H]; W5[cn] = v[W_5N]; W5[ct] = v[W_5T]; W5[3] = v[W_5M]; W5[4] = v[W_5P]; W5[5] = v[W_5C];
}

// the A2 state (two qfix passes) of a cell with its species field
DC_HD void full_load_a2(const dclaw_params& P, const WorkF& W, size_t pi, int cn, int ct, double& h, double& hn,
                        double& ht, double& hm, double& hchi) {
    h = W.qB[pi];
    if (h <= P.dry_tolerance) { h = 0.0; hn = 0.0; ht = 0.0; hm = 0.0; hchi = 0.0; return; }
    hn = W.qB[(size_t)cn * W.npad + pi];
    ht = W.qB[(size_t)ct * W.npad + pi];
    hm = W.qB[(size_t)F_HM * W.npad + pi];
    hchi = W.qB[(size_t)F_HCHI * W.npad + pi];
    double p = W.qB[(size_t)F_PB * W.npad + pi], m, chi;
    qfix_mp(P, h, hm, p, m, P.grav);
    qfix_c(h, hchi, chi);
    qfix_mp(P, h, hm, p, m, P.grav);
    qfix_c(h, hchi, chi);
}

// Stage D. Interface i (1..n+1) of slice r (stage_flux on six components)
template <int DIR>
DC_HD void full_flux(const dclaw_params& P, const Geom& g, const WorkF& W, int r, int i, double dtdx, uint32_t* br) {
    const double* wv = DIR == 0 ? W.wx : W.wy;
    double* fo = DIR == 0 ? W.fx : W.fy;
    const size_t nplane = DIR == 0 ? W.nxi : W.nyi;
    auto oidx = [&](int ii) -> size_t { return DIR == 0 ? xidx(g, r, ii) : yidx(g, ii, r); };
    auto cidx = [&](int ii) -> size_t { return DIR == 0 ? pidx(g, ii, r) : pidx(g, r, ii); };
    const int cn = DIR == 0 ? 1 : 2, ct = DIR == 0 ? 2 : 1;
    const size_t oi = oidx(i);

    double s[3], W1[NQC], W2[NQC], W5[NQC];
    full_expand_waves<DIR>(wv, nplane, oi, s, W1, W2, W5);
    double amdq[NQC], apdq[NQC];
    for (int m = 0; m < NQC; ++m) {
        double am = 0.0, ap = 0.0;
        if (s[0] < 0.0) am = am + W1[m]; else if (s[0] > 0.0) ap = ap + W1[m];
        if (s[1] < 0.0) am = am + W2[m]; else if (s[1] > 0.0) ap = ap + W2[m];
        if (s[2] < 0.0) am = am + W5[m]; else if (s[2] > 0.0) ap = ap + W5[m];
        amdq[m] = am;
        apdq[m] = ap;
    }
    double faddm[NQC], faddp[NQC], cqxx[NQC];
    for (int m = 0; m < NQC; ++m) {
        faddm[m] = 0.0 + amdq[m];
        faddp[m] = 0.0 - apdq[m];
        cqxx[m] = 0.0;
    }
    if (P.order != 1) {
        if (P.limiter != 0) {
            double sm[3], Wm1[NQC], Wm2[NQC], Wm5[NQC], sp[3], Wp1[NQC], Wp2[NQC], Wp5[NQC];
            full_expand_waves<DIR>(wv, nplane, oidx(i - 1), sm, Wm1, Wm2, Wm5);
            full_expand_waves<DIR>(wv, nplane, oidx(i + 1), sp, Wp1, Wp2, Wp5);
            limit_family<NQC>(P.limiter, 1, s[0], Wm1, W1, Wp1, br);
            limit_family<NQC>(P.limiter, 2, s[1], Wm2, W2, Wp2, br);
            limit_family<NQC>(P.limiter, 5, s[2], Wm5, W5, Wp5, br);
        }
        double hl2 = W.qB[cidx(i - 2)], hl = W.qB[cidx(i - 1)], hr = W.qB[cidx(i)], hr2 = W.qB[cidx(i + 1)];
        bool wet4 = hl * hr * hl2 * hr2 > 0.0;
        if (wet4) {
            if (br) *br |= BR_WET4;
            const double c1 = fsign(1.0, s[0]) * (1.0 - fabs(s[0]) * dtdx);
            const double c2 = fsign(1.0, s[1]) * (1.0 - fabs(s[1]) * dtdx);
            const double c5 = fsign(1.0, s[2]) * (1.0 - fabs(s[2]) * dtdx);
            for (int m = 0; m < NQC; ++m) {
                double cq = 0.0;
                cq = cq + c1 * W1[m];
                cq = cq + c2 * W2[m];
                cq = cq + c5 * W5[m];
                cqxx[m] = cq;
            }
        }
        for (int m = 0; m < NQC; ++m) {
            faddm[m] = faddm[m] + 0.5 * cqxx[m];
            faddp[m] = faddp[m] + 0.5 * cqxx[m];
        }
    }
    double U1m[NQC], U1p[NQC], U2m[NQC], U2p[NQC];
    for (int m = 0; m < NQC; ++m) { U1m[m] = 0.0; U1p[m] = 0.0; U2m[m] = 0.0; U2p[m] = 0.0; }
    if (P.transverse_waves != 0) {
        if (P.order > 1 && P.transverse_waves == 2) {
            for (int m = 0; m < NQC; ++m) {
                amdq[m] = amdq[m] + cqxx[m];
                apdq[m] = apdq[m] - cqxx[m];
            }
        }
        const double half = 0.5 * dtdx;
        for (int imp = 1; imp <= 2; ++imp) {
            const int cc = imp == 1 ? i - 1 : i;
            const size_t pc = cidx(cc);
            double h, hn, ht, hm, hchi;
            full_load_a2(P, W, pc, cn, ct, h, hn, ht, hm, hchi);
            // rpt2's neighbours' beds are aux(1) itself (rpt2_dclaw.f:107-108)
            double topo1, topo3;
            if (DIR == 0) { topo1 = W.bP[pidx(g, cc, r - 1)]; topo3 = W.bP[pidx(g, cc, r + 1)]; }
            else { topo1 = W.bP[pidx(g, r - 1, cc)]; topo3 = W.bP[pidx(g, r + 1, cc)]; }
            double asdq[5], bm[5], bp[5], b6[2];
            const double* src = imp == 1 ? amdq : apdq;
            asdq[0] = src[0]; asdq[1] = src[cn]; asdq[2] = src[ct]; asdq[3] = src[3]; asdq[4] = src[4];
            bool done = rpt2_split(P, h, hn, ht, hm, W.beff(pc), topo1, topo3, asdq, bm, bp, hchi, b6);
            if (done && br) *br |= (imp == 1 ? BR_RPT1 : BR_RPT2);
            double bmq[NQC] = {bm[0], 0.0, 0.0, bm[3], bm[4], b6[0]}, bpq[NQC] = {bp[0], 0.0, 0.0, bp[3], bp[4], b6[1]};
            bmq[cn] = bm[1]; bmq[ct] = bm[2];
            bpq[cn] = bp[1]; bpq[ct] = bp[2];
            double* Um = imp == 1 ? U1m : U2m;
            double* Up = imp == 1 ? U1p : U2p;
            for (int m = 0; m < NQC; ++m) {
                Um[m] = half * bmq[m];
                Up[m] = half * bpq[m];
            }
        }
    }
    for (int m = 0; m < NQC; ++m) {
        fo[(size_t)(0 * NQC + m) * nplane + oi] = faddm[m];
        fo[(size_t)(1 * NQC + m) * nplane + oi] = faddp[m];
        fo[(size_t)(2 * NQC + m) * nplane + oi] = U1m[m];
        fo[(size_t)(3 * NQC + m) * nplane + oi] = U1p[m];
        fo[(size_t)(4 * NQC + m) * nplane + oi] = U2m[m];
        fo[(size_t)(5 * NQC + m) * nplane + oi] = U2p[m];
    }
}

// Stage E's update (stage_update on six components; bdif passes through:
// no wave carries it, so its flux difference is an exact zero)
DC_HD bool full_update(const Geom& g, const WorkF& W, int i, int j, double dt, double qn[NQF]) {
    const double dtdx = dt / g.dx, dtdy = dt / g.dy;
    const double* fx = W.fx;
    const double* fy = W.fy;
    const size_t nx = W.nxi, ny = W.nyi;
    const size_t pc = pidx(g, i, j);
    for (int m = 0; m < NQC; ++m) {
        auto G1y = [&](int c) -> double {
            return (0.0 - fy[(size_t)(2 * NQC + m) * ny + yidx(g, j + 1, c)]) - fy[(size_t)(4 * NQC + m) * ny + yidx(g, j, c)];
        };
        auto G2y = [&](int c) -> double {
            return (0.0 - fy[(size_t)(3 * NQC + m) * ny + yidx(g, j + 1, c)]) - fy[(size_t)(5 * NQC + m) * ny + yidx(g, j, c)];
        };
        auto G1x = [&](int rr) -> double {
            return (0.0 - fx[(size_t)(2 * NQC + m) * nx + xidx(g, rr, i + 1)]) - fx[(size_t)(4 * NQC + m) * nx + xidx(g, rr, i)];
        };
        auto G2x = [&](int rr) -> double {
            return (0.0 - fx[(size_t)(3 * NQC + m) * nx + xidx(g, rr, i + 1)]) - fx[(size_t)(5 * NQC + m) * nx + xidx(g, rr, i)];
        };
        double fm = ((0.0 + fx[(size_t)(0 * NQC + m) * nx + xidx(g, j, i + 1)]) + G2y(i)) + G1y(i + 1);
        double fp = ((0.0 + fx[(size_t)(1 * NQC + m) * nx + xidx(g, j, i)]) + G2y(i - 1)) + G1y(i);
        double gm = ((0.0 + G2x(j)) + G1x(j + 1)) + fy[(size_t)(0 * NQC + m) * ny + yidx(g, j + 1, i)];
        double gp = ((0.0 + G2x(j - 1)) + G1x(j)) + fy[(size_t)(1 * NQC + m) * ny + yidx(g, j, i)];
        double q = W.qB[(size_t)m * W.npad + pc];
        qn[m] = q - dtdx * (fm - fp) - dtdy * (gm - gp);
    }
    qn[F_BDIF] = W.qB[(size_t)F_BDIF * W.npad + pc];
    bool nan = false;
    for (int m = 0; m < NQC; ++m) nan = nan || (qn[m] != qn[m]);
    return nan;
}

// ---------------------------------------------------------------------------
// mp_update_relax_Dclaw4 with the species fraction (mp_update.f90:710-789)
DC_HD void mp_update_relax_chi(const dclaw_params& P, double phi, double dt, double& h, double& u, double& v,
                               double& m, double& p, double& chi, double rhoh, double gz) {
    SetVars sv = setvars<true>(P, phi, h, u, v, m, p, gz, chi);
    double hu = h * u, hv = h * v, hm = h * m, hchi = h * chi;
    double vnorm = sqrt(sq(hu) + sq(hv)) / h;
    p = p - dt * 3.0 * vnorm * sv.tanpsi * sv.alphainv / h;
    qfix_chi(P, h, hu, hv, hm, p, hchi, u, v, m, chi, gz);
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
        hchi = h * chi;
        double e = em::d_exp(dt * krate);
        hu = hu * e;
        hv = hv * e;
        qfix_chi(P, h, hu, hv, hm, p, hchi, u, v, m, chi, gz);
    } else {
        h = (rhoh - hm * (P.rho_s - P.rho_f)) / P.rho_f;
        hu = h * u;
        hv = h * v;
        hchi = h * chi;
        qfix_chi(P, h, hu, hv, hm, p, hchi, u, v, m, chi, gz);
    }
}

// ent_dclaw4 (entrainment.f90:27-100): erosion of the bed layer into the
// flow. Its own hm is local (the caller's hm is not updated).
DC_HD void ent_dclaw4(const dclaw_params& P, double dt, double& h, double u, double v, double& m, double& p,
                      double& rho, double& hchi, double gz, double tau, double& b_eroded, double b_remaining) {
    const double coeff = P.friction_forcing ? P.manning_coefficient : 0.0;
    const double vnorm = sqrt(sq(u) + sq(v));
    const double vlow = 0.1;
    if (vnorm > vlow) {
        if (b_remaining > 0.0) {
            const double rhoe = P.me * P.rho_s + (1.0 - P.me) * P.rho_f;
            const double beta = fmax2(1.0 - m, 0.1);
            const double th = em::d_tanh(h + 1.0e-2);
            const double visc = beta * vnorm * 2.0 * P.mu * (1.0 - m) / (th);
            const double gamma = rho * beta * (sq(vnorm)) * (beta * gz * sq(coeff)) / (em::d_pow(th, 1.0 / 3.0));
            const double t1bot = visc + gamma + tau;
            const double t2top = fmin2(t1bot, (1.0 - beta * P.entrainment_rate) * tau);
            const double prat = p / (rho * h);
            double dh = P.entrainment_rate * dt * (t1bot - t2top) / (rhoe * beta * vnorm);
            dh = fmin2(dh, b_remaining);
            h = h + dh;
            const double hm = h * m + dh * P.me;
            m = hm / h;
            hchi = hchi + dh * P.chie;
            const double hrho = hm * P.rho_s + (h - hm) * P.rho_f;
            rho = hrho / h;
            b_eroded = b_eroded + dh;
            p = prat * hrho;
        }
    }
}

// src2 on one interior cell of the full state (src2.f90:100-300), in place;
// he: the erodible depth aux(i_ent) of the cell
DC_BIG void src2_cell_full(const dclaw_params& P, double phi, double dt, double q[NQF], double he) {
    double h = q[F_H];
    if (h <= P.dry_tolerance) {
        for (int f = 0; f < F_BDIF; ++f) q[f] = 0.0;
        return;
    }
    double hu = q[F_HU], hv = q[F_HV], hm = q[F_HM], p = q[F_PB], hchi = q[F_HCHI];
    double rhoh = hm * P.rho_s + (h - hm) * P.rho_f;
    if (hm < 0.0) return;
    const double gz = P.grav;
    const double gx = 0.0;
    double u, v, m, chi;
    qfix_chi(P, h, hu, hv, hm, p, hchi, u, v, m, chi, gz);
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
        hu = h * u; hv = h * v; hm = h * m; hchi = h * chi;
    } else if (P.src2method == 2) {
        double dtremaining = dt;
        int itercount = 0;
        while (dtremaining > 1.0e-99) {
            const double dtk = mp_update_fe4quad(P, phi, dtremaining, h, u, v, m, p, rhoh, gz, chi);
            dtremaining = dtremaining - dtk;
            itercount = itercount + 1;
            if (dtk == 0.0) break;
            if (h < P.dry_tolerance) break;
            if (itercount >= 100) break;
        }
        hu = h * u; hv = h * v; hm = h * m; hchi = h * chi;
        qfix_chi(P, h, hu, hv, hm, p, hchi, u, v, m, chi, gz);
    } else {
        mp_update_relax_chi(P, phi, dt, h, u, v, m, p, chi, rhoh, gz);
        hu = h * u; hv = h * v; hm = h * m; hchi = h * chi;
    }
    if (h <= P.dry_tolerance) {
        for (int f = 0; f < F_BDIF; ++f) q[f] = 0.0;
        return;
    }
    if (P.entrainment == 1 && P.entrainment_method == 0) {
        SetVars se = setvars<false>(P, phi, h, u, v, m, p, gz);
        double rho = se.rho, b_eroded = q[F_BDIF];
        ent_dclaw4(P, dt, h, u, v, m, p, rho, hchi, gz, se.tau, b_eroded, he - b_eroded);
        q[F_BDIF] = b_eroded;
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
            qfix_chi(P, h, hu, hv, hm, p, hchi, u, v, m, chi, gz);
        }
    }
    q[F_H] = h; q[F_HU] = hu; q[F_HV] = hv; q[F_HM] = hm; q[F_PB] = p; q[F_HCHI] = hchi;
}

// Stage E: update + src2, written to q_out (interior layout, NQF planes)
DC_HD bool full_finalize(const dclaw_params& P, const Geom& g, const WorkF& W, const double* __restrict__ he,
                         double* __restrict__ q_out, int i, int j, double dt) {
    double qn[NQF];
    bool nan = full_update(g, W, i, j, dt, qn);
    const size_t plane = (size_t)g.mx * g.my;
    const size_t c = (size_t)(j - 1) * g.mx + (size_t)(i - 1);
    src2_cell_full(P, P.phi, dt, qn, he ? he[c] : 0.0);
    for (int f = 0; f < NQF; ++f) q_out[(size_t)f * plane + c] = qn[f];
    return nan;
}

}  // namespace dclaw
