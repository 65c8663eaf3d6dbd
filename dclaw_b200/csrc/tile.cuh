// tile.cuh -- the fused uniform-patch step as two kernels.
//
// K1 (one thread per padded cell) builds a per-cell record: the b4step2
// state (ghost fill, qfix, speed limit), the quotients hu/h and hv/h, the
// solid fractions of the two rpn2 qfix passes (A1: once, A2: twice), the
// Coulomb stress tau of both states (setvars once per distinct state, not
// once per interface side), and calc_taudir's fsphi / taudir_x / taudir_y.
// K2 (one CTA per TX x TY tile) runs, in shared memory, the x-sweep Riemann
// solves of the tile rows +-1, the wave limiter, 2nd-order corrections and
// transverse splits, folds the transverse increments in step2's order, then
// the y-sweep likewise, and finishes with the flux-differencing update and
// src2. Every per-item function below is DC_HD so that a host emulation
// (tests/emu) runs the same arithmetic phase by phase.
//
// Shared-memory regions of a tile (TX x TY interior cells, origin i0, j0):
//   A  waves of one sweep direction: NW planes x (TY+2)(TX+3) items
//   B  x-fluxes faddm/faddp of the tile rows at interfaces i0..i0+TX
//   C  x-sweep transverse increments G1x/G2x (rows j0-1..j0+TY), then
//      T(k) = (0 + G2x(k-1)) + G1x(k), then gm/gp = T + faddm_y/faddp_y
//   D  y-sweep transverse increments G1y/G2y (columns i0-1..i0+TX)
#pragma once
#include "stages.cuh"

namespace dclaw {

// record planes (padded layout)
enum { R_H = 0, R_HU, R_HV, R_HM, R_P, R_UQ, R_VQ, R_M1, R_M2, R_TAU1, R_TAU2, R_FS, R_TDX, R_TDY, NREC };

struct Rec {
    double* r;     // NREC padded planes
    size_t npad;
    DC_HD double get(int f, size_t pi) const { return r[(size_t)f * npad + pi]; }
    DC_HD void put(int f, size_t pi, double v) const { r[(size_t)f * npad + pi] = v; }
};

// qB h of a padded cell straight from the interior input state (for
// calc_taudir's neighbours): the ghost fill only mirrors or copies h, and
// qfix turns h <= dry_tolerance into 0.
DC_HD double qB_h(const dclaw_params& P, const Geom& g, const double* q_in, int i, int j) {
    int si = i < 1 ? (P.bc_lower[0] == DCLAW_BC_WALL ? 1 - i : 1)
                   : (i > g.mx ? (P.bc_upper[0] == DCLAW_BC_WALL ? 2 * g.mx + 1 - i : g.mx) : i);
    int sj = j < 1 ? (P.bc_lower[1] == DCLAW_BC_WALL ? 1 - j : 1)
                   : (j > g.my ? (P.bc_upper[1] == DCLAW_BC_WALL ? 2 * g.my + 1 - j : g.my) : j);
    double h = q_in[(size_t)(sj - 1) * g.mx + (size_t)(si - 1)];
    return h <= P.dry_tolerance ? 0.0 : h;
}

DC_HD double bed_at(const Geom& g, const double* b_in, int i, int j) {
    int bi = i < 1 ? 1 : (i > g.mx ? g.mx : i);
    int bj = j < 1 ? 1 : (j > g.my ? g.my : j);
    return b_in[(size_t)(bj - 1) * g.mx + (size_t)(bi - 1)];
}

// rho of qfix for solid fraction m, and the admissible pressure clip
DC_HD double clip_p(const dclaw_params& P, double h, double m, double p) {
    double rho = P.rho_s * m + (1.0 - m) * P.rho_f;
    double pmax = rho * P.grav * h;
    p = fmax2(0.0, p);
    return fmin2(pmax, p);
}

// ---------------------------------------------------------------------------
// K1: record of padded cell (i, j), i in -1..mx+2, j in -1..my+2.
// Returns true when the source cell of the input holds a NaN.
DC_HD bool cell_record(const dclaw_params& P, const Geom& g, const double* __restrict__ q_in,
                       const double* __restrict__ b_in, const Rec& R, int i, int j) {
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
    const size_t pi = pidx(g, i, j);
    // every field is read: a NaN anywhere in the state is reported, as the
    // reference's check4nans does before b4step2
    double h = q_in[c];
    double hu = q_in[plane + c], hv = q_in[2 * plane + c], hm = q_in[3 * plane + c], p = q_in[4 * plane + c];
    bool nan = (h != h) || (hu != hu) || (hv != hv) || (hm != hm) || (p != p);
    bool wet = h > P.dry_tolerance;
    if (wet) {
        if (flip_u) hu = -hu;
        if (flip_v) hv = -hv;
        double u, v, m;
        qfix(P, h, hu, hv, hm, p, u, v, m, P.grav);   // b4step2
        double s = sqrt((sq(hu) + sq(hv))) / h;      // speed limit (h > 0)
        if (s > P.speed_limit) {
            double sratio = P.speed_limit / s;
            hu = hu * sratio;
            hv = hv * sratio;
        }
    } else {
        h = 0.0;
        hu = 0.0;
        hv = 0.0;
    }
    R.put(R_H, pi, h);
    double fs = 0.0, tdx = 0.0, tdy = 0.0;
    double tau1 = 0.0, rho1 = 0.0;
    if (wet) {
        const double uq = hu / h, vq = hv / h;
        double m1 = fmin2(fmax2(hm / h, 0.0), 1.0);
        double hm1 = h * m1;
        double p1 = clip_p(P, h, m1, p);
        double m2 = fmin2(fmax2(hm1 / h, 0.0), 1.0);
        double p2 = clip_p(P, h, m2, p1);
        SetVars s1 = setvars<false>(P, P.phi, h, uq, vq, m1, p1, P.grav);
        tau1 = s1.tau;
        rho1 = s1.rho;
        double tau2 = s1.tau;
        if (!(m2 == m1 && p2 == p1)) tau2 = setvars<false>(P, P.phi, h, uq, vq, m2, p2, P.grav).tau;
        R.put(R_HU, pi, hu);
        R.put(R_HV, pi, hv);
        R.put(R_HM, pi, hm);
        R.put(R_P, pi, p);
        R.put(R_UQ, pi, uq);
        R.put(R_VQ, pi, vq);
        R.put(R_M1, pi, m1);
        R.put(R_M2, pi, m2);
        R.put(R_TAU1, pi, tau1);
        R.put(R_TAU2, pi, tau2);
    }
    // calc_taudir on the inner ghost ring and the interior
    if (i >= 0 && j >= 0 && i <= mx + 1 && j <= my + 1) {
        const double dry = P.dry_tolerance, gz = P.grav;
        double hL = qB_h(P, g, q_in, i - 1, j), hR = qB_h(P, g, q_in, i + 1, j);
        double hB = qB_h(P, g, q_in, i, j - 1), hT = qB_h(P, g, q_in, i, j + 1);
        if (!((h + hL + hB + hR + hT) < dry)) {
            double b = bed_at(g, b_in, i, j);
            double eta = h + b;
            double etaL = hL + bed_at(g, b_in, i - 1, j);
            if (hL < dry) etaL = fmin2(etaL, eta);
            double etaR = hR + bed_at(g, b_in, i + 1, j);
            if (hR < dry) etaR = fmin2(etaR, eta);
            double etaB = hB + bed_at(g, b_in, i, j - 1);
            if (hB < dry) etaB = fmin2(etaB, eta);
            double etaT = hT + bed_at(g, b_in, i, j + 1);
            if (hT < dry) etaT = fmin2(etaT, eta);
            if (h < dry) {
                eta = fmin2(etaL, eta);
                eta = fmin2(etaB, eta);
            }
            const double dx = g.dx, dy = g.dy;
            const double sint = 0.0;
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
            if (hvnorm > 0.0) {
                tdx = -dx * hu / hvnorm;
                tdy = -dy * hv / hvnorm;
                double dot = fmin2(fmax2(0.0, Fx * hu), fmax2(0.0, Fy * hv));
                if (dot > 0.0) {
                    double Fproj = dot / hvnorm;
                    fs = fmin2(1.0, Fproj * rho1 / fmax2(tau1, 1.0e-16));
                }
            } else {
                if ((sq(FxL) + sq(Fy)) > 0.0) tdx = -dx * FxL / sqrt(sq(FxL) + sq(Fy));
                else tdx = dx * 1.0;
                if ((sq(Fx) + sq(FyL)) > 0.0) tdy = -dy * FyL / sqrt(sq(Fx) + sq(FyL));
                else tdy = dy * 1.0;
                if ((sq(tdy) + sq(tdx)) > 0.0) fs = 1.0;
            }
        }
    }
    R.put(R_FS, pi, fs);
    R.put(R_TDX, pi, tdx);
    R.put(R_TDY, pi, tdy);
    return nan;
}

// ---------------------------------------------------------------------------
template <int TX, int TY>
struct TileGeom {
    static constexpr int NXW = (TY + 2) * (TX + 3);   // x solves: rows j0-1..j0+TY, ifaces i0-1..i0+TX+1
    static constexpr int NYW = (TX + 2) * (TY + 3);   // y solves: cols i0-1..i0+TX, ifaces j0-1..j0+TY+1
    // The y solves' waves are stored column by column (y_slot), with an odd
    // pitch: the solves write them along rows and the flux phase reads them
    // down columns, both without shared-memory bank conflicts.
    static constexpr int YP = (TY + 3) | 1;
    static constexpr int NYS = (TX + 2) * YP;
    static constexpr int NA = NXW > NYS ? NXW : NYS;  // wave slots of either sweep
    static constexpr int NB = TY * (TX + 1);          // x-fluxes of tile rows, ifaces i0..i0+TX
    static constexpr int NC = (TY + 2) * TX;          // G1x/G2x rows j0-1..j0+TY (then gm/gp rows j0..j0+TY)
    static constexpr int ND = (TX + 2) * TY;          // G1y/G2y cols i0-1..i0+TX, rows j0..j0+TY-1 (by column)
    // h and bed of cells within 3 of the tile, rows of an odd pitch (one
    // unused column when TX + 6 is even): read along rows and down columns
    static constexpr int HW = (TX + 6) | 1;
    static constexpr int NHB = HW * (TY + 6);
    static constexpr int NTS = (TY + 1) * TX;         // T of tile columns, y-interfaces j0..j0+TY
    static constexpr size_t SMEM_DOUBLES = (size_t)NW * NA + 10 * NB + 10 * NC + 10 * ND + 2 * NHB + 5 * NTS;
    // + branch bits of the sweep's items, the list of items that need a
    // solve, and its length
    static constexpr size_t SMEM_BYTES = SMEM_DOUBLES * 8 + 4 * (size_t)NA + 4 * (size_t)NA + 16;
};

struct TileMem {
    double* A;   // NW planes of NA
    double* B;   // [NB][10]
    double* C;   // [NC][10]
    double* D;   // [ND][10], column by column
    double* H;   // record h of cells (i0-3..i0+TX+2) x (j0-3..j0+TY+2), row pitch hw
    double* Bd;  // bed of the same cells
    double* T5;  // [NTS][5]: T(k, c) of the x-sweep, read by the y-sweep's flux phase
    uint32_t* bits;  // NA Riemann branch bits of the current sweep
    int* list;       // NA: items of the current sweep that need a solve
    int* nlist;      // length of the list
    int NA;
    int hi0, hj0, hw;  // origin and row pitch of the H/Bd block
    int hv;            // staged cells per row (TX + 6)
    DC_HD double h(int i, int j) const { return H[(j - hj0) * hw + (i - hi0)]; }
    DC_HD double bed(int i, int j) const { return Bd[(j - hj0) * hw + (i - hi0)]; }
};

// stage record h and bed of block item `it` (cells within 3 of the tile);
// returns whether the cell is wet. Cells outside the padded patch are never
// read and are left unset.
DC_HD bool tile_stage_hb(const Geom& g, const Rec& R, const double* b_in, const TileMem& M, int it) {
    if (it % M.hw >= M.hv) return false;  // the pitch's unused column
    int i = M.hi0 + it % M.hw, j = M.hj0 + it / M.hw;
    if (i < -1 || i > g.mx + 2 || j < -1 || j > g.my + 2) return false;
    double h = R.get(R_H, pidx(g, i, j));
    M.H[it] = h;
    M.Bd[it] = bed_at(g, b_in, i, j);
    return h > 0.0;
}

// Slot of y-interface k (between rows k-1 and k) of column c in the wave
// planes: column-major with the odd pitch TileGeom::YP. The x-sweep's slot
// of an item is the item.
DC_HD int y_slot(int TY, int i0, int j0, int c, int k) { return (c - (i0 - 1)) * ((TY + 3) | 1) + (k - (j0 - 1)); }

// Solver side of a record cell after one (A1) or two (A2) qfix passes
DC_HD Side rec_side(const dclaw_params& P, const Rec& R, const Geom& g, const TileMem& M, int i, int j, int dir,
                    bool twice) {
    const size_t pi = pidx(g, i, j);
    Side s;
    s.b = M.bed(i, j);
    s.fs = R.get(R_FS, pi);
    s.taudir = R.get(dir == 0 ? R_TDX : R_TDY, pi);
    double h = M.h(i, j);
    if (h <= P.dry_tolerance) {
        s.h = 0.0; s.hn = 0.0; s.ht = 0.0; s.hm = 0.0; s.p = 0.0;
        s.un = 0.0; s.ut = 0.0; s.m = 0.0; s.rho_sv = 0.0; s.tau_sv = 0.0;
        return s;
    }
    double hu = R.get(R_HU, pi), hv = R.get(R_HV, pi);
    double uq = R.get(R_UQ, pi), vq = R.get(R_VQ, pi);
    double m1 = R.get(R_M1, pi);
    double p1 = clip_p(P, h, m1, R.get(R_P, pi));
    double m, p, tau;
    if (twice) {
        m = R.get(R_M2, pi);
        p = clip_p(P, h, m, p1);
        tau = R.get(R_TAU2, pi);
    } else {
        m = m1;
        p = p1;
        tau = R.get(R_TAU1, pi);
    }
    s.h = h;
    s.hn = dir == 0 ? hu : hv;
    s.ht = dir == 0 ? hv : hu;
    s.un = dir == 0 ? uq : vq;
    s.ut = dir == 0 ? vq : uq;
    s.m = m;
    s.hm = h * m;
    s.p = p;
    s.rho_sv = m * (P.rho_s - P.rho_f) + P.rho_f;
    s.tau_sv = tau;
    return s;
}

// expand a stored solve into q-ordered 5-vectors (dir 0: normal = hu,
// tangential = hv; dir 1: normal = hv, tangential = hu)
DC_HD void tile_waves(const TileMem& M, int dir, int item, double s[3], double W1[5], double W2[5], double W5[5]) {
    double v[NW];
    for (int k = 0; k < NW; ++k) v[k] = M.A[(size_t)k * M.NA + item];
    s[0] = v[W_S1]; s[1] = v[W_S2]; s[2] = v[W_S5];
    const bool y = dir != 0;
    W1[0] = v[W_1H]; W1[1] = y ? v[W_1T] : v[W_1N]; W1[2] = y ? v[W_1N] : v[W_1T]; W1[3] = v[W_1M]; W1[4] = v[W_1P];
    W2[0] = v[W_2H]; W2[1] = y ? 0.0 : v[W_2N]; W2[2] = y ? v[W_2N] : 0.0; W2[3] = 0.0; W2[4] = 0.0;
    W5[0] = v[W_5H]; W5[1] = y ? v[W_5T] : v[W_5N]; W5[2] = y ? v[W_5N] : v[W_5T]; W5[3] = v[W_5M]; W5[4] = v[W_5P];
}

// Whether item `item` of sweep `dir` needs a Riemann solve (inside the
// patch and not dry-dry); tile_riemann handles every other item with a
// store of zero waves.
DC_HD bool tile_needs_solve(const dclaw_params& P, const Geom& g, const TileMem& M, int dir, int item, int i0,
                            int j0, int TX) {
    int sl, k;
    if (dir == 0) { sl = j0 - 1 + item / (TX + 3); k = i0 - 1 + item % (TX + 3); }
    else { sl = i0 - 1 + item % (TX + 2); k = j0 - 1 + item / (TX + 2); }
    const int nslice = dir == 0 ? g.my : g.mx, nlen = dir == 0 ? g.mx : g.my;
    if (sl < 0 || sl > nslice + 1 || k < 0 || k > nlen + 2) return false;
    int iL = dir == 0 ? k - 1 : sl, jL = dir == 0 ? sl : k - 1;
    int iR = dir == 0 ? k : sl, jR = dir == 0 ? sl : k;
    return !(M.h(iL, jL) <= P.dry_tolerance && M.h(iR, jR) <= P.dry_tolerance);
}

// Riemann solve of sweep `dir` for tile-local item (slice s, interface k).
// dir 0: s = row r, k = x-interface; dir 1: s = column c, k = y-interface.
// Returns max |s| (0 for skipped items); cfl_ok tells whether the item
// counts for the Courant number.
DC_HD double tile_riemann(const dclaw_params& P, const Geom& g, const Rec& R, const TileMem& M, int dir,
                          int item, int i0, int j0, int TX, int TY, bool& cfl_ok) {
    int sl, k;
    if (dir == 0) { sl = j0 - 1 + item / (TX + 3); k = i0 - 1 + item % (TX + 3); }
    else { sl = i0 - 1 + item % (TX + 2); k = j0 - 1 + item / (TX + 2); }
    const int nslice = dir == 0 ? g.my : g.mx, nlen = dir == 0 ? g.mx : g.my;
    cfl_ok = false;
    Waves w;
    uint32_t bits = 0;
    if (sl < 0 || sl > nslice + 1 || k < 0 || k > nlen + 2) {
        zero_waves(w);
    } else {
        int iL = dir == 0 ? k - 1 : sl, jL = dir == 0 ? sl : k - 1;
        int iR = dir == 0 ? k : sl, jR = dir == 0 ? sl : k;
        double hL0 = M.h(iL, jL), hR0 = M.h(iR, jR);
        if (hL0 <= P.dry_tolerance && hR0 <= P.dry_tolerance) {
            zero_waves(w);
            bits |= BR_DRY;
        } else {
            Side Rs = rec_side(P, R, g, M, iR, jR, dir, false);
            Side Ls = rec_side(P, R, g, M, iL, jL, dir, k - 1 >= 0);
            w = riemann_solve(P, Ls, Rs, &bits);
        }
        cfl_ok = k >= 1 && k <= nlen + 1;
    }
    const double vals[NW] = {w.s1, w.s2, w.s5, w.w1h, w.w1n, w.w1t, w.w1m, w.w1p,
                             w.w2h, w.w2n, w.w5h, w.w5n, w.w5t, w.w5m, w.w5p};
    const int slot = dir == 0 ? item : y_slot(TY, i0, j0, sl, k);
    for (int f = 0; f < NW; ++f) M.A[(size_t)f * M.NA + slot] = vals[f];
    M.bits[slot] = bits;
    return fmax2(fmax2(fabs(w.s1), fabs(w.s2)), fabs(w.s5));
}

// A2 state (h, hn, ht, hm) of a record cell
DC_HD void rec_a2(const dclaw_params& P, const Rec& R, const Geom& g, const TileMem& M, int i, int j, int dir,
                  double& h, double& hn, double& ht, double& hm) {
    const size_t pi = pidx(g, i, j);
    h = M.h(i, j);
    if (h <= P.dry_tolerance) { h = 0.0; hn = 0.0; ht = 0.0; hm = 0.0; return; }
    double hu = R.get(R_HU, pi), hv = R.get(R_HV, pi);
    hn = dir == 0 ? hu : hv;
    ht = dir == 0 ? hv : hu;
    hm = h * R.get(R_M2, pi);
}

// limited waves + fluctuations at one interface (local position `pos` in
// the sweep's item grid; neighbours at pos-1, pos+1). Returns wet4.
DC_HD bool iface_limited(const dclaw_params& P, const TileMem& M, int dir, int item_m, int item, int item_p,
                         const double hcells[4], double dtdx, double amdq[5], double apdq[5], double cqxx[5],
                         uint32_t* bits) {
    double s[3], W1[5], W2[5], W5[5];
    tile_waves(M, dir, item, s, W1, W2, W5);
    for (int m = 0; m < 5; ++m) {
        double am = 0.0, ap = 0.0;
        if (s[0] < 0.0) am = am + W1[m]; else if (s[0] > 0.0) ap = ap + W1[m];
        if (s[1] < 0.0) am = am + W2[m]; else if (s[1] > 0.0) ap = ap + W2[m];
        if (s[2] < 0.0) am = am + W5[m]; else if (s[2] > 0.0) ap = ap + W5[m];
        amdq[m] = am;
        apdq[m] = ap;
        cqxx[m] = 0.0;
    }
    bool wet4 = false;
    if (P.order != 1) {
        if (P.limiter != 0) {
            double sm[3], Wm1[5], Wm2[5], Wm5[5], sp[3], Wp1[5], Wp2[5], Wp5[5];
            tile_waves(M, dir, item_m, sm, Wm1, Wm2, Wm5);
            tile_waves(M, dir, item_p, sp, Wp1, Wp2, Wp5);
            limit_family(P.limiter, 1, s[0], Wm1, W1, Wp1, bits);
            limit_family(P.limiter, 2, s[1], Wm2, W2, Wp2, bits);
            limit_family(P.limiter, 5, s[2], Wm5, W5, Wp5, bits);
        }
        wet4 = hcells[1] * hcells[2] * hcells[0] * hcells[3] > 0.0;
        if (wet4) {
            if (bits) *bits |= BR_WET4;
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
    }
    return wet4;
}

// transverse split (rpt2) of one fluctuation with the Jacobian of cell (ci, cj)
DC_HD bool split_cell(const dclaw_params& P, const Rec& R, const Geom& g, const TileMem& M, int dir, int ci,
                      int cj, const double src[5], double half, double Um[5], double Up[5]) {
    const bool y = dir != 0;
    double h, hn, ht, hm;
    rec_a2(P, R, g, M, ci, cj, dir, h, hn, ht, hm);
    double topo1, topo3;
    if (!y) { topo1 = M.bed(ci, cj - 1); topo3 = M.bed(ci, cj + 1); }
    else { topo1 = M.bed(ci - 1, cj); topo3 = M.bed(ci + 1, cj); }
    double asdq[5] = {src[0], y ? src[2] : src[1], y ? src[1] : src[2], src[3], src[4]}, bm[5], bp[5];
    bool done = rpt2_split(P, h, hn, ht, hm, M.bed(ci, cj), topo1, topo3, asdq, bm, bp);
    double bmq[5] = {bm[0], y ? bm[2] : bm[1], y ? bm[1] : bm[2], bm[3], bm[4]};
    double bpq[5] = {bp[0], y ? bp[2] : bp[1], y ? bp[1] : bp[2], bp[3], bp[4]};
    for (int m = 0; m < 5; ++m) {
        Um[m] = half * bmq[m];
        Up[m] = half * bpq[m];
    }
    return done;
}

// the two fluctuations a cell splits in one sweep (A-dq of its next
// interface, A+dq of its own), with the cell's Jacobian computed once:
// the same bits as two split_cell calls
DC_HD void split_cell2(const dclaw_params& P, const Rec& R, const Geom& g, const TileMem& M, int dir, int ci,
                       int cj, const double src1[5], const double src2[5], double half, double U1m[5],
                       double U1p[5], double U2m[5], double U2p[5], bool& d1, bool& d2) {
    const bool y = dir != 0;
    double h, hn, ht, hm;
    rec_a2(P, R, g, M, ci, cj, dir, h, hn, ht, hm);
    double topo1, topo3;
    if (!y) { topo1 = M.bed(ci, cj - 1); topo3 = M.bed(ci, cj + 1); }
    else { topo1 = M.bed(ci - 1, cj); topo3 = M.bed(ci + 1, cj); }
    const Rpt2Cell cell = rpt2_cell(P, h, hn, ht, hm, M.bed(ci, cj), topo1, topo3);
    auto one = [&](const double* src, double* Um, double* Up) -> bool {
        double asdq[5] = {src[0], y ? src[2] : src[1], y ? src[1] : src[2], src[3], src[4]}, bm[5], bp[5];
        bool done = rpt2_apply(cell, topo1, topo3, asdq, bm, bp);
        double bmq[5] = {bm[0], y ? bm[2] : bm[1], y ? bm[1] : bm[2], bm[3], bm[4]};
        double bpq[5] = {bp[0], y ? bp[2] : bp[1], y ? bp[1] : bp[2], bp[3], bp[4]};
        for (int m = 0; m < 5; ++m) {
            Um[m] = half * bmq[m];
            Up[m] = half * bpq[m];
        }
        return done;
    };
    d1 = one(src1, U1m, U1p);
    d2 = one(src2, U2m, U2p);
}

DC_HD void bits_or(uint32_t* log, size_t off, uint32_t b) {
    if (!log || !b) return;
#if defined(__CUDA_ARCH__)
    atomicOr(log + off, b);
#else
    log[off] |= b;
#endif
}

DC_HD size_t xlog_off(const Geom& g, int r, int k) { return (size_t)r * (g.mx + 1) + (size_t)(k - 1); }
DC_HD size_t ylog_off(const Geom& g, int c, int k) {
    return (size_t)(g.my + 2) * (g.mx + 1) + (size_t)c * (g.my + 1) + (size_t)(k - 1);
}

// Limited waves and fluctuations of x-interface a (between cells a-1 and a)
// on row r, packed as v = (amdq[5], apdq[5], cqxx[5]); the limiter's bits
// go to *bits. a and its neighbours a-1, a+1 lie in the x item grid.
template <int TX, int TY>
DC_HD void tile_x_iface(const dclaw_params& P, const TileMem& M, int r, int a, int i0, int j0, double dtdx,
                        double v[15], uint32_t* bits) {
    auto witem = [&](int k) -> int { return (r - (j0 - 1)) * (TX + 3) + (k - (i0 - 1)); };
    const double h0[4] = {M.h(a - 2, r), M.h(a - 1, r), M.h(a, r), M.h(a + 1, r)};
    iface_limited(P, M, 0, witem(a - 1), witem(a), witem(a + 1), h0, dtdx, v, v + 5, v + 10, bits);
}

// The same for y-interface a (between rows a-1 and a) of column c.
template <int TX, int TY>
DC_HD void tile_y_iface(const dclaw_params& P, const TileMem& M, int c, int a, int i0, int j0, double dtdy,
                        double v[15], uint32_t* bits) {
    auto witem = [&](int k) -> int { return y_slot(TY, i0, j0, c, k); };
    const double h0[4] = {M.h(c, a - 2), M.h(c, a - 1), M.h(c, a), M.h(c, a + 1)};
    iface_limited(P, M, 1, witem(a - 1), witem(a), witem(a + 1), h0, dtdy, v, v + 5, v + 10, bits);
}

template <int TX, int TY>
DC_HD void tile_flux_cell(const dclaw_params& P, const Geom& g, const Rec& R, const TileMem& M, int dir, int c,
                          int r, int i0, int j0, double dtdx, const double* v0, const double* v1, uint32_t lb0,
                          uint32_t lb1, uint32_t* log);

// Sweep flux phase for one cell of the sweep (dir 0: cell (c, r) of rows
// j0-1..j0+TY, columns i0..i0+TX-1; dir 1: cell (c, j) of columns
// i0-1..i0+TX, rows j0..j0+TY-1). Computes the fluxes of its own interface
// (and of the next one for the last cell), and the cell's transverse
// increments G1 = (0 - U1m(next iface)) - U2m(own iface), G2 likewise.
template <int TX, int TY>
DC_HD void tile_flux(const dclaw_params& P, const Geom& g, const Rec& R, const TileMem& M, int dir, int item,
                     int i0, int j0, double dtdx, uint32_t* log) {
    int c, r;  // cell column / row
    if (dir == 0) { r = j0 - 1 + item / TX; c = i0 + item % TX; }
    else { c = i0 - 1 + item % (TX + 2); r = j0 + item / (TX + 2); }
    const int mx = g.mx, my = g.my;
    if (c < (dir == 0 ? 1 : 0) || c > (dir == 0 ? mx : mx + 1)) return;
    if (r < (dir == 0 ? 0 : 1) || r > (dir == 0 ? my + 1 : my)) return;
    const int a = dir == 0 ? c : r;                 // this cell along the sweep
    auto witem = [&](int k) -> int {
        return dir == 0 ? (r - (j0 - 1)) * (TX + 3) + (k - (i0 - 1)) : y_slot(TY, i0, j0, c, k);
    };
    auto hcell = [&](int aa) -> double { return dir == 0 ? M.h(aa, r) : M.h(c, aa); };
    // own interface a (between cells a-1 and a) and the next one a+1
    double v0[15], v1[15];
    uint32_t b0 = 0, b1 = 0;
    const double h0[4] = {hcell(a - 2), hcell(a - 1), hcell(a), hcell(a + 1)};
    const double h1[4] = {h0[1], h0[2], h0[3], hcell(a + 2)};
    iface_limited(P, M, dir, witem(a - 1), witem(a), witem(a + 1), h0, dtdx, v0, v0 + 5, v0 + 10,
                  log ? &b0 : nullptr);
    iface_limited(P, M, dir, witem(a), witem(a + 1), witem(a + 2), h1, dtdx, v1, v1 + 5, v1 + 10,
                  log ? &b1 : nullptr);
    tile_flux_cell<TX, TY>(P, g, R, M, dir, c, r, i0, j0, dtdx, v0, v1, b0, b1, log);
}

// The rest of tile_flux for cell (c, r), given the limited fluctuations of
// its own interface (v0, limiter bits lb0) and of the next one (v1, lb1).
template <int TX, int TY>
DC_HD void tile_flux_cell(const dclaw_params& P, const Geom& g, const Rec& R, const TileMem& M, int dir, int c,
                          int r, int i0, int j0, double dtdx, const double* v0, const double* v1, uint32_t lb0,
                          uint32_t lb1, uint32_t* log) {
    const int mx = g.mx, my = g.my;
    const int a = dir == 0 ? c : r;                 // this cell along the sweep
    const int nlen = dir == 0 ? mx : my;
    auto witem = [&](int k) -> int {
        return dir == 0 ? (r - (j0 - 1)) * (TX + 3) + (k - (i0 - 1)) : y_slot(TY, i0, j0, c, k);
    };
    const double half = 0.5 * dtdx;
    const bool last = dir == 0 ? (c == (i0 + TX - 1 < mx ? i0 + TX - 1 : mx)) : (r == (j0 + TY - 1 < my ? j0 + TY - 1 : my));
    const bool in_tile = dir == 0 ? (r >= j0 && r <= j0 + TY - 1 && r <= my) : (c >= i0 && c <= i0 + TX - 1 && c <= mx);
    uint32_t b_own = lb0, b_next = lb1;
    const double *am0 = v0, *ap0 = v0 + 5, *cq0 = v0 + 10, *am1 = v1, *ap1 = v1 + 5, *cq1 = v1 + 10;
    const bool ord2 = P.order != 1;
    auto fadd = [&](const double* am, const double* ap, const double* cq, double fm[5], double fp[5]) {
        for (int m = 0; m < 5; ++m) {
            fm[m] = 0.0 + am[m];
            fp[m] = 0.0 - ap[m];
            if (ord2) {
                fm[m] = fm[m] + 0.5 * cq[m];
                fp[m] = fp[m] + 0.5 * cq[m];
            }
        }
    };
    if (in_tile) {
        double fm[5], fp[5];
        if (dir == 0) {
            fadd(am0, ap0, cq0, fm, fp);
            double* dst = M.B + (size_t)((r - j0) * (TX + 1) + (c - i0)) * 10;
            for (int m = 0; m < 5; ++m) { dst[m] = fm[m]; dst[5 + m] = fp[m]; }
            if (last) {
                fadd(am1, ap1, cq1, fm, fp);
                dst = M.B + (size_t)((r - j0) * (TX + 1) + (c + 1 - i0)) * 10;
                for (int m = 0; m < 5; ++m) { dst[m] = fm[m]; dst[5 + m] = fp[m]; }
            }
        } else {
            // gm/gp = T + faddm_y/faddp_y in region C slot (r, c)
            fadd(am0, ap0, cq0, fm, fp);
            double* slot = M.C + (size_t)((r - j0) * TX + (c - i0)) * 10;
            const double* ts = M.T5 + (size_t)((r - j0) * TX + (c - i0)) * 5;
            for (int m = 0; m < 5; ++m) {
                double t = ts[m];
                slot[m] = t + fm[m];
                slot[5 + m] = t + fp[m];
            }
            if (last) {
                fadd(am1, ap1, cq1, fm, fp);
                slot = M.C + (size_t)((r + 1 - j0) * TX + (c - i0)) * 10;
                ts = M.T5 + (size_t)((r + 1 - j0) * TX + (c - i0)) * 5;
                for (int m = 0; m < 5; ++m) {
                    double t = ts[m];
                    slot[m] = t + fm[m];
                    slot[5 + m] = t + fp[m];
                }
            }
        }
    }
    // transverse increments of this cell
    double U1m[5], U1p[5], U2m[5], U2p[5];
    for (int m = 0; m < 5; ++m) { U1m[m] = 0.0; U1p[m] = 0.0; U2m[m] = 0.0; U2p[m] = 0.0; }
    if (P.transverse_waves != 0) {
        const bool fold = ord2 && P.transverse_waves == 2;
        double src1[5], src2[5];
        for (int m = 0; m < 5; ++m) {
            src1[m] = fold ? am1[m] + cq1[m] : am1[m];   // A-dq at the next interface (imp = 1)
            src2[m] = fold ? ap0[m] - cq0[m] : ap0[m];   // A+dq at the own interface (imp = 2)
        }
        bool d1, d2;
        split_cell2(P, R, g, M, dir, c, r, src1, src2, half, U1m, U1p, U2m, U2p, d1, d2);
        if (d1) b_next |= BR_RPT1;
        if (d2) b_own |= BR_RPT2;
        if (log) {
            // splits the reference logs but the interior update does not use
            double Xm[5], Xp[5];
            if (a == 1) {   // imp = 1 at interface 1 (this cell's own) uses cell 0
                double s0[5];
                for (int m = 0; m < 5; ++m) s0[m] = fold ? am0[m] + cq0[m] : am0[m];
                int ci = dir == 0 ? 0 : c, cj = dir == 0 ? r : 0;
                if (split_cell(P, R, g, M, dir, ci, cj, s0, half, Xm, Xp)) b_own |= BR_RPT1;
            }
            if (a == nlen) {   // imp = 2 at interface n+1 uses cell n+1
                double s0[5];
                for (int m = 0; m < 5; ++m) s0[m] = fold ? ap1[m] - cq1[m] : ap1[m];
                int ci = dir == 0 ? a + 1 : c, cj = dir == 0 ? r : a + 1;
                if (split_cell(P, R, g, M, dir, ci, cj, s0, half, Xm, Xp)) b_next |= BR_RPT2;
            }
        }
    }
    double* G = dir == 0 ? M.C + (size_t)((r - (j0 - 1)) * TX + (c - i0)) * 10
                         : M.D + (size_t)((c - (i0 - 1)) * TY + (r - j0)) * 10;
    for (int m = 0; m < 5; ++m) {
        G[m] = (0.0 - U1m[m]) - U2m[m];
        G[5 + m] = (0.0 - U1p[m]) - U2p[m];
    }
    if (log) {
        const int s = dir == 0 ? r : c;
        if (a >= 1 && a <= nlen + 1)
            bits_or(log, dir == 0 ? xlog_off(g, s, a) : ylog_off(g, s, a), b_own | M.bits[witem(a)]);
        if (a + 1 >= 1 && a + 1 <= nlen + 1)
            bits_or(log, dir == 0 ? xlog_off(g, s, a + 1) : ylog_off(g, s, a + 1), b_next | M.bits[witem(a + 1)]);
    }
}

// T(k, c) = (0 + G2x(k-1, c)) + G1x(k, c) for tile columns, k = j0..j0+TY
template <int TX, int TY>
DC_HD bool tile_T(const Geom& g, const TileMem& M, int item, int i0, int j0, double T[5]) {
    int k = j0 + item / TX, c = i0 + item % TX;
    if (c > g.mx || k > g.my + 1) return false;
    const double* Gm = M.C + (size_t)((k - 1 - (j0 - 1)) * TX + (c - i0)) * 10;  // row k-1
    const double* Gk = M.C + (size_t)((k - (j0 - 1)) * TX + (c - i0)) * 10;      // row k
    for (int m = 0; m < 5; ++m) T[m] = (0.0 + Gm[5 + m]) + Gk[m];
    return true;
}

template <int TX, int TY>
DC_HD void tile_T_store(const TileMem& M, int item, const double T[5]) {
    double* slot = M.T5 + (size_t)item * 5;  // slot (k - j0, c - i0) == item
    for (int m = 0; m < 5; ++m) slot[m] = T[m];
}

// flux-differencing update of tile cell (i, j), written to q_out (interior
// layout); with WITH_SRC2 the cell's src2 follows in the same thread,
// otherwise q_out holds the updated state before src2. Returns true on NaN.
template <int TX, int TY, bool WITH_SRC2>
DC_HD bool tile_final(const dclaw_params& P, const Geom& g, const Rec& R, const TileMem& M, int item, int i0,
                      int j0, double dt, double* __restrict__ q_out) {
    int i = i0 + item % TX, j = j0 + item / TX;
    if (i > g.mx || j > g.my) return false;
    const double dtdx = dt / g.dx, dtdy = dt / g.dy;
    const size_t pc = pidx(g, i, j);
    double qb[5];
    qb[0] = M.h(i, j);
    if (qb[0] > 0.0) {
        qb[1] = R.get(R_HU, pc); qb[2] = R.get(R_HV, pc); qb[3] = R.get(R_HM, pc); qb[4] = R.get(R_P, pc);
    } else {
        qb[1] = 0.0; qb[2] = 0.0; qb[3] = 0.0; qb[4] = 0.0;
    }
    const double* Fx0 = M.B + (size_t)((j - j0) * (TX + 1) + (i - i0)) * 10;       // iface i
    const double* Fx1 = Fx0 + 10;                                                   // iface i+1
    const double* Gy_im = M.D + (size_t)((i - 1 - (i0 - 1)) * TY + (j - j0)) * 10;  // column i-1
    const double* Gy_i = Gy_im + (size_t)10 * TY;
    const double* Gy_ip = Gy_im + (size_t)20 * TY;
    const double* C0 = M.C + (size_t)((j - j0) * TX + (i - i0)) * 10;       // y-iface j
    const double* C1 = M.C + (size_t)((j + 1 - j0) * TX + (i - i0)) * 10;   // y-iface j+1
    double qn[5];
    for (int m = 0; m < 5; ++m) {
        double fm = ((0.0 + Fx1[m]) + Gy_i[5 + m]) + Gy_ip[m];
        double fp = ((0.0 + Fx0[5 + m]) + Gy_im[5 + m]) + Gy_i[m];
        double gm = C1[m];
        double gp = C0[5 + m];
        qn[m] = qb[m] - dtdx * (fm - fp) - dtdy * (gm - gp);
    }
    bool nan = (qn[0] != qn[0]) || (qn[1] != qn[1]) || (qn[2] != qn[2]) || (qn[3] != qn[3]) || (qn[4] != qn[4]);
    if (WITH_SRC2) src2_cell(P, P.phi, dt, qn[0], qn[1], qn[2], qn[3], qn[4]);
    const size_t plane = (size_t)g.mx * g.my;
    const size_t c = (size_t)(j - 1) * g.mx + (size_t)(i - 1);
    for (int m = 0; m < 5; ++m) q_out[(size_t)m * plane + c] = qn[m];
    return nan;
}

// src2 of interior cell c (0-based linear index) from the updated state
// q_star to q_out (interior layout)
DC_HD void cell_src2(const dclaw_params& P, const Geom& g, double dt, const double* __restrict__ q_star,
                     double* __restrict__ q_out, size_t c) {
    const size_t plane = (size_t)g.mx * g.my;
    double h = q_star[c];
    if (h <= P.dry_tolerance) {
        for (int m = 0; m < 5; ++m) q_out[(size_t)m * plane + c] = 0.0;
        return;
    }
    double a = h, b = q_star[plane + c], cc = q_star[2 * plane + c], d = q_star[3 * plane + c],
           e = q_star[4 * plane + c];
    src2_cell(P, P.phi, dt, a, b, cc, d, e);
    q_out[c] = a;
    q_out[plane + c] = b;
    q_out[2 * plane + c] = cc;
    q_out[3 * plane + c] = d;
    q_out[4 * plane + c] = e;
}

}  // namespace dclaw
