// adj_check.cpp -- TEST INFRASTRUCTURE: host builds of the adjoint routines
// (dclaw_b200/csrc/adjoint.cuh) checked against central finite differences
// of their forward routines, plus a host run of the whole adjoint step over
// the staged forward intermediates (same item functions as the kernels).
// Not a product path.
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <functional>
#include <random>
#include <vector>

#include "../../dclaw_b200/csrc/adjoint.cuh"

using namespace dclaw;
using Vec = std::vector<double>;

namespace {

struct Rng {
    std::mt19937_64 g;
    explicit Rng(uint64_t s) : g(s) {}
    double u(double a, double b) { return std::uniform_real_distribution<double>(a, b)(g); }
    bool coin(double p) { return u(0.0, 1.0) < p; }
};

dclaw_params default_params() {
    dclaw_params p;
    memset(&p, 0, sizeof(p));
    p.grav = 9.81; p.dry_tolerance = 1e-3; p.speed_limit = 1e6; p.friction_depth = 1e6; p.manning_max = 0.06;
    p.rho_s = 2700; p.rho_f = 1000; p.m_crit = 0.64; p.m0 = 0.62; p.mref = 0.60; p.kref = 1e-10;
    p.phi = 32.0 * 3.14159265358979323846 / 180.0; p.delta = 0.01; p.mu = 0.005; p.alpha_c = 0.01; p.c1 = 1.0;
    p.sigma_0 = 1e3; p.order = 2; p.transverse_waves = 2; p.limiter = 4;
    p.bc_lower[0] = p.bc_lower[1] = p.bc_upper[0] = p.bc_upper[1] = DCLAW_BC_WALL;
    p.cfl_desired = 0.9; p.cfl_max = 1.0; p.dt_max = 1e99;
    return p;
}

// directional check: ad = <xb, dx>, fd = <yb, (f(x+e dx) - f(x-e dx)) / 2e>.
// Returns the relative error, or -1 when two step sizes disagree (a kink of
// the forward function lies within the step: the sample is skipped).
double dircheck(const std::function<Vec(const Vec&)>& f, const Vec& x, const Vec& dx, const Vec& yb, double ad) {
    auto fd_at = [&](double e) {
        Vec xp(x), xm(x);
        for (size_t k = 0; k < x.size(); ++k) { xp[k] += e * dx[k]; xm[k] -= e * dx[k]; }
        Vec yp = f(xp), ym = f(xm);
        double s = 0.0;
        for (size_t k = 0; k < yb.size(); ++k) s += yb[k] * (yp[k] - ym[k]);
        return s / (2.0 * e);
    };
    double f1 = fd_at(1e-6), f2 = fd_at(2.5e-7);
    double scale = fmax(fabs(f1), fmax(fabs(f2), fabs(ad)));
    if (scale < 1e-300) return 0.0;
    if (fabs(f1 - f2) > 1e-5 * scale + 1e-14) return -1.0;
    return fabs(ad - f1) / fmax(scale, 1e-12);
}

struct Stat {
    double maxerr = 0.0;
    int skipped = 0, n = 0;
    void add(double e) {
        ++n;
        if (e < 0) ++skipped;
        else if (e > maxerr) maxerr = e;
    }
};

Vec randv(Rng& r, size_t n, double a = -1.0, double b = 1.0) {
    Vec v(n);
    for (auto& x : v) x = r.u(a, b);
    return v;
}

double dot(const Vec& a, const Vec& b) {
    double s = 0.0;
    for (size_t k = 0; k < a.size(); ++k) s += a[k] * b[k];
    return s;
}

// a wet cell state (h, hu, hv, hm, p); clip = allow m and p outside their bounds
Vec rand_state(Rng& r, bool clip) {
    double h = r.u(0.05, 3.0);
    double hu = h * r.u(-2.0, 2.0), hv = h * r.u(-2.0, 2.0);
    double m = clip ? r.u(-0.1, 1.1) : r.u(0.45, 0.68);
    double rho = 2700.0 * fmin(fmax(m, 0.0), 1.0) + (1.0 - fmin(fmax(m, 0.0), 1.0)) * 1000.0;
    double p = (clip ? r.u(-0.2, 1.2) : r.u(0.3, 0.95)) * rho * 9.81 * h;
    return {h, hu, hv, h * m, p};
}

// ---- local routine checks ---------------------------------------------------
Stat check_qfix(Rng& r, int n) {
    dclaw_params P = default_params();
    Stat st;
    auto f = [&](const Vec& x) {
        double h = x[0], hu = x[1], hv = x[2], hm = x[3], p = x[4], u, v, m;
        qfix(P, h, hu, hv, hm, p, u, v, m, P.grav);
        return Vec{h, hu, hv, hm, p, u, v, m};
    };
    for (int s = 0; s < n; ++s) {
        Vec x = rand_state(r, true);
        Vec dx = randv(r, 5), yb = randv(r, 8);
        for (int k = 0; k < 5; ++k) dx[k] *= fabs(x[k]) + 1e-3;
        double hb = yb[0], hub = yb[1], hvb = yb[2], hmb = yb[3], pb = yb[4];
        qfix_b(P, x[0], x[1], x[2], x[3], x[4], P.grav, hb, hub, hvb, hmb, pb, yb[5], yb[6], yb[7]);
        st.add(dircheck(f, x, dx, yb, hb * dx[0] + hub * dx[1] + hvb * dx[2] + hmb * dx[3] + pb * dx[4]));
    }
    return st;
}

Stat check_qfix_cmass(Rng& r, int n) {
    dclaw_params P = default_params();
    Stat st;
    // inputs m, p_exc, u, v, rhoh
    auto f = [&](const Vec& x) {
        double h = 0, m = x[0], p = 0, rho = 0, pex = x[1], hu = 0, hv = 0, hm = 0;
        qfix_cmass(P, h, m, p, rho, pex, hu, hv, hm, x[2], x[3], x[4], P.grav);
        return Vec{h, m, p, rho, pex, hu, hv, hm};
    };
    for (int s = 0; s < n; ++s) {
        double h = r.u(0.05, 3.0);
        double rhoh = h * r.u(1100.0, 2600.0);
        Vec x{r.u(-0.1, 1.1), r.u(-1.5, 1.5) * 9.81 * rhoh, r.u(-2, 2), r.u(-2, 2), rhoh};
        Vec dx = randv(r, 5), yb = randv(r, 8);
        for (int k = 0; k < 5; ++k) dx[k] *= fabs(x[k]) + 1e-3;
        double mb = yb[1], pexb = yb[4], ub = 0, vb = 0, rhohb = 0;
        qfix_cmass_b(P, x[0], x[1], x[2], x[3], x[4], P.grav, yb[0], mb, yb[2], yb[3], pexb, yb[5], yb[6], yb[7],
                     ub, vb, rhohb);
        st.add(dircheck(f, x, dx, yb, mb * dx[0] + pexb * dx[1] + ub * dx[2] + vb * dx[3] + rhohb * dx[4]));
    }
    return st;
}

// setvars with the differentiated parameters as extra inputs (phi, kref, alpha_c, mu)
template <bool ALL>
Stat check_setvars(Rng& r, int n, int alphamethod) {
    dclaw_params P0 = default_params();
    P0.alphamethod = alphamethod;
    Stat st;
    auto f = [&](const Vec& x) {
        dclaw_params P = P0;
        P.kref = x[7]; P.alpha_c = x[8]; P.mu = x[9];
        SetVars o = setvars<ALL>(P, x[0], x[1], x[2], x[3], x[4], x[5], P.grav);
        (void)x[6];
        return Vec{o.rho, o.kperm, o.alphainv, o.m_eq, o.tanpsi, o.tau};
    };
    for (int s = 0; s < n; ++s) {
        Vec q = rand_state(r, false);
        double h = q[0];
        Vec x{r.u(0.4, 0.7), h, q[1] / h, q[2] / h, q[3] / h, q[4], 0.0, 1e-10 * r.u(0.5, 2), 0.01 * r.u(0.5, 2),
              0.005 * r.u(0.5, 2)};
        if (r.coin(0.2)) { x[2] = 0.0; x[3] = 0.0; }
        Vec dx = randv(r, 10), yb = randv(r, 6);
        for (int k = 0; k < 10; ++k) dx[k] *= fabs(x[k]) + (k < 6 ? 1e-3 : 0.0);
        if (x[2] == 0.0) { dx[2] = 0.0; dx[3] = 0.0; }
        dclaw_params P = P0;
        P.kref = x[7]; P.alpha_c = x[8]; P.mu = x[9];
        SetVars ob{yb[0], yb[1], yb[2], yb[3], yb[4], yb[5]};
        double phib = 0, hb = 0, ub = 0, vb = 0, mb = 0, pb = 0, pbar[NPB] = {0, 0, 0, 0};
        setvars_b<ALL>(P, x[0], x[1], x[2], x[3], x[4], x[5], P.grav, ob, phib, hb, ub, vb, mb, pb, pbar);
        double ad = phib * dx[0] + hb * dx[1] + ub * dx[2] + vb * dx[3] + mb * dx[4] + pb * dx[5] +
                    pbar[PB_KREF] * dx[7] + pbar[PB_ALPHA] * dx[8] + pbar[PB_MU] * dx[9];
        st.add(dircheck(f, x, dx, yb, ad));
    }
    return st;
}

Stat check_riemanntype(Rng& r, int n) {
    Stat st;
    const double drytol = 1e-3, g = 9.81;
    auto f = [&](const Vec& x) {
        RType t = riemanntype(x[0], x[1], x[2], x[3], drytol, g);
        return Vec{t.hm, t.s1m, t.s2m};
    };
    for (int s = 0; s < n; ++s) {
        Vec x{r.u(0.05, 3.0), r.u(0.05, 3.0), r.u(-4, 4), r.u(-4, 4)};
        if (r.coin(0.15)) x[r.coin(0.5) ? 0 : 1] = 0.0;
        Vec dx = randv(r, 4), yb = randv(r, 3);
        for (int k = 0; k < 2; ++k) dx[k] = x[k] == 0.0 ? 0.0 : dx[k] * x[k];
        double hLb = 0, hRb = 0, uLb = 0, uRb = 0;
        riemanntype_b(x[0], x[1], x[2], x[3], drytol, g, yb[0], yb[1], yb[2], hLb, hRb, uLb, uRb);
        st.add(dircheck(f, x, dx, yb, hLb * dx[0] + hRb * dx[1] + uLb * dx[2] + uRb * dx[3]));
    }
    return st;
}

// Side <-> flat vector of its 13 fields
Vec side_vec(const Side& s) {
    return {s.h, s.hn, s.ht, s.hm, s.p, s.un, s.ut, s.m, s.b, s.taudir, s.fs, s.rho_sv, s.tau_sv};
}
Side vec_side(const double* v) {
    Side s;
    s.h = v[0]; s.hn = v[1]; s.ht = v[2]; s.hm = v[3]; s.p = v[4]; s.un = v[5]; s.ut = v[6]; s.m = v[7];
    s.b = v[8]; s.taudir = v[9]; s.fs = v[10]; s.rho_sv = v[11]; s.tau_sv = v[12];
    return s;
}
Vec sideb_vec(const SideB& s) {
    return {s.h, s.hn, s.ht, s.hm, s.p, s.un, s.ut, s.m, s.b, s.taudir, s.fs, s.rho_sv, s.tau_sv};
}
Vec waves_vec(const Waves& w) {
    return {w.s1, w.s2, w.s5, w.w1h, w.w1n, w.w1t, w.w1m, w.w1p, w.w2h, w.w2n, w.w5h, w.w5n, w.w5t, w.w5m, w.w5p};
}

Side rand_side(Rng& r, const dclaw_params& P, bool dry, bool still) {
    Side s;
    if (dry) {
        s.h = s.hn = s.ht = s.hm = s.p = s.un = s.ut = s.m = s.rho_sv = s.tau_sv = 0.0;
    } else {
        Vec q = rand_state(r, false);
        s.h = q[0]; s.hn = still ? 0.0 : q[1]; s.ht = still ? 0.0 : q[2]; s.hm = q[3]; s.p = q[4];
        s.un = s.hn / s.h; s.ut = s.ht / s.h; s.m = s.hm / s.h;
        SetVars sv = setvars<false>(P, P.phi, s.h, s.un, s.ut, s.m, s.p, P.grav);
        s.rho_sv = sv.rho; s.tau_sv = sv.tau;
    }
    s.b = r.u(-1.0, 1.0);
    s.taudir = r.u(-0.5, 0.5);
    s.fs = r.u(0.0, 1.0);
    return s;
}

// the rare-wave corrector changes the middle wave of this interface
static bool corrector_acts(const dclaw_params& P, const Side& L, const Side& R) {
    dclaw_params Q = P;
    Q.rarecorrectortest = 0;
    Waves a = riemann_solve(P, L, R, nullptr), b = riemann_solve(Q, L, R, nullptr);
    return a.s2 != b.s2 || a.w2h != b.w2h;
}

Stat check_riemann(Rng& r, int n, int mode) {
    dclaw_params P = default_params();
    if (mode == 3) P.src2method = -1;
    if (mode == 4) P.rarecorrectortest = 1;
    Stat st;
    auto f = [&](const Vec& x) { return waves_vec(riemann_solve(P, vec_side(&x[0]), vec_side(&x[13]), nullptr)); };
    for (int s = 0; s < n; ++s) {
        bool dryL = mode == 1 && r.coin(0.5), dryR = mode == 1 && !dryL;
        bool still = mode == 2;
        Side L = rand_side(r, P, dryL, still), R = rand_side(r, P, dryR, still);
        if (mode == 4) {
            // spreading flows whose rarefaction the corrector picks as the middle wave
            for (int tries = 0; tries < 400 && !corrector_acts(P, L, R); ++tries) {
                L = rand_side(r, P, false, false);
                R = rand_side(r, P, false, false);
                const double du = r.u(0.2, 3.0);
                L.un = -du; L.hn = L.h * L.un;
                R.un = du * r.u(0.2, 1.0); R.hn = R.h * R.un;
            }
        }
        if (mode == 1 && r.coin(0.5)) {  // make a wall problem likely
            if (dryR) R.b = L.b + L.h + r.u(0.5, 2.0);
            else L.b = R.b + R.h + r.u(0.5, 2.0);
        }
        Vec x = side_vec(L), xr = side_vec(R);
        x.insert(x.end(), xr.begin(), xr.end());
        Vec dx = randv(r, 26), yb = randv(r, 15);
        for (int k = 0; k < 26; ++k) {
            int fld = k % 13;
            dx[k] *= fabs(x[k]) + 1e-3;
            if ((k < 13 && dryL) || (k >= 13 && dryR)) if (fld != 8 && fld != 9 && fld != 10) dx[k] = 0.0;
            if (still && (fld == 1 || fld == 2 || fld == 5 || fld == 6)) dx[k] = 0.0;
        }
        Waves wb;
        wb.s1 = yb[0]; wb.s2 = yb[1]; wb.s5 = yb[2]; wb.w1h = yb[3]; wb.w1n = yb[4]; wb.w1t = yb[5]; wb.w1m = yb[6];
        wb.w1p = yb[7]; wb.w2h = yb[8]; wb.w2n = yb[9]; wb.w5h = yb[10]; wb.w5n = yb[11]; wb.w5t = yb[12];
        wb.w5m = yb[13]; wb.w5p = yb[14];
        SideB Lb, Rb;
        zero_sideb(Lb);
        zero_sideb(Rb);
        riemann_solve_b(P, L, R, wb, Lb, Rb);
        Vec xb = sideb_vec(Lb), xbr = sideb_vec(Rb);
        xb.insert(xb.end(), xbr.begin(), xbr.end());
        // a sample where the corrector does not act counts as skipped
        if (mode == 4 && !corrector_acts(P, L, R)) st.add(-1.0);
        else st.add(dircheck(f, x, dx, yb, dot(xb, dx)));
    }
    return st;
}

Stat check_limiter(Rng& r, int n, int mth) {
    Stat st;
    for (int s = 0; s < n; ++s) {
        double sp = r.coin(0.5) ? r.u(0.1, 3) : -r.u(0.1, 3);
        Vec x = randv(r, 15);
        auto f = [&](const Vec& v) {
            double Wi[5];
            for (int m = 0; m < 5; ++m) Wi[m] = v[5 + m];
            limit_family(mth, 1, sp, &v[0], Wi, &v[10], nullptr);
            return Vec{Wi[0], Wi[1], Wi[2], Wi[3], Wi[4]};
        };
        Vec dx = randv(r, 15), yb = randv(r, 5);
        double Wib[5], Wmb[5] = {0, 0, 0, 0, 0}, Wpb[5] = {0, 0, 0, 0, 0};
        for (int m = 0; m < 5; ++m) Wib[m] = yb[m];
        limit_family_b(mth, sp, &x[0], &x[5], &x[10], Wib, Wmb, Wpb);
        double ad = 0.0;
        for (int m = 0; m < 5; ++m) ad += Wmb[m] * dx[m] + Wib[m] * dx[5 + m] + Wpb[m] * dx[10 + m];
        st.add(dircheck(f, x, dx, yb, ad));
    }
    return st;
}

Stat check_rpt2(Rng& r, int n) {
    dclaw_params P = default_params();
    Stat st;
    for (int s = 0; s < n; ++s) {
        Vec q = rand_state(r, false);
        double b = r.u(-0.5, 0.5);
        double t1 = r.coin(0.8) ? b + r.u(-1, 0.5) : b + q[0] + 0.5, t3 = b + r.u(-1, 0.5);
        Vec x{q[0], q[1], q[2], q[3], r.u(-1, 1), r.u(-1, 1), r.u(-1, 1), r.u(-1, 1), r.u(-1, 1)};
        auto f = [&](const Vec& v) {
            double bm[5], bp[5];
            rpt2_split(P, v[0], v[1], v[2], v[3], b, t1, t3, &v[4], bm, bp);
            return Vec{bm[0], bm[1], bm[2], bm[3], bm[4], bp[0], bp[1], bp[2], bp[3], bp[4]};
        };
        Vec dx = randv(r, 9), yb = randv(r, 10);
        for (int k = 0; k < 4; ++k) dx[k] *= fabs(x[k]) + 1e-3;
        double xb[4] = {0, 0, 0, 0}, asb[5] = {0, 0, 0, 0, 0};
        rpt2_split_b(P, x[0], x[1], x[2], x[3], b, t1, t3, &x[4], &yb[0], &yb[5], xb, asb);
        double ad = xb[0] * dx[0] + xb[1] * dx[1] + xb[2] * dx[2] + xb[3] * dx[3];
        for (int k = 0; k < 5; ++k) ad += asb[k] * dx[4 + k];
        st.add(dircheck(f, x, dx, yb, ad));
    }
    return st;
}

// src2 on one cell, with phi, kref, alpha_c, mu as extra inputs; manning:
// 1 Manning friction with a constant coefficient, 2 depth-dependent
Stat check_src2(Rng& r, int n, int method, bool still, int manning = 0) {
    dclaw_params P0 = default_params();
    P0.src2method = method;
    if (manning) {
        P0.friction_forcing = 1;
        P0.manning_coefficient = 0.06;
        P0.friction_depth = 1.0e6;
        P0.dd_manning = manning == 2 ? 1 : 0;
        P0.manning_max = 0.1;
    }
    Stat st;
    const double dt = 0.01;
    auto f = [&](const Vec& x) {
        dclaw_params P = P0;
        P.kref = x[6]; P.alpha_c = x[7]; P.mu = x[8];
        double q[5] = {x[0], x[1], x[2], x[3], x[4]};
        src2_cell(P, x[5], dt, q[0], q[1], q[2], q[3], q[4]);
        return Vec{q[0], q[1], q[2], q[3], q[4]};
    };
    for (int s = 0; s < n; ++s) {
        Vec q = rand_state(r, false);
        if (still) { q[1] = 0.0; q[2] = 0.0; }
        Vec x{q[0], q[1], q[2], q[3], q[4], r.u(0.45, 0.65), 1e-10 * r.u(0.5, 2), 0.01 * r.u(0.5, 2),
              0.005 * r.u(0.5, 2)};
        Vec dx = randv(r, 9), yb = randv(r, 5);
        for (int k = 0; k < 9; ++k) dx[k] *= fabs(x[k]) + (k < 5 ? 1e-3 : 0.0);
        if (still) { dx[1] = 0.0; dx[2] = 0.0; }
        dclaw_params P = P0;
        P.kref = x[6]; P.alpha_c = x[7]; P.mu = x[8];
        double qb[5] = {yb[0], yb[1], yb[2], yb[3], yb[4]};
        double phib = 0.0, pbar[NPB] = {0, 0, 0, 0};
        src2_cell_b(P, x[5], dt, &x[0], qb, phib, pbar);
        double ad = phib * dx[5] + pbar[PB_KREF] * dx[6] + pbar[PB_ALPHA] * dx[7] + pbar[PB_MU] * dx[8];
        for (int k = 0; k < 5; ++k) ad += qb[k] * dx[k];
        st.add(dircheck(f, x, dx, yb, ad));
    }
    return st;
}

}  // namespace

extern "C" {

// which: 0 qfix, 1 qfix_cmass, 2 setvars, 3 setvars<all>, 4 setvars<all> alphamethod 1,
// 5 riemanntype, 6 riemann wet, 7 riemann dry side / wall, 8 riemann at rest, 9 riemann src2method -1,
// 10..13 limiter 1..4, 14 rpt2, 15 src2 m0, 16 src2 m1, 17 src2 m-1, 18 src2 at rest,
// 19 src2 with Manning friction, 20 with depth-dependent Manning friction
int adj_check_local(int which, int seed, int n, double* maxerr, int* skipped) {
    Rng r((uint64_t)seed * 7919u + (uint64_t)which);
    Stat st;
    switch (which) {
        case 0: st = check_qfix(r, n); break;
        case 1: st = check_qfix_cmass(r, n); break;
        case 2: st = check_setvars<false>(r, n, 0); break;
        case 3: st = check_setvars<true>(r, n, 0); break;
        case 4: st = check_setvars<true>(r, n, 1); break;
        case 5: st = check_riemanntype(r, n); break;
        case 6: st = check_riemann(r, n, 0); break;
        case 7: st = check_riemann(r, n, 1); break;
        case 8: st = check_riemann(r, n, 2); break;
        case 9: st = check_riemann(r, n, 3); break;
        case 10: case 11: case 12: case 13: st = check_limiter(r, n, which - 9); break;
        case 14: st = check_rpt2(r, n); break;
        case 15: st = check_src2(r, n, 0, false); break;
        case 16: st = check_src2(r, n, 1, false); break;
        case 17: st = check_src2(r, n, -1, false); break;
        case 18: st = check_src2(r, n, 0, true); break;
        case 19: st = check_src2(r, n, 0, false, 1); break;
        case 20: st = check_src2(r, n, 0, false, 2); break;
        case 21: st = check_riemann(r, n, 4); break;
        default: return -1;
    }
    *maxerr = st.maxerr;
    *skipped = st.skipped;
    return st.n;
}

// ---- whole step --------------------------------------------------------------
struct HostWork {
    std::vector<double> qB, bP, td, wx, wy, fx, fy;
    Work W;
    HostWork(int mx, int my) {
        size_t npad = (size_t)(mx + 4) * (my + 4), nxi = (size_t)(mx + 3) * (my + 2),
               nyi = (size_t)(my + 3) * (mx + 2);
        qB.assign(5 * npad, 0.0); bP.assign(npad, 0.0); td.assign(3 * npad, 0.0);
        wx.assign(NW * nxi, 0.0); wy.assign(NW * nyi, 0.0); fx.assign(NF * nxi, 0.0); fy.assign(NF * nyi, 0.0);
        W = Work{qB.data(), bP.data(), td.data(), wx.data(), wy.data(), fx.data(), fy.data(), npad, nxi, nyi};
    }
};

static void forward_stages(const dclaw_params& P, const Geom& g, const double* q, const double* b, HostWork& H,
                           double dt) {
    const int mx = g.mx, my = g.my;
    Work& W = H.W;
    for (int j = -1; j <= my + 2; ++j)
        for (int i = -1; i <= mx + 2; ++i) stage_b4(P, g, q, b, W, i, j);
    for (int j = -1; j <= my + 2; ++j)
        for (int i = -1; i <= mx + 2; ++i) stage_taudir(P, g, W, i, j);
    for (int r = 0; r <= my + 1; ++r)
        for (int i = 0; i <= mx + 2; ++i) stage_riemann<0>(P, g, W, r, i, nullptr);
    for (int k = 0; k <= my + 2; ++k)
        for (int c = 0; c <= mx + 1; ++c) stage_riemann<1>(P, g, W, c, k, nullptr);
    for (int r = 0; r <= my + 1; ++r)
        for (int i = 1; i <= mx + 1; ++i) stage_flux<0>(P, g, W, r, i, dt / g.dx, nullptr);
    for (int k = 1; k <= my + 1; ++k)
        for (int c = 0; c <= mx + 1; ++c) stage_flux<1>(P, g, W, c, k, dt / g.dy, nullptr);
}

// one step at fixed dt (no tick), q_out = S(q)
int adj_step_fwd(const dclaw_params* P, int mx, int my, double dx, double dy, const double* q, const double* b,
                 double dt, double* q_out) {
    Geom g{mx, my, mx + 4, my + 4, dx, dy};
    HostWork H(mx, my);
    forward_stages(*P, g, q, b, H, dt);
    int st = 0;
    for (int j = 1; j <= my; ++j)
        for (int i = 1; i <= mx; ++i)
            if (stage_finalize(*P, g, H.W, q_out, i, j, dt)) st = 1;
    return st;
}

// adjoint of one step: lam_in = (dS/dq)^T lam_out, pbar += (dS/dtheta)^T lam_out
int adj_step_vjp(const dclaw_params* P, int mx, int my, double dx, double dy, const double* q, const double* b,
                 double dt, const double* lam_out, double* lam_in, double* pbar, double* bbar) {
    Geom g{mx, my, mx + 4, my + 4, dx, dy};
    HostWork H(mx, my);
    forward_stages(*P, g, q, b, H, dt);
    const Work& W = H.W;
    std::vector<double> lamq(5 * (size_t)mx * my), xfb(NFB * W.nxi), yfb(NFB * W.nyi), xcb(NCB * W.nxi),
        ycb(NCB * W.nyi), tdq(NTD * W.npad), qsb(NQSB * W.npad), sv(NSV * W.npad);
    AdjWork A{lamq.data(), xfb.data(), yfb.data(), xcb.data(), ycb.data(), tdq.data(), qsb.data(), sv.data()};
    A.bed = bbar != nullptr;
    for (int j = -1; j <= my + 2; ++j)
        for (int i = -1; i <= mx + 2; ++i) adj_item_svrec(*P, g, W, A, i, j);
    for (int j = 1; j <= my; ++j)
        for (int i = 1; i <= mx; ++i) adj_item_src2(*P, g, W, A, lam_out, i, j, dt, pbar);
    for (int r = 0; r <= my + 1; ++r)
        for (int i = 1; i <= mx + 1; ++i) adj_item_flux<0>(*P, g, W, A, r, i, dt);
    for (int k = 1; k <= my + 1; ++k)
        for (int c = 0; c <= mx + 1; ++c) adj_item_flux<1>(*P, g, W, A, c, k, dt);
    int ok = 1;
    for (int r = 0; r <= my + 1; ++r)
        for (int i = 0; i <= mx + 2; ++i) ok &= adj_item_riemann<0>(*P, g, W, A, r, i, pbar) ? 1 : 0;
    for (int k = 0; k <= my + 2; ++k)
        for (int c = 0; c <= mx + 1; ++c) ok &= adj_item_riemann<1>(*P, g, W, A, c, k, pbar) ? 1 : 0;
    for (int j = -1; j <= my + 2; ++j)
        for (int i = -1; i <= mx + 2; ++i) adj_item_taudir(*P, g, W, A, i, j, pbar);
    for (int j = -1; j <= my + 2; ++j)
        for (int i = -1; i <= mx + 2; ++i) adj_item_b4(*P, g, W, A, q, i, j);
    for (int j = 1; j <= my; ++j)
        for (int i = 1; i <= mx; ++i) adj_item_gather(*P, g, A, W, lam_in, i, j);
    if (bbar)
        for (int j = 1; j <= my; ++j)
            for (int i = 1; i <= mx; ++i) adj_item_gather_bed(g, A, W, bbar, i, j);
    return ok ? 0 : 2;
}

}  // extern "C"
