// emu_step.cpp -- TEST INFRASTRUCTURE: runs the CUDA step's stage functions
// (dclaw_b200/csrc/stages.cuh) on the host, in the kernels' launch order, so
// that the CPU test suite can check the device arithmetic against the oracle
// bit for bit (both sides use glibc libm and no FMA contraction here; on the
// GPU only CUDA's exp/atan/tan/tanh differ). This is not a product path.
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <vector>
#include "../../dclaw_b200/csrc/full_state.cuh"
#include "../../dclaw_b200/csrc/stages.cuh"
#include "../../dclaw_b200/csrc/tile.cuh"

using namespace dclaw;

extern "C" int emu_run(const dclaw_params* P, int mx, int my, double dx, double dy, double* q, const double* b,
                       int nsteps, double dt_initial, double t_final, int fixed_dt, double* dt_hist,
                       double* cfl_hist, uint32_t* brlog, double* t_out) {
    Geom g{mx, my, mx + 4, my + 4, dx, dy};
    size_t npad = (size_t)(mx + 4) * (my + 4), nxi = (size_t)(mx + 3) * (my + 2), nyi = (size_t)(my + 3) * (mx + 2);
    std::vector<double> qB(5 * npad), bP(npad), td(3 * npad), wx(NW * nxi), wy(NW * nyi), fx(NF * nxi), fy(NF * nyi);
    Work W{qB.data(), bP.data(), td.data(), wx.data(), wy.data(), fx.data(), fy.data(), npad, nxi, nyi};
    std::vector<double> qa(q, q + 5 * (size_t)mx * my), qb(5 * (size_t)mx * my);
    double t = 0.0, dt = t_final > 0.0 ? fmax2(fmin2(dt_initial, t_final), 0.0) : dt_initial;
    int status = 0;
    for (int n = 0; n < nsteps; ++n) {
        const bool last = n == nsteps - 1;
        uint32_t* br = (last && brlog) ? brlog : nullptr;
        for (int j = -1; j <= my + 2; ++j)
            for (int i = -1; i <= mx + 2; ++i)
                if (stage_b4(*P, g, qa.data(), b, W, i, j)) status = DCLAW_ERR_NAN;
        if (status) break;
        for (int j = -1; j <= my + 2; ++j)
            for (int i = -1; i <= mx + 2; ++i) stage_taudir(*P, g, W, i, j);
        double cfl = 0.0;
        for (int r = 0; r <= my + 1; ++r)
            for (int i = 0; i <= mx + 2; ++i) {
                uint32_t bits = 0;
                double s = stage_riemann<0>(*P, g, W, r, i, &bits);
                if (i >= 1 && i <= mx + 1) {
                    cfl = fmax2(cfl, (dt / dx) * s);
                    if (br) br[(size_t)r * (mx + 1) + (i - 1)] = bits;
                }
            }
        for (int c = 0; c <= mx + 1; ++c)
            for (int k = 0; k <= my + 2; ++k) {
                uint32_t bits = 0;
                double s = stage_riemann<1>(*P, g, W, c, k, &bits);
                if (k >= 1 && k <= my + 1) {
                    cfl = fmax2(cfl, (dt / dy) * s);
                    if (br) br[(size_t)(my + 2) * (mx + 1) + (size_t)c * (my + 1) + (k - 1)] = bits;
                }
            }
        for (int r = 0; r <= my + 1; ++r)
            for (int i = 1; i <= mx + 1; ++i) {
                uint32_t bits = 0;
                stage_flux<0>(*P, g, W, r, i, dt / dx, br ? &bits : nullptr);
                if (br) br[(size_t)r * (mx + 1) + (i - 1)] |= bits;
            }
        for (int c = 0; c <= mx + 1; ++c)
            for (int k = 1; k <= my + 1; ++k) {
                uint32_t bits = 0;
                stage_flux<1>(*P, g, W, c, k, dt / dy, br ? &bits : nullptr);
                if (br) br[(size_t)(my + 2) * (mx + 1) + (size_t)c * (my + 1) + (k - 1)] |= bits;
            }
        for (int j = 1; j <= my; ++j)
            for (int i = 1; i <= mx; ++i)
                if (stage_finalize(*P, g, W, qb.data(), i, j, dt)) status = DCLAW_ERR_NAN;
        qa.swap(qb);
        if (dt_hist) dt_hist[n] = dt;
        if (cfl_hist) cfl_hist[n] = cfl;
        t = t + dt;
        double dtn = fixed_dt ? dt : tick_next_dt(*P, dt, cfl);
        if (t_final > 0.0) dtn = fmax2(fmin2(dtn, t_final - t), 0.0);
        dt = dtn;
        if (status) break;
    }
    memcpy(q, qa.data(), sizeof(double) * 5 * (size_t)mx * my);
    if (t_out) *t_out = t;
    return status;
}

// The fused two-kernel step (tile.cuh): K1 records, then every tile's phases
// in the kernel's order with host buffers standing in for shared memory.
template <int TX, int TY>
static int run_fused(const dclaw_params* P, int mx, int my, double dx, double dy, double* q, const double* b,
                     int nsteps, double dt_initial, double t_final, int fixed_dt, double* dt_hist,
                     double* cfl_hist, uint32_t* brlog, double* t_out, bool src2_in_tile) {
    using TG = TileGeom<TX, TY>;
    Geom g{mx, my, mx + 4, my + 4, dx, dy};
    size_t npad = (size_t)(mx + 4) * (my + 4);
    std::vector<double> rec(NREC * npad), sm(TG::SMEM_DOUBLES);
    std::vector<uint32_t> bits(TG::NA);
    Rec R{rec.data(), npad};
    TileMem M;
    M.A = sm.data();
    M.B = M.A + (size_t)NW * TG::NA;
    M.C = M.B + (size_t)10 * TG::NB;
    M.D = M.C + (size_t)10 * TG::NC;
    M.H = M.D + (size_t)10 * TG::ND;
    M.Bd = M.H + TG::NHB;
    M.T5 = M.Bd + TG::NHB;
    M.bits = bits.data();
    M.NA = TG::NA;
    M.hw = TG::HW;
    M.hv = TX + 6;
    std::vector<double> qa(q, q + 5 * (size_t)mx * my), qb(5 * (size_t)mx * my), qs(5 * (size_t)mx * my);
    double t = 0.0, dt = t_final > 0.0 ? fmax2(fmin2(dt_initial, t_final), 0.0) : dt_initial;
    int status = 0;
    const size_t nlog = (size_t)(my + 2) * (mx + 1) + (size_t)(mx + 2) * (my + 1);
    for (int n = 0; n < nsteps; ++n) {
        uint32_t* br = (n == nsteps - 1 && brlog) ? brlog : nullptr;
        if (br) memset(br, 0, nlog * sizeof(uint32_t));
        for (int j = -1; j <= my + 2; ++j)
            for (int i = -1; i <= mx + 2; ++i)
                if (cell_record(*P, g, qa.data(), b, R, i, j)) status = DCLAW_ERR_NAN;
        if (status) break;
        double cfl = 0.0;
        const double dtdx = dt / dx, dtdy = dt / dy;
        for (int ty = 0; ty < (my + TY - 1) / TY; ++ty)
            for (int tx = 0; tx < (mx + TX - 1) / TX; ++tx) {
                const int i0 = 1 + tx * TX, j0 = 1 + ty * TY;
                M.hi0 = i0 - 3;
                M.hj0 = j0 - 3;
                for (int it = 0; it < TG::NHB; ++it) tile_stage_hb(g, R, b, M, it);
                for (int dir = 0; dir < 2; ++dir) {
                    const int nsolve = dir == 0 ? TG::NXW : TG::NYW;
                    const double dtd = dir == 0 ? dtdx : dtdy;
                    for (int it = 0; it < nsolve; ++it) {
                        bool ok;
                        double s = tile_riemann(*P, g, R, M, dir, it, i0, j0, TX, TY, ok);
                        if (ok) cfl = fmax2(cfl, dtd * s);
                    }
                    // the kernels' flux phase: for slices up to 15 cells
                    // (x: TX + 1 <= 16, y: TY + 1 <= 16, and a half-warp per
                    // slice within 256 threads) each interface is limited
                    // once and a cell is given its own and its next
                    // interface's results
                    const bool pair = dir == 0 ? (TX + 1 <= 16 && (TY + 2) * 16 <= 256)
                                               : (TY + 1 <= 16 && (TX + 2) * 16 <= 256);
                    if (pair) {
                        const int nsl = dir == 0 ? TY + 2 : TX + 2, span = dir == 0 ? TX : TY;
                        const int smax = dir == 0 ? my + 1 : mx + 1, amax = dir == 0 ? mx : my;
                        for (int sl = 0; sl < nsl; ++sl) {
                            const int s = (dir == 0 ? j0 : i0) - 1 + sl, a0 = dir == 0 ? i0 : j0;
                            if (s < 0 || s > smax) continue;
                            std::vector<double> v(16 * 15, 0.0);
                            std::vector<uint32_t> lb(16, 0u);
                            for (int k = 0; k <= span && a0 + k <= amax + 1; ++k) {
                                if (dir == 0) tile_x_iface<TX, TY>(*P, M, s, a0 + k, i0, j0, dtd, &v[15 * k], br ? &lb[k] : nullptr);
                                else tile_y_iface<TX, TY>(*P, M, s, a0 + k, i0, j0, dtd, &v[15 * k], br ? &lb[k] : nullptr);
                            }
                            for (int k = 0; k < span && a0 + k <= amax; ++k) {
                                const int c = dir == 0 ? a0 + k : s, r = dir == 0 ? s : a0 + k;
                                tile_flux_cell<TX, TY>(*P, g, R, M, dir, c, r, i0, j0, dtd, &v[15 * k],
                                                       &v[15 * (k + 1)], lb[k], lb[k + 1], br);
                            }
                        }
                    } else {
                        const int ncell = dir == 0 ? (TY + 2) * TX : TY * (TX + 2);
                        for (int it = 0; it < ncell; ++it) tile_flux<TX, TY>(*P, g, R, M, dir, it, i0, j0, dtd, br);
                    }
                    if (dir == 0) {
                        std::vector<double> T((size_t)(TY + 1) * TX * 5);
                        std::vector<char> v((size_t)(TY + 1) * TX);
                        for (int it = 0; it < (TY + 1) * TX; ++it) v[it] = tile_T<TX, TY>(g, M, it, i0, j0, &T[5 * it]);
                        for (int it = 0; it < (TY + 1) * TX; ++it)
                            if (v[it]) tile_T_store<TX, TY>(M, it, &T[5 * it]);
                    }
                }
                for (int it = 0; it < TX * TY; ++it) {
                    bool nan = src2_in_tile ? tile_final<TX, TY, true>(*P, g, R, M, it, i0, j0, dt, qb.data())
                                            : tile_final<TX, TY, false>(*P, g, R, M, it, i0, j0, dt, qs.data());
                    if (nan) status = DCLAW_ERR_NAN;
                }
            }
        if (!src2_in_tile)
            for (size_t c = 0; c < (size_t)mx * my; ++c) cell_src2(*P, g, dt, qs.data(), qb.data(), c);
        qa.swap(qb);
        if (dt_hist) dt_hist[n] = dt;
        if (cfl_hist) cfl_hist[n] = cfl;
        t = t + dt;
        double dtn = fixed_dt ? dt : tick_next_dt(*P, dt, cfl);
        if (t_final > 0.0) dtn = fmax2(fmin2(dtn, t_final - t), 0.0);
        dt = dtn;
        if (status) break;
    }
    memcpy(q, qa.data(), sizeof(double) * 5 * (size_t)mx * my);
    if (t_out) *t_out = t;
    return status;
}

extern "C" int emu_run_fused(const dclaw_params* P, int mx, int my, double dx, double dy, double* q, const double* b,
                             int nsteps, double dt_initial, double t_final, int fixed_dt, double* dt_hist,
                             double* cfl_hist, uint32_t* brlog, double* t_out, int tx, int ty, int src2_in_tile) {
#define DCLAW_EMU_TILE(X, Y)                                                                              \
    if (tx == X && ty == Y)                                                                              \
        return run_fused<X, Y>(P, mx, my, dx, dy, q, b, nsteps, dt_initial, t_final, fixed_dt, dt_hist, \
                               cfl_hist, brlog, t_out, src2_in_tile != 0);
    DCLAW_EMU_TILE(16, 16)
    DCLAW_EMU_TILE(16, 14)
    DCLAW_EMU_TILE(13, 14)
    DCLAW_EMU_TILE(14, 13)
    DCLAW_EMU_TILE(8, 8)
    return -1;
}

// The full-state step (full_state.cuh) in the kernels' launch order.
extern "C" int emu_run_full(const dclaw_params* P, int mx, int my, double dx, double dy, double* q, const double* b,
                            const double* he, int nsteps, double dt_initial, double* dt_hist, double* cfl_hist,
                            uint32_t* brlog) {
    Geom g{mx, my, mx + 4, my + 4, dx, dy};
    const FullLayout L = full_layout(mx, my);
    std::vector<unsigned char> mem(L.total);
    WorkF W = make_work_full(mem.data(), L);
    const size_t nq = (size_t)NQF * mx * my;
    std::vector<double> qa(q, q + nq), qb(nq);
    double dt = dt_initial;
    int status = 0;
    for (int n = 0; n < nsteps; ++n) {
        uint32_t* br = (n == nsteps - 1 && brlog) ? brlog : nullptr;
        for (int j = -1; j <= my + 2; ++j)
            for (int i = -1; i <= mx + 2; ++i)
                if (full_b4(*P, g, qa.data(), b, W, i, j)) status = DCLAW_ERR_NAN;
        if (status) break;
        for (int j = -1; j <= my + 2; ++j)
            for (int i = -1; i <= mx + 2; ++i) full_taudir(*P, g, W, i, j);
        double cfl = 0.0;
        for (int r = 0; r <= my + 1; ++r)
            for (int i = 0; i <= mx + 2; ++i) {
                uint32_t bits = 0;
                double s = full_riemann<0>(*P, g, W, r, i, &bits);
                if (i >= 1 && i <= mx + 1) {
                    cfl = fmax2(cfl, (dt / dx) * s);
                    if (br) br[(size_t)r * (mx + 1) + (i - 1)] = bits;
                }
            }
        for (int c = 0; c <= mx + 1; ++c)
            for (int k = 0; k <= my + 2; ++k) {
                uint32_t bits = 0;
                double s = full_riemann<1>(*P, g, W, c, k, &bits);
                if (k >= 1 && k <= my + 1) {
                    cfl = fmax2(cfl, (dt / dy) * s);
                    if (br) br[(size_t)(my + 2) * (mx + 1) + (size_t)c * (my + 1) + (k - 1)] = bits;
                }
            }
        for (int r = 0; r <= my + 1; ++r)
            for (int i = 1; i <= mx + 1; ++i) {
                uint32_t bits = 0;
                full_flux<0>(*P, g, W, r, i, dt / dx, br ? &bits : nullptr);
                if (br) br[(size_t)r * (mx + 1) + (i - 1)] |= bits;
            }
        for (int c = 0; c <= mx + 1; ++c)
            for (int k = 1; k <= my + 1; ++k) {
                uint32_t bits = 0;
                full_flux<1>(*P, g, W, c, k, dt / dy, br ? &bits : nullptr);
                if (br) br[(size_t)(my + 2) * (mx + 1) + (size_t)c * (my + 1) + (k - 1)] |= bits;
            }
        for (int j = 1; j <= my; ++j)
            for (int i = 1; i <= mx; ++i)
                if (full_finalize(*P, g, W, he, qb.data(), i, j, dt)) status = DCLAW_ERR_NAN;
        qa.swap(qb);
        if (dt_hist) dt_hist[n] = dt;
        if (cfl_hist) cfl_hist[n] = cfl;
        dt = tick_next_dt(*P, dt, cfl);
        if (status) break;
    }
    memcpy(q, qa.data(), sizeof(double) * nq);
    return status;
}
