// kernels.cu -- CUDA kernels (sm_100a, FP64) and the C ABI of include/dclaw_b200.h.
//
// One launch per stage of stages.cuh, all on the caller's stream, all
// reading dt from the device-resident clock so that a sequence of steps can
// be captured in a CUDA graph. The Courant number is max-reduced with warp
// shuffles, one shared-memory pass per block and one 64-bit atomicMax per
// block on the order-preserving bit pattern of a non-negative double.
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <atomic>
#include <mutex>

#include "full_state.cuh"
#include "stages.cuh"
#include "tile.cuh"
#include "workspace.cuh"

namespace dclaw {

constexpr int TPB = 256;
// threads per CTA of the single-patch tile kernel
#ifndef DCLAW_TILE_TPB
#define DCLAW_TILE_TPB 256
#endif
constexpr int TILE_TPB = DCLAW_TILE_TPB;
constexpr int MAX_DEVICES = 64;
// One-time per-device set-up (function attributes, the SM count, symbol
// addresses) is filled under this lock and published through atomics, so
// host threads making their first calls on a device at the same time do not
// race on the caches.
static std::mutex g_setup_mu;
// tile of the fused step: with 14 x 13 the solves of each sweep fit in one
// round of 256 threads (255 and 256 interfaces), and the flux phases' half-
// warp per slice does too (15 rows, 16 columns). Before the flux phases
// exchanged interfaces between lanes, 14 x 13 stepped the 4096^2 random
// field 2 % faster than 16 x 14 (whose solves take two rounds) and 7 %
// faster than 12 x 14.
#ifndef DCLAW_TILE_X
#define DCLAW_TILE_X 14
#endif
#ifndef DCLAW_TILE_Y
#define DCLAW_TILE_Y 13
#endif
// resident tile CTAs per SM the register allocation is sized for
#ifndef DCLAW_TILE_MINBLOCKS
#define DCLAW_TILE_MINBLOCKS 2
#endif
// src2 in its own per-cell kernel (1) or as the tile kernel's last phase (0)
#ifndef DCLAW_SRC2_KERNEL
#define DCLAW_SRC2_KERNEL 1
#endif
// the same choice for the step over tile lists: k_src2_list (1), or src2 and
// the tick in k_tile_list (0)
#ifndef DCLAW_LIST_SRC2_KERNEL
#define DCLAW_LIST_SRC2_KERNEL 1
#endif
// and for the ensemble step: k_src2_batch (1), or src2 in k_tile_batch (0)
#ifndef DCLAW_BATCH_SRC2_KERNEL
#define DCLAW_BATCH_SRC2_KERNEL 1
#endif
constexpr int TILE_X = DCLAW_TILE_X, TILE_Y = DCLAW_TILE_Y;
// resident blocks per SM the ensemble's streaming scan is sized for
#ifndef DCLAW_SCAN_MINB
#define DCLAW_SCAN_MINB 4
#endif
// resident blocks per SM the ensemble's per-cell kernels (records of the
// listed tiles, src2) are sized for
#ifndef DCLAW_CELL_MINB
#define DCLAW_CELL_MINB 4
#endif
// threads per CTA of those two (one tile's cells per CTA pass), with the
// register budget of DCLAW_CELL_MINB blocks of 256 threads. 192 (as the
// single patch's) measured 3 % slower on the 256-flume ensemble.
#ifndef DCLAW_BATCH_CELL_TPB
#define DCLAW_BATCH_CELL_TPB 256
#endif
constexpr int BATCH_CELL_TPB = DCLAW_BATCH_CELL_TPB;
constexpr int BATCH_CELL_MINB = DCLAW_CELL_MINB * 256 / DCLAW_BATCH_CELL_TPB;
// resident blocks per SM the single-patch per-cell kernels (k_records,
// k_src2_cells) are sized for: on the 4096^2 random field 6 (40 registers,
// with spills) steps 1.9 % faster than 4 (64 registers), 5 1.2 % and 8
// (32 registers) 0.8 %; 3 and 2 (80 and 110 registers, no spills) 4 % and
// 10 % slower. The ensemble's per-cell kernels are fastest at 4 (6 is 5 %
// slower there).
#ifndef DCLAW_PLAIN_CELL_MINB
#define DCLAW_PLAIN_CELL_MINB 6
#endif
// threads per CTA of k_src2_list and k_src2_cells (the register budget is
// that of DCLAW_PLAIN_CELL_MINB blocks of 256 threads whatever the CTA
// size). k_src2_list gives each CTA one tile's 14 x 13 = 182 cells per
// pass, which 192 threads cover in six warps (256 left two warps idle):
// with the records likewise the step takes 3.87 ms on the 4096^2 field
// against 3.96 ms at 256, with the same bits.
#ifndef DCLAW_SRC2_TPB
#define DCLAW_SRC2_TPB 192
#endif
constexpr int SRC2_TPB = DCLAW_SRC2_TPB;
constexpr int SRC2_MINB = DCLAW_PLAIN_CELL_MINB * 256 / DCLAW_SRC2_TPB;
// threads per CTA of k_records_list (one tile's records per CTA pass, 182
// for an interior tile), with the register budget of DCLAW_PLAIN_CELL_MINB
// blocks of 256 threads
#ifndef DCLAW_RECORDS_TPB
#define DCLAW_RECORDS_TPB 192
#endif
constexpr int RECORDS_TPB = DCLAW_RECORDS_TPB;
constexpr int RECORDS_MINB = DCLAW_PLAIN_CELL_MINB * 256 / DCLAW_RECORDS_TPB;

__device__ __forceinline__ double warp_max(double v) {
    for (int o = 16; o > 0; o >>= 1) {
        double w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w > v ? w : v;
    }
    return v;
}

// block-wide max of a non-negative value into *acc (bit pattern of a double)
__device__ __forceinline__ void block_max_to(double v, unsigned long long* acc) {
    __shared__ double red[32];
    v = warp_max(v);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) red[wid] = v;
    __syncthreads();
    if (wid == 0) {
        double x = lane < (int)(blockDim.x >> 5) ? red[lane] : 0.0;
        x = warp_max(x);
        if (lane == 0 && x > 0.0) atomicMax(acc, (unsigned long long)__double_as_longlong(x));
    }
}

__device__ __forceinline__ void flag_status(dclaw_clock* clk, int code) { atomicCAS(&clk->status, 0, code); }

// column and row of a flat index over rows of width w, in 32-bit arithmetic
// when the index fits (a 64-bit division is a long instruction sequence,
// a large share of a per-cell kernel's issue slots)
__device__ __forceinline__ void split_index(long long idx, int w, int& col, int& row) {
    if (idx <= 0xffffffffLL) {
        const unsigned u = (unsigned)idx, q = u / (unsigned)w;
        row = (int)q;
        col = (int)(u - q * (unsigned)w);
    } else {
        row = (int)(idx / w);
        col = (int)(idx - (long long)row * w);
    }
}

// ---- tile activity flags ------------------------------------------------------
// A tile is active in a step when a cell within distance 3 of it is wet after
// b4step2 (the cells whose records the tile reads). k_records writes the
// step's number into the flag of every tile a wet padded cell makes active;
// a tile whose flag holds another number has only dry-dry interfaces and
// dry cells, so the tile kernel skips it and src2 writes its cells' zeros.
// Stale numbers from earlier runs can only mark a dry tile active, which
// costs time and changes no result.
__device__ __forceinline__ int fdiv(int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }

__device__ __forceinline__ void mark_tiles(uint32_t* __restrict__ tflag, uint32_t epoch, int i, int j, int TX, int TY,
                                           int ntx, int nty) {
    // tile t covers i0 = 1 + t TX .. i0 + TX - 1 and reads i0 - 3 .. i0 + TX + 2
    int x0 = fdiv(i - TX - 3 + TX - 1, TX), x1 = fdiv(i + 2, TX);
    int y0 = fdiv(j - TY - 3 + TY - 1, TY), y1 = fdiv(j + 2, TY);
    if (x0 < 0) x0 = 0;
    if (y0 < 0) y0 = 0;
    if (x1 > ntx - 1) x1 = ntx - 1;
    if (y1 > nty - 1) y1 = nty - 1;
    for (int ty = y0; ty <= y1; ++ty)
        for (int tx = x0; tx <= x1; ++tx) tflag[ty * ntx + tx] = epoch;
}

// The records in two passes. A wet padded cell is a ghost copy of a wet
// interior cell within 2 of the edge (mirror or copy), and every tile whose
// read range holds the ghost also holds its source, so the interior cells'
// marks are all the marks. Pass 1 (the scan) reads every interior cell's
// five fields -- the NaN check -- and marks; pass 2 builds the records of
// the padded cells an active tile reads, and no others: far from the flow
// a cell costs its 40 bytes of state and nothing more.
// a cell's column and row are only worked out when it is wet (the marks);
// a dry cell costs its five loads and the NaN test
__device__ __forceinline__ bool scan_cell(const dclaw_params& P, const double* __restrict__ q, size_t plane,
                                          size_t c, int mx, uint32_t* __restrict__ tflag, const dclaw_clock* clk,
                                          int TX, int TY, int ntx, int nty) {
    const double h = q[c], hu = q[plane + c], hv = q[2 * plane + c], hm = q[3 * plane + c], pb = q[4 * plane + c];
    if (h > P.dry_tolerance) {
        int i, j;
        split_index((long long)c, mx, i, j);
        mark_tiles(tflag, clk->nsteps + 1u, i + 1, j + 1, TX, TY, ntx, nty);
    }
    return (h != h) || (hu != hu) || (hv != hv) || (hm != hm) || (pb != pb);
}

// Pass 2 of the records works tile by tile: a tile builds the records of
// the padded cells it owns -- its own cells, and the ghost cells beside it
// when it lies on the patch edge -- when it or one of its eight neighbours
// is active. A tile that reads a cell (within 3 of it) is the cell's owner
// or a neighbour of the owner (tiles are wider than 3), so every record an
// active tile reads is built, once.
__device__ __forceinline__ bool near_active(const uint32_t* __restrict__ tflag, uint32_t epoch, int tx, int ty,
                                            int ntx, int nty) {
    bool act = false;
    for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
            const int x = tx + dx, y = ty + dy;
            if (x >= 0 && y >= 0 && x < ntx && y < nty) act |= tflag[y * ntx + x] == epoch;
        }
    return act;
}

// the records of the cells tile (tx, ty) owns (all threads of the CTA)
template <int TX, int TY>
__device__ __forceinline__ void tile_records(const dclaw_params& P, const Geom& g, const double* __restrict__ q_in,
                                             const double* __restrict__ b, const Rec& R, int tx, int ty, int ntx,
                                             int nty) {
    const int i0 = 1 + tx * TX, j0 = 1 + ty * TY;
    const int xa = tx == 0 ? -1 : i0, xb = tx == ntx - 1 ? g.mx + 2 : i0 + TX - 1;
    const int ya = ty == 0 ? -1 : j0, yb = ty == nty - 1 ? g.my + 2 : j0 + TY - 1;
    const int w = xb - xa + 1, n = w * (yb - ya + 1);
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const int r = k / w;
        cell_record(P, g, q_in, b, R, xa + (k - r * w), ya + r);
    }
}

__device__ __forceinline__ bool tile_active(const uint32_t* __restrict__ tflag, uint32_t epoch, int i, int j, int TX,
                                            int TY, int ntx) {
    return !tflag || tflag[((j - 1) / TY) * ntx + (i - 1) / TX] == epoch;
}

// ---- fused step (interior layout) -----------------------------------------
__global__ void __launch_bounds__(TPB) k_b4(dclaw_params P, Geom g, const double* __restrict__ q_in,
                                            const double* __restrict__ b, Work W, dclaw_clock* clk) {
    const long long n = (long long)g.PX * g.PY;
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n) return;
    int i = (int)(idx % g.PX) - 1, j = (int)(idx / g.PX) - 1;
    if (stage_b4(P, g, q_in, b, W, i, j)) flag_status(clk, DCLAW_ERR_NAN);
}

__global__ void __launch_bounds__(TPB) k_taudir(dclaw_params P, Geom g, Work W, int inner_only) {
    const long long n = (long long)g.PX * g.PY;
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n) return;
    int i = (int)(idx % g.PX) - 1, j = (int)(idx / g.PX) - 1;
    if (inner_only && (i < 0 || j < 0 || i > g.mx + 1 || j > g.my + 1)) return;
    stage_taudir(P, g, W, i, j);
}

template <int DIR>
__global__ void __launch_bounds__(TPB) k_riemann(dclaw_params P, Geom g, Work W, dclaw_clock* clk,
                                                 uint32_t* __restrict__ brlog) {
    // DIR 0: rows r = 0..my+1, interfaces i = 0..mx+2 (x fastest)
    // DIR 1: interfaces k = 0..my+2, columns c = 0..mx+1 (column fastest)
    const int nfast = DIR == 0 ? g.mx + 3 : g.mx + 2;
    const int nslow = DIR == 0 ? g.my + 2 : g.my + 3;
    const long long n = (long long)nfast * nslow;
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double cflv = 0.0;
    if (idx < n) {
        int a = (int)(idx % nfast), s = (int)(idx / nfast);
        int r = DIR == 0 ? s : a;   // slice
        int i = DIR == 0 ? a : s;   // interface along the slice
        const int nlen = DIR == 0 ? g.mx : g.my;
        uint32_t bits = 0;
        double smax = stage_riemann<DIR>(P, g, W, r, i, &bits);
        if (i >= 1 && i <= nlen + 1) {
            const double dt = clk->dt;
            const double dtdx = DIR == 0 ? dt / g.dx : dt / g.dy;
            cflv = dtdx * smax;
            if (brlog) {
                size_t off = DIR == 0 ? (size_t)r * (g.mx + 1) + (size_t)(i - 1)
                                      : (size_t)(g.my + 2) * (g.mx + 1) + (size_t)r * (g.my + 1) + (size_t)(i - 1);
                brlog[off] = bits;
            }
        }
        if (!(cflv == cflv)) cflv = 0.0;
    }
    block_max_to(cflv, reinterpret_cast<unsigned long long*>(&clk->cfl_bits));
}

template <int DIR>
__global__ void __launch_bounds__(TPB) k_flux(dclaw_params P, Geom g, Work W, const dclaw_clock* clk,
                                              uint32_t* __restrict__ brlog) {
    // DIR 0: rows 0..my+1, interfaces 1..mx+1; DIR 1: interfaces 1..my+1, columns 0..mx+1
    const int nfast = DIR == 0 ? g.mx + 1 : g.mx + 2;
    const int nslow = DIR == 0 ? g.my + 2 : g.my + 1;
    const long long n = (long long)nfast * nslow;
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n) return;
    int a = (int)(idx % nfast), s = (int)(idx / nfast);
    int r = DIR == 0 ? s : a;
    int i = DIR == 0 ? a + 1 : s + 1;
    const double dt = clk->dt;
    const double dtdx = DIR == 0 ? dt / g.dx : dt / g.dy;
    uint32_t bits = 0;
    stage_flux<DIR>(P, g, W, r, i, dtdx, brlog ? &bits : nullptr);
    if (brlog) {
        size_t off = DIR == 0 ? (size_t)r * (g.mx + 1) + (size_t)(i - 1)
                              : (size_t)(g.my + 2) * (g.mx + 1) + (size_t)r * (g.my + 1) + (size_t)(i - 1);
        brlog[off] |= bits;
    }
}

__global__ void __launch_bounds__(TPB) k_final(dclaw_params P, Geom g, Work W, double* __restrict__ q_out,
                                               dclaw_clock* clk) {
    const long long n = (long long)g.mx * g.my;
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n) return;
    int i = (int)(idx % g.mx) + 1, j = (int)(idx / g.mx) + 1;
    if (stage_finalize(P, g, W, q_out, i, j, clk->dt)) flag_status(clk, DCLAW_ERR_NAN);
}

// ---- the full-state step (segregation, entrainment) -------------------------
// Without a branch log the stages after b4 skip what no active cell reads.
// A tile is active when a wet padded cell lies within 3 of its cells (the
// fused step's marks, step-numbered in tflag). A cell of an inactive tile
// has only dry cells within 3: every interface within 2 of it is dry-dry,
// so its waves and fluxes are exact zeros and its new state is zero with
// the eroded depth passed through, which the final stage writes without
// reading any flux. An interface's flux is read by the updates of the cells
// within one row (x) or column (y) of its two cells; its waves by its own
// flux and its two neighbours' along the slice. Each is computed when one
// of those readers is, so nothing skipped is ever read.
__device__ __forceinline__ bool full_any_active(const uint32_t* __restrict__ tflag, uint32_t epoch, const Geom& g,
                                                int ia, int ib, int ja, int jb) {
    ia = ia < 1 ? 1 : ia;
    ja = ja < 1 ? 1 : ja;
    ib = ib > g.mx ? g.mx : ib;
    jb = jb > g.my ? g.my : jb;
    if (ia > ib || ja > jb) return false;
    const int ntx = (g.mx + TILE_X - 1) / TILE_X;
    for (int ty = (ja - 1) / TILE_Y; ty <= (jb - 1) / TILE_Y; ++ty)
        for (int tx = (ia - 1) / TILE_X; tx <= (ib - 1) / TILE_X; ++tx)
            if (tflag[ty * ntx + tx] == epoch) return true;
    return false;
}

__global__ void __launch_bounds__(TPB) k_full_b4(dclaw_params P, Geom g, const double* __restrict__ q_in,
                                                 const double* __restrict__ b, WorkF W, dclaw_clock* clk,
                                                 uint32_t* __restrict__ tflag) {
    const long long n = (long long)g.PX * g.PY;
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n) return;
    int i = (int)(idx % g.PX) - 1, j = (int)(idx / g.PX) - 1;
    if (full_b4(P, g, q_in, b, W, i, j)) flag_status(clk, DCLAW_ERR_NAN);
    if (tflag && W.qB[pidx(g, i, j)] > 0.0)
        mark_tiles(tflag, clk->nsteps + 1u, i, j, TILE_X, TILE_Y, (g.mx + TILE_X - 1) / TILE_X,
                   (g.my + TILE_Y - 1) / TILE_Y);
}

__global__ void __launch_bounds__(TPB) k_full_taudir(dclaw_params P, Geom g, WorkF W) {
    const long long n = (long long)g.PX * g.PY;
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n) return;
    int i = (int)(idx % g.PX) - 1, j = (int)(idx / g.PX) - 1;
    full_taudir(P, g, W, i, j);
}

template <int DIR>
__global__ void __launch_bounds__(TPB) k_full_riemann(dclaw_params P, Geom g, WorkF W, dclaw_clock* clk,
                                                      uint32_t* __restrict__ brlog,
                                                      const uint32_t* __restrict__ tflag) {
    const int nfast = DIR == 0 ? g.mx + 3 : g.mx + 2;
    const int nslow = DIR == 0 ? g.my + 2 : g.my + 3;
    const long long n = (long long)nfast * nslow;
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double cflv = 0.0;
    if (idx < n) {
        int a = (int)(idx % nfast), s = (int)(idx / nfast);
        int r = DIR == 0 ? s : a;
        int i = DIR == 0 ? a : s;
        const int nlen = DIR == 0 ? g.mx : g.my;
        // read by the fluxes at i-1, i, i+1 of the slice: cells i-2..i+1 along
        // it, one slice either side (a skipped interface is dry-dry: no speed)
        const uint32_t ep = clk->nsteps + 1u;
        const bool need = !tflag || (DIR == 0 ? full_any_active(tflag, ep, g, i - 2, i + 1, r - 1, r + 1)
                                              : full_any_active(tflag, ep, g, r - 1, r + 1, i - 2, i + 1));
        if (need) {
            uint32_t bits = 0;
            double smax = full_riemann<DIR>(P, g, W, r, i, &bits);
            if (i >= 1 && i <= nlen + 1) {
                const double dt = clk->dt;
                const double dtdx = DIR == 0 ? dt / g.dx : dt / g.dy;
                cflv = dtdx * smax;
                if (brlog) {
                    size_t off = DIR == 0 ? (size_t)r * (g.mx + 1) + (size_t)(i - 1)
                                          : (size_t)(g.my + 2) * (g.mx + 1) + (size_t)r * (g.my + 1) + (size_t)(i - 1);
                    brlog[off] = bits;
                }
            }
            if (!(cflv == cflv)) cflv = 0.0;
        }
    }
    block_max_to(cflv, reinterpret_cast<unsigned long long*>(&clk->cfl_bits));
}

template <int DIR>
__global__ void __launch_bounds__(TPB) k_full_flux(dclaw_params P, Geom g, WorkF W, const dclaw_clock* clk,
                                                   uint32_t* __restrict__ brlog, const uint32_t* __restrict__ tflag) {
    const int nfast = DIR == 0 ? g.mx + 1 : g.mx + 2;
    const int nslow = DIR == 0 ? g.my + 2 : g.my + 1;
    const long long n = (long long)nfast * nslow;
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n) return;
    int a = (int)(idx % nfast), s = (int)(idx / nfast);
    int r = DIR == 0 ? s : a;
    int i = DIR == 0 ? a + 1 : s + 1;
    // read by the updates of cells i-1, i along the slice, one slice either side
    if (tflag) {
        const uint32_t ep = clk->nsteps + 1u;
        if (!(DIR == 0 ? full_any_active(tflag, ep, g, i - 1, i, r - 1, r + 1)
                       : full_any_active(tflag, ep, g, r - 1, r + 1, i - 1, i)))
            return;
    }
    const double dt = clk->dt;
    const double dtdx = DIR == 0 ? dt / g.dx : dt / g.dy;
    uint32_t bits = 0;
    full_flux<DIR>(P, g, W, r, i, dtdx, brlog ? &bits : nullptr);
    if (brlog) {
        size_t off = DIR == 0 ? (size_t)r * (g.mx + 1) + (size_t)(i - 1)
                              : (size_t)(g.my + 2) * (g.mx + 1) + (size_t)r * (g.my + 1) + (size_t)(i - 1);
        brlog[off] |= bits;
    }
}

__global__ void __launch_bounds__(TPB) k_full_final(dclaw_params P, Geom g, WorkF W, const double* __restrict__ he,
                                                    double* __restrict__ q_out, dclaw_clock* clk,
                                                    const uint32_t* __restrict__ tflag);

// the next dt after the tick rule's choice dtn: clipped at the next
// observation time (with the tick rule and t_obs > 0), then at t_final
__device__ __forceinline__ double clip_next_dt(const dclaw_clock* clk, double dtn) {
    if (!clk->fixed_dt && clk->t_obs > 0.0) {
        const double tn = (floor(clk->t / clk->t_obs + 1.0e-9) + 1.0) * clk->t_obs;
        dtn = fmin2(dtn, tn - clk->t);
    }
    if (clk->t_final > 0.0) dtn = fmax2(fmin2(dtn, clk->t_final - clk->t), 0.0);
    return dtn;
}

__global__ void k_tick(dclaw_params P, dclaw_clock* clk) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double cfl = __longlong_as_double((long long)clk->cfl_bits);
    double dt = clk->dt;
    clk->cfl = cfl;
    clk->dt_last = dt;
    clk->t = clk->t + dt;
    clk->nsteps = clk->nsteps + 1;
    clk->dt = clip_next_dt(clk, clk->fixed_dt ? dt : tick_next_dt(P, dt, cfl));
    clk->cfl_bits = 0ull;
}

__global__ void k_clock_init(dclaw_clock* clk, double t, double dt, double t_final, int fixed_dt) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    clk->t = t;
    clk->t_final = t_final;
    clk->dt = t_final > 0.0 ? fmax2(fmin2(dt, t_final - t), 0.0) : dt;
    clk->cfl = 0.0;
    clk->dt_last = 0.0;
    clk->cfl_bits = 0ull;
    clk->nsteps = 0;
    clk->blocks_done = 0;
    clk->status = 0;
    clk->fixed_dt = fixed_dt;
    clk->t_obs = 0.0;
}

__global__ void k_clock_set_obs(dclaw_clock* clk, double t_obs) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    clk->t_obs = t_obs;
    clk->dt = clip_next_dt(clk, clk->dt);
}

// ---- fused step: K1 cell records + K2 tiles --------------------------------
// Records of every padded cell, and the marks. prow0 / nprow: the padded
// rows (0 .. my+3 for j = -1 .. my+2) this launch covers, all of them by
// default.
__global__ void __launch_bounds__(TPB, DCLAW_PLAIN_CELL_MINB) k_records(dclaw_params P, Geom g, const double* __restrict__ q_in,
                                                 const double* __restrict__ b, Rec R, dclaw_clock* clk,
                                                 uint32_t* __restrict__ tflag, int prow0 = 0, int nprow = -1) {
    const long long n = (long long)g.PX * (nprow < 0 ? g.PY : nprow);
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n) return;
    int i, j;
    split_index(idx, g.PX, i, j);
    i -= 1;
    j += prow0 - 1;
    if (cell_record(P, g, q_in, b, R, i, j)) flag_status(clk, DCLAW_ERR_NAN);
    if (tflag && R.get(R_H, pidx(g, i, j)) > 0.0)
        mark_tiles(tflag, clk->nsteps + 1u, i, j, TILE_X, TILE_Y, (g.mx + TILE_X - 1) / TILE_X,
                   (g.my + TILE_Y - 1) / TILE_Y);
}

__device__ __forceinline__ void tick_device(const dclaw_params& P, dclaw_clock* clk) {
    double cfl = __longlong_as_double((long long)atomicAdd(reinterpret_cast<unsigned long long*>(&clk->cfl_bits), 0ull));
    double dt = clk->dt;
    clk->cfl = cfl;
    clk->dt_last = dt;
    clk->t = clk->t + dt;
    clk->nsteps = clk->nsteps + 1;
    clk->dt = clip_next_dt(clk, clk->fixed_dt ? dt : tick_next_dt(P, dt, cfl));
    clk->cfl_bits = 0ull;
    clk->blocks_done = 0u;
}

// the block finishing last (after its Courant-number atomic) runs the tick
__device__ __forceinline__ void last_block_tick(const dclaw_params& P, dclaw_clock* clk) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        unsigned int done = atomicAdd(&clk->blocks_done, 1u);
        if (done == gridDim.x * gridDim.y - 1) {
            __threadfence();
            tick_device(P, clk);
        }
    }
}

// update + src2 of the full state; the last block applies the tick
__global__ void __launch_bounds__(TPB) k_full_final(dclaw_params P, Geom g, WorkF W, const double* __restrict__ he,
                                                    double* __restrict__ q_out, dclaw_clock* clk,
                                                    const uint32_t* __restrict__ tflag) {
    const long long n = (long long)g.mx * g.my;
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx < n) {
        int i = (int)(idx % g.mx) + 1, j = (int)(idx / g.mx) + 1;
        if (tflag && !full_any_active(tflag, clk->nsteps + 1u, g, i, i, j, j)) {
            // a cell of an inactive tile: zero, its eroded depth passed through
            const size_t plane = (size_t)g.mx * g.my;
            for (int f = 0; f < F_BDIF; ++f) q_out[(size_t)f * plane + (size_t)idx] = 0.0;
            q_out[(size_t)F_BDIF * plane + (size_t)idx] = W.qB[(size_t)F_BDIF * W.npad + pidx(g, i, j)];
        } else if (full_finalize(P, g, W, he, q_out, i, j, clk->dt)) {
            flag_status(clk, DCLAW_ERR_NAN);
        }
    }
    last_block_tick(P, clk);
}

// One tile of the fused step (all threads of the CTA call it). smem holds
// TileGeom<TX,TY>::SMEM_BYTES. Returns this thread's Courant-number
// contribution; *nan is set when an updated state holds a NaN.
template <int TX, int TY, bool WITH_SRC2, int NT>
__device__ __forceinline__ double tile_body(const dclaw_params& P, const Geom& g, const Rec& R,
                                            const double* __restrict__ b, double* __restrict__ q_out, double dt,
                                            int i0, int j0, double* smem, uint32_t* __restrict__ brlog, bool& nan,
                                            bool active = true) {
    using TG = TileGeom<TX, TY>;
    TileMem M;
    M.A = smem;
    M.B = M.A + (size_t)NW * TG::NA;
    M.C = M.B + (size_t)10 * TG::NB;
    M.D = M.C + (size_t)10 * TG::NC;
    M.H = M.D + (size_t)10 * TG::ND;
    M.Bd = M.H + TG::NHB;
    M.T5 = M.Bd + TG::NHB;
    M.bits = reinterpret_cast<uint32_t*>(M.T5 + (size_t)5 * TG::NTS);
    M.list = reinterpret_cast<int*>(M.bits + TG::NA);
    M.nlist = M.list + TG::NA;
    M.NA = TG::NA;
    const int tid = threadIdx.x;
    M.hi0 = i0 - 3;
    M.hj0 = j0 - 3;
    M.hw = TG::HW;
    M.hv = TX + 6;
    const double dtdx = dt / g.dx, dtdy = dt / g.dy;
    if (!active) {
        // flagged inactive: with src2 in this kernel its cells' zeros are
        // written here, otherwise src2's kernel writes them
        nan = false;
        if (WITH_SRC2) {
            const size_t plane = (size_t)g.mx * g.my;
            for (int it = tid; it < TX * TY; it += NT) {
                int i = i0 + it % TX, j = j0 + it / TX;
                if (i > g.mx || j > g.my) continue;
                size_t c = (size_t)(j - 1) * g.mx + (size_t)(i - 1);
                for (int m = 0; m < 5; ++m) q_out[(size_t)m * plane + c] = 0.0;
            }
        }
        return 0.0;
    }
    // stage h and bed of the cells within 3 of the tile; a tile whose cells
    // within distance 3 are all dry stays dry: all its interfaces are
    // dry-dry (skipped) and src2 zeroes dry cells
    bool any = false;
    if (tid == 0) *M.nlist = 0;  // the x-sweep's solve list (the y-sweep's is reset after the x solves)
    for (int it = tid; it < TG::NHB; it += NT)
        if (tile_stage_hb(g, R, b, M, it)) any = true;
    any = __syncthreads_or(any) != 0;
    double cfl = 0.0;
    nan = false;
    const size_t plane = (size_t)g.mx * g.my;
    if (!any && !brlog) {
        for (int it = tid; it < TX * TY; it += NT) {
            int i = i0 + it % TX, j = j0 + it / TX;
            if (i > g.mx || j > g.my) continue;
            size_t c = (size_t)(j - 1) * g.mx + (size_t)(i - 1);
            for (int m = 0; m < 5; ++m) q_out[(size_t)m * plane + c] = 0.0;
        }
    } else {
        // Items that need a solve are gathered into a dense list first, so
        // that every warp of the solve loop is full of them: wet interfaces
        // cluster in space, and handing items out by index leaves warps of
        // dry items idle at the barrier while others solve twice. The other
        // items store zero waves here. Each item writes only its own slots
        // and the Courant number is a max, so the list's order changes no
        // result. The x-sweep's list is built after the staging, the
        // y-sweep's beside the T phase (neither reads what the other writes).
        const int lane = tid & 31;
        auto build_list = [&](int dir) {
            const int nsolve = dir == 0 ? TG::NXW : TG::NYW;
            for (int it0 = 0; it0 < nsolve; it0 += NT) {
                const int it = it0 + tid;
                bool need = it < nsolve && tile_needs_solve(P, g, M, dir, it, i0, j0, TX);
                if (it < nsolve && !need) {
                    bool ok;
                    tile_riemann(P, g, R, M, dir, it, i0, j0, TX, TY, ok);
                }
                const unsigned bal = __ballot_sync(0xffffffffu, need);
                int base = 0;
                if (lane == 0 && bal) base = atomicAdd(M.nlist, __popc(bal));
                base = __shfl_sync(0xffffffffu, base, 0);
                if (need) M.list[base + __popc(bal & ((1u << lane) - 1u))] = it;
            }
        };
        build_list(0);
        // the two sweeps share one copy of the solver, limiter and rpt2 code
#pragma unroll 1
        for (int dir = 0; dir < 2; ++dir) {
            const double dtd = dir == 0 ? dtdx : dtdy;
            __syncthreads();  // this sweep's list is complete
            const int nneed = *M.nlist;
            for (int w = tid; w < nneed; w += NT) {
                bool ok;
                double s = tile_riemann(P, g, R, M, dir, M.list[w], i0, j0, TX, TY, ok);
                if (ok) cfl = fmax2(cfl, dtd * s);
            }
            __syncthreads();
            // every thread has read this sweep's list length: reset it for the
            // next sweep, whose list is built after one more barrier
            if (tid == 0) *M.nlist = 0;
            // A half-warp per slice (x: a row, y: a column), lane k on
            // interface k of it. Each interface is limited once; a cell
            // takes its own interface's fluctuations and, from the next
            // lane, those of the next interface (a cell limited both
            // before). Every thread reaches the shuffles.
            constexpr bool XPAIR = TX + 1 <= 16 && (TY + 2) * 16 <= NT && NT % 32 == 0;
            constexpr bool YPAIR = TY + 1 <= 16 && (TX + 2) * 16 <= NT && NT % 32 == 0;
            if ((XPAIR && dir == 0) || (YPAIR && dir == 1)) {
                const int sl = tid >> 4, k = tid & 15;
                const int nsl = dir == 0 ? TY + 2 : TX + 2, span = dir == 0 ? TX : TY;
                const int s = (dir == 0 ? j0 : i0) - 1 + sl, a = (dir == 0 ? i0 : j0) + k;
                const int smax = dir == 0 ? g.my + 1 : g.mx + 1, amax = dir == 0 ? g.mx : g.my;
                const bool sl_ok = sl < nsl && s >= 0 && s <= smax;
                double v[15];
                uint32_t lb = 0;
                if (sl_ok && k <= span && a <= amax + 1) {
                    if (dir == 0) tile_x_iface<TX, TY>(P, M, s, a, i0, j0, dtd, v, brlog ? &lb : nullptr);
                    else tile_y_iface<TX, TY>(P, M, s, a, i0, j0, dtd, v, brlog ? &lb : nullptr);
                } else {
                    for (int m = 0; m < 15; ++m) v[m] = 0.0;
                }
                double vn[15];
                for (int m = 0; m < 15; ++m) vn[m] = __shfl_down_sync(0xffffffffu, v[m], 1);
                const uint32_t lbn = __shfl_down_sync(0xffffffffu, lb, 1);
                if (sl_ok && k < span && a <= amax) {
                    if (dir == 0) tile_flux_cell<TX, TY>(P, g, R, M, 0, a, s, i0, j0, dtd, v, vn, lb, lbn, brlog);
                    else tile_flux_cell<TX, TY>(P, g, R, M, 1, s, a, i0, j0, dtd, v, vn, lb, lbn, brlog);
                }
            } else {
                const int ncell = dir == 0 ? (TY + 2) * TX : TY * (TX + 2);
                for (int it = tid; it < ncell; it += NT) tile_flux<TX, TY>(P, g, R, M, dir, it, i0, j0, dtd, brlog);
            }
            __syncthreads();
            if (dir == 0) {
                // T into its own buffer (the y-sweep's flux phase reads it
                // and writes gm/gp over C), so no barrier between the
                // reads of C and the stores
                const int nT = TG::NTS;
                for (int it = tid; it < nT; it += NT) {
                    double T0[5];
                    if (tile_T<TX, TY>(g, M, it, i0, j0, T0)) tile_T_store<TX, TY>(M, it, T0);
                }
                // the x waves are no longer read: the y-sweep's zero waves
                // and list go in beside T
                build_list(1);
            }
        }
        for (int it = tid; it < TX * TY; it += NT)
            if (tile_final<TX, TY, WITH_SRC2>(P, g, R, M, it, i0, j0, dt, q_out)) nan = true;
    }
    if (!(cfl == cfl)) cfl = 0.0;
    return cfl;
}

// ty0: the first tile row of the launch (grid.y tile rows from there)
template <int TX, int TY, bool WITH_SRC2>
__global__ void __launch_bounds__(TILE_TPB, DCLAW_TILE_MINBLOCKS) k_tile(dclaw_params P, Geom g, Rec R, const double* __restrict__ b,
                                                 double* __restrict__ q_out, dclaw_clock* clk,
                                                 uint32_t* __restrict__ brlog, const uint32_t* __restrict__ tflag,
                                                 int ty0 = 0) {
    extern __shared__ double smem[];
    const int ty = (int)blockIdx.y + ty0;
    const int i0 = 1 + blockIdx.x * TX, j0 = 1 + ty * TY;
    const bool active = !tflag || brlog || tflag[ty * gridDim.x + blockIdx.x] == clk->nsteps + 1u;
    bool nan;
    double cfl = tile_body<TX, TY, WITH_SRC2, TILE_TPB>(P, g, R, b, q_out, clk->dt, i0, j0, smem, brlog, nan, active);
    if (nan) flag_status(clk, DCLAW_ERR_NAN);
    block_max_to(cfl, reinterpret_cast<unsigned long long*>(&clk->cfl_bits));
    if (WITH_SRC2) last_block_tick(P, clk);
}

// src2 of the interior cells c0 .. c0 + ncell - 1 (all by default) from the
// updated state; with `tick` the last block applies the tick rule
__global__ void __launch_bounds__(SRC2_TPB, SRC2_MINB) k_src2_cells(dclaw_params P, Geom g, const double* __restrict__ q_star,
                                                    double* __restrict__ q_out, dclaw_clock* clk,
                                                    const uint32_t* __restrict__ tflag, long long c0 = 0,
                                                    long long ncell = -1, int tick = 1) {
    const long long n = ncell < 0 ? (long long)g.mx * g.my : ncell;
    long long idx = c0 + (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx < c0 + n) {
        int i, j;
        split_index(idx, g.mx, i, j);
        i += 1;
        j += 1;
        if (tile_active(tflag, clk->nsteps + 1u, i, j, TILE_X, TILE_Y, (g.mx + TILE_X - 1) / TILE_X)) {
            cell_src2(P, g, clk->dt, q_star, q_out, (size_t)idx);
        } else {
            const size_t plane = (size_t)g.mx * g.my;
            for (int m = 0; m < 5; ++m) q_out[(size_t)m * plane + (size_t)idx] = 0.0;
        }
    }
    if (tick) last_block_tick(P, clk);
}

// ---- single patch over tile lists -------------------------------------------
// dclaw_step without a branch log: the records, tiles and src2 run only
// where the flow is. (1) k_scan_patch reads every interior cell's five
// fields (the NaN check), marks the tiles whose read range holds a wet cell
// and writes the zero state into q_out; (2) k_list_patch lists the active
// tiles and the tiles that are active or next to one; (3) k_records_list
// builds the records of the second list's tiles (every record an active tile
// reads, once); (4) k_tile_list, a persistent kernel, takes the active tiles
// from a queue; (5) k_src2_list overwrites the zeros of the active tiles'
// cells with src2 of the updated state, and its last block applies the tick.
// Each cell's arithmetic is that of the full-grid kernels, so the results
// are the same bits; far from the flow a cell costs its 80 bytes of scan.
// cells [s0, s1) are scanned, cells [z0, z1) of q_out zeroed (linear
// interior indices; the whole patch for dclaw_step, a row range and the rows
// within 3 of it for dclaw_step_rows)
__global__ void __launch_bounds__(TPB, DCLAW_SCAN_MINB) k_scan_patch(dclaw_params P, int mx, int my,
                                                                    const double* __restrict__ q_in,
                                                                    double* __restrict__ q_out, dclaw_clock* clk,
                                                                    unsigned int* counters,
                                                                    uint32_t* __restrict__ tflag, size_t s0,
                                                                    size_t s1, size_t z0, size_t z1) {
    if (blockIdx.x == 0 && threadIdx.x < 3) counters[threadIdx.x] = 0u;  // tile queue and list lengths
    const size_t n = (size_t)mx * my;
    const int ntx = (mx + TILE_X - 1) / TILE_X, nty = (my + TILE_Y - 1) / TILE_Y;
    const size_t lo = s0 < z0 ? s0 : z0, hi = s1 > z1 ? s1 : z1;
    bool nan = false;
    for (size_t idx = lo + (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < hi;
         idx += (size_t)gridDim.x * blockDim.x) {
        if (idx >= s0 && idx < s1 && scan_cell(P, q_in, n, idx, mx, tflag, clk, TILE_X, TILE_Y, ntx, nty)) nan = true;
        if (idx >= z0 && idx < z1)
            for (int f = 0; f < 5; ++f) q_out[(size_t)f * n + idx] = 0.0;
    }
    if (nan) flag_status(clk, DCLAW_ERR_NAN);
}

// active tiles of tile rows ty0..ty1, and the tiles of rows ty0-1..ty1+1
// that are active or next to one (the whole patch: 0..nty-1)
__global__ void __launch_bounds__(TPB) k_list_patch(int ntx, int nty, const dclaw_clock* clk,
                                                    const uint32_t* __restrict__ tflag, unsigned int* counters,
                                                    uint32_t* __restrict__ list_act, uint32_t* __restrict__ list_rec,
                                                    int ty0, int ty1) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t ntiles = (uint32_t)ntx * (uint32_t)nty;
    const uint32_t epoch = clk->nsteps + 1u;
    bool act = false, rec = false;
    if (t < ntiles) {
        const int ty = (int)(t / ntx);
        const bool flag = tflag[t] == epoch;
        act = flag && ty >= ty0 && ty <= ty1;
        rec = ty >= ty0 - 1 && ty <= ty1 + 1 && (flag || near_active(tflag, epoch, (int)(t % ntx), ty, ntx, nty));
    }
    const int lane = threadIdx.x & 31;
    const unsigned ba = __ballot_sync(0xffffffffu, act), br = __ballot_sync(0xffffffffu, rec);
    unsigned base_a = 0, base_r = 0;
    if (lane == 0) {
        if (ba) base_a = atomicAdd(counters + 1, (unsigned)__popc(ba));
        if (br) base_r = atomicAdd(counters + 2, (unsigned)__popc(br));
    }
    base_a = __shfl_sync(0xffffffffu, base_a, 0);
    base_r = __shfl_sync(0xffffffffu, base_r, 0);
    const unsigned below = (1u << lane) - 1u;
    if (act) list_act[base_a + __popc(ba & below)] = t;
    if (rec) list_rec[base_r + __popc(br & below)] = t;
}

__global__ void __launch_bounds__(RECORDS_TPB, RECORDS_MINB) k_records_list(dclaw_params P, Geom g,
                                                                            const double* __restrict__ q_in,
                                                                            const double* __restrict__ b, Rec R,
                                                                            const unsigned int* counters,
                                                                            const uint32_t* __restrict__ list_rec) {
    const uint32_t n = counters[2];
    const int ntx = (g.mx + TILE_X - 1) / TILE_X, nty = (g.my + TILE_Y - 1) / TILE_Y;
    for (uint32_t k = blockIdx.x; k < n; k += gridDim.x) {
        const uint32_t t = list_rec[k];
        tile_records<TILE_X, TILE_Y>(P, g, q_in, b, R, (int)(t % ntx), (int)(t / ntx), ntx, nty);
    }
}

// persistent: each CTA takes active tiles from the queue until it is empty;
// the Courant number is max-reduced once per CTA at the end. WITH_SRC2:
// q_out receives the state after src2 and the last CTA applies the tick
// (no k_src2_list); otherwise the pre-src2 state.
template <bool WITH_SRC2>
__global__ void __launch_bounds__(TILE_TPB, DCLAW_TILE_MINBLOCKS) k_tile_list(dclaw_params P, Geom g, Rec R,
                                                                             const double* __restrict__ b,
                                                                             double* __restrict__ q_out,
                                                                             dclaw_clock* clk, unsigned int* counters,
                                                                             const uint32_t* __restrict__ list_act) {
    extern __shared__ double smem[];
    // the tile of this pass and the next one's, claimed at the start of this
    // pass: the barrier that ends a pass also publishes the next index
    __shared__ uint32_t s_t[2];
    const unsigned int nact = counters[1];
    const uint32_t ntx = (uint32_t)((g.mx + TILE_X - 1) / TILE_X);
    const double dt = clk->dt;
    double cfl = 0.0;
    bool nan_any = false;
    if (threadIdx.x == 0) {
        const unsigned int k = atomicAdd(counters, 1u);
        s_t[0] = k < nact ? list_act[k] : 0xffffffffu;
    }
    __syncthreads();
    for (int pass = 0;; ++pass) {
        const uint32_t t = s_t[pass & 1];
        if (t == 0xffffffffu) break;
        // s_t[(pass + 1) & 1] was last read before the previous pass's barrier
        if (threadIdx.x == 0) {
            const unsigned int k = atomicAdd(counters, 1u);
            s_t[(pass + 1) & 1] = k < nact ? list_act[k] : 0xffffffffu;
        }
        const int i0 = 1 + (int)(t % ntx) * TILE_X, j0 = 1 + (int)(t / ntx) * TILE_Y;
        bool nan;
        const double c =
            tile_body<TILE_X, TILE_Y, WITH_SRC2, TILE_TPB>(P, g, R, b, q_out, dt, i0, j0, smem, nullptr, nan);
        cfl = fmax2(cfl, c);
        nan_any = nan_any || nan;
        // the next tile's staging overwrites shared memory
        __syncthreads();
    }
    if (nan_any) flag_status(clk, DCLAW_ERR_NAN);
    block_max_to(cfl, reinterpret_cast<unsigned long long*>(&clk->cfl_bits));
    if (WITH_SRC2) last_block_tick(P, clk);
}

__global__ void __launch_bounds__(SRC2_TPB, SRC2_MINB) k_src2_list(dclaw_params P, Geom g,
                                                                  const double* __restrict__ q_star,
                                                                  double* __restrict__ q_out, dclaw_clock* clk,
                                                                  const unsigned int* counters,
                                                                  const uint32_t* __restrict__ list_act,
                                                                  int tick = 1) {
    const uint32_t nact = counters[1];
    const uint32_t ntx = (uint32_t)((g.mx + TILE_X - 1) / TILE_X);
    const double dt = clk->dt;
    for (uint32_t k = blockIdx.x; k < nact; k += gridDim.x) {
        const uint32_t t = list_act[k];
        const int i0 = 1 + (int)(t % ntx) * TILE_X, j0 = 1 + (int)(t / ntx) * TILE_Y;
        for (int c = threadIdx.x; c < TILE_X * TILE_Y; c += blockDim.x) {
            const int i = i0 + c % TILE_X, j = j0 + c / TILE_X;
            if (i > g.mx || j > g.my) continue;
            cell_src2(P, g, dt, q_star, q_out, (size_t)(j - 1) * g.mx + (size_t)(i - 1));
        }
    }
    if (tick) last_block_tick(P, clk);
}

// ---- batched ensemble -------------------------------------------------------
// the ensemble's tile shapes: 14 x 13 (the single patch's), 13 x 14, 16 x 14
constexpr int NBATCH_SHAPES = 3;
__host__ __device__ constexpr int batch_tx(int k) { return k == 0 ? 14 : (k == 1 ? 13 : 16); }
__host__ __device__ constexpr int batch_ty(int k) { return k == 0 ? 13 : (k == 1 ? 14 : 14); }

// index of the member owning global chunk/tile `x` (largest k with first[k] <= x)
template <typename F>
__device__ __forceinline__ int find_member(int n, uint32_t x, F first) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (first(mid) <= x) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// copy member m's table entry and parameters into shared memory (whole CTA)
__device__ __forceinline__ void load_member(const dclaw_member* __restrict__ mem, const dclaw_params* __restrict__ prm,
                                            int m, dclaw_member& sM, dclaw_params& sP) {
    const int nM = (int)(sizeof(dclaw_member) / 4), nP = (int)(sizeof(dclaw_params) / 4);
    for (int k = threadIdx.x; k < nM + nP; k += blockDim.x) {
        if (k < nM) reinterpret_cast<int*>(&sM)[k] = reinterpret_cast<const int*>(mem + m)[k];
        else reinterpret_cast<int*>(&sP)[k - nM] = reinterpret_cast<const int*>(prm + m)[k - nM];
    }
}

// Every thread finds its chunk's member by binary search over the member
// table (read through the cache; all threads of a block share the chunk, so
// the search is uniform) and reads the member's entry and parameters in
// place: no shared-memory broadcast and no barrier per chunk.
// the member owning chunk ch, starting from the previous chunk's member m
// (grid-stride loops mostly stay inside one member: no search then)
template <typename F>
__device__ __forceinline__ int member_of(int nmem, uint32_t nchunks, uint32_t ch, int m, F first) {
    if (m >= 0 && first(m) <= ch && ch < (m + 1 < nmem ? first(m + 1) : nchunks)) return m;
    return find_member(nmem, ch, first);
}

// After the scan: the active tiles (for the tile kernel) and the tiles
// whose records an active tile reads (for pass 2), each appended to its
// list in one warp-aggregated atomic per warp. One thread per tile.
__global__ void __launch_bounds__(TPB) k_list_batch(int nmem, uint32_t ntiles, const dclaw_member* __restrict__ mem,
                                                    const dclaw_clock* clocks, const uint32_t* __restrict__ tflag,
                                                    unsigned int* counters, uint32_t* __restrict__ list_act,
                                                    uint32_t* __restrict__ list_rec) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    bool act = false, rec = false;
    if (t < ntiles) {
        const int m = find_member(nmem, t, [&](int k) { return mem[k].tile0; });
        const dclaw_member& M = mem[m];
        const uint32_t epoch = clocks[m].nsteps + 1u;
        const int ntx = (int)M.ntiles_x, lt = (int)(t - M.tile0);
        act = tflag[t] == epoch;
        rec = act || near_active(tflag + M.tile0, epoch, lt % ntx, lt / ntx, ntx, (int)(M.ntiles / M.ntiles_x));
    }
    const int lane = threadIdx.x & 31;
    const unsigned ba = __ballot_sync(0xffffffffu, act), br = __ballot_sync(0xffffffffu, rec);
    unsigned base_a = 0, base_r = 0;
    if (lane == 0) {
        if (ba) base_a = atomicAdd(counters + 1, (unsigned)__popc(ba));
        if (br) base_r = atomicAdd(counters + 2, (unsigned)__popc(br));
    }
    base_a = __shfl_sync(0xffffffffu, base_a, 0);
    base_r = __shfl_sync(0xffffffffu, base_r, 0);
    const unsigned below = (1u << lane) - 1u;
    if (act) list_act[base_a + __popc(ba & below)] = t;
    if (rec) list_rec[base_r + __popc(br & below)] = t;
}

// pass 2 of the records over the listed tiles (grid-stride over the list)
template <int TX, int TY>
__global__ void __launch_bounds__(BATCH_CELL_TPB, BATCH_CELL_MINB) k_records_tiles_batch(int nmem, uint32_t ntiles,
                                                                              const dclaw_member* __restrict__ mem,
                                                                              const dclaw_params* __restrict__ prm,
                                                                              const double* __restrict__ q_in,
                                                                              const double* __restrict__ b,
                                                                              double* __restrict__ work,
                                                                              const unsigned int* counters,
                                                                              const uint32_t* __restrict__ list_rec) {
    const uint32_t n = counters[2];
    int m = -1;
    for (uint32_t k = blockIdx.x; k < n; k += gridDim.x) {
        const uint32_t t = list_rec[k];
        m = member_of(nmem, ntiles, t, m, [&](int j) { return mem[j].tile0; });
        const dclaw_member& M = mem[m];
        const Geom g{M.mx, M.my, M.mx + 4, M.my + 4, M.dx, M.dy};
        const Rec R{work + M.rec_off, (size_t)g.PX * g.PY};
        const int ntx = (int)M.ntiles_x, lt = (int)(t - M.tile0);
        tile_records<TX, TY>(prm[m], g, q_in + M.q_off, b + M.b_off, R, lt % ntx, lt / ntx, ntx,
                             (int)(M.ntiles / M.ntiles_x));
    }
}

// pass 1 of the two-pass records over every member's interior chunks
// It also writes the zero state into q_out for every cell: the cells of
// inactive tiles keep it, src2 over the active tiles overwrites the others.
__global__ void __launch_bounds__(TPB, DCLAW_SCAN_MINB) k_scan_batch(int nmem, uint32_t nchunks, const dclaw_member* __restrict__ mem,
                                                    const dclaw_params* __restrict__ prm, dclaw_clock* clocks,
                                                    const double* __restrict__ q_in, double* __restrict__ q_out,
                                                    unsigned int* counters, uint32_t* __restrict__ tflag, int TX,
                                                    int TY) {
    if (blockIdx.x == 0 && threadIdx.x < 3) counters[threadIdx.x] = 0u;  // tile queue and list lengths
    int m = -1;
    for (uint32_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
        m = member_of(nmem, nchunks, ch, m, [&](int k) { return mem[k].schunk0; });
        const dclaw_member& M = mem[m];
        const size_t n = (size_t)M.mx * M.my;
        const size_t idx = (size_t)(ch - M.schunk0) * TPB + threadIdx.x;
        if (idx < n) {
            if (scan_cell(prm[m], q_in + M.q_off, n, idx, M.mx, tflag + M.tile0, clocks + m, TX, TY, (int)M.ntiles_x,
                          (int)(M.ntiles / M.ntiles_x)))
                flag_status(clocks + m, DCLAW_ERR_NAN);
            double* qo = q_out + M.q_off + idx;
            for (int f = 0; f < 5; ++f) qo[(size_t)f * n] = 0.0;
        }
    }
}

template <int TX, int TY>
__global__ void __launch_bounds__(TPB, 2) k_tile_batch(int nmem, uint32_t ntiles, const dclaw_member* __restrict__ mem,
                                                       const dclaw_params* __restrict__ prm, dclaw_clock* clocks,
                                                       const double* __restrict__ b, double* __restrict__ work,
                                                       unsigned int* counters, const uint32_t* __restrict__ list_act,
                                                       double* __restrict__ q_out) {
    extern __shared__ double smem[];
    __shared__ dclaw_member sM;
    __shared__ dclaw_params sP;
    __shared__ unsigned int s_t;
    __shared__ int s_m;
    __shared__ double red[TPB / 32];
    // the queue hands out the active tiles only (inactive tiles: no wet
    // cell within 3; src2 writes their zeros)
    const unsigned int nact = counters[1];
    int cur = -1;
    for (;;) {
        if (threadIdx.x == 0) {
            const unsigned int k = atomicAdd(counters, 1u);
            s_t = k < nact ? list_act[k] : ntiles;
            s_m = s_t < ntiles ? find_member(nmem, s_t, [&](int j) { return mem[j].tile0; }) : -1;
        }
        __syncthreads();
        const unsigned int t = s_t;
        const int m = s_m;
        if (t >= ntiles) break;
        if (m != cur) {
            load_member(mem, prm, m, sM, sP);
            __syncthreads();
            cur = m;
        }
        const Geom g{sM.mx, sM.my, sM.mx + 4, sM.my + 4, sM.dx, sM.dy};
        const Rec R{work + sM.rec_off, (size_t)g.PX * g.PY};
        const unsigned int lt = t - sM.tile0;
        const int i0 = 1 + (int)(lt % sM.ntiles_x) * TX, j0 = 1 + (int)(lt / sM.ntiles_x) * TY;
        bool nan;
        // with src2 in this kernel the tile writes the member's new state,
        // otherwise its pre-src2 state (k_src2_batch follows)
        double* dst = DCLAW_BATCH_SRC2_KERNEL ? work + sM.qs_off : q_out + sM.q_off;
        double cfl = tile_body<TX, TY, !DCLAW_BATCH_SRC2_KERNEL, TPB>(sP, g, R, b + sM.b_off, dst, clocks[m].dt, i0, j0,
                                                                     smem, nullptr, nan);
        if (nan) flag_status(clocks + m, DCLAW_ERR_NAN);
        // block max of this tile's Courant number into member m's clock
        cfl = warp_max(cfl);
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        if (lane == 0) red[wid] = cfl;
        __syncthreads();
        if (wid == 0) {
            double x = lane < TPB / 32 ? red[lane] : 0.0;
            x = warp_max(x);
            if (lane == 0 && x > 0.0)
                atomicMax(reinterpret_cast<unsigned long long*>(&clocks[m].cfl_bits),
                          (unsigned long long)__double_as_longlong(x));
        }
        __syncthreads();
    }
}

// src2 of the active tiles' cells (grid-stride over the active list; the
// scan has written the zeros of every other cell)
template <int TX, int TY>
__global__ void __launch_bounds__(BATCH_CELL_TPB, BATCH_CELL_MINB) k_src2_batch(int nmem, uint32_t ntiles, const dclaw_member* __restrict__ mem,
                                                    const dclaw_params* __restrict__ prm, const dclaw_clock* clocks,
                                                    double* __restrict__ q_out, const double* __restrict__ work,
                                                    const unsigned int* counters,
                                                    const uint32_t* __restrict__ list_act) {
    const uint32_t nact = counters[1];
    int m = -1;
    for (uint32_t k = blockIdx.x; k < nact; k += gridDim.x) {
        const uint32_t t = list_act[k];
        m = member_of(nmem, ntiles, t, m, [&](int j) { return mem[j].tile0; });
        const dclaw_member& M = mem[m];
        const Geom g{M.mx, M.my, M.mx + 4, M.my + 4, M.dx, M.dy};
        const int lt = (int)(t - M.tile0), ntx = (int)M.ntiles_x;
        const int i0 = 1 + (lt % ntx) * TX, j0 = 1 + (lt / ntx) * TY;
        const double dt = clocks[m].dt;
        for (int c = threadIdx.x; c < TX * TY; c += blockDim.x) {
            const int i = i0 + c % TX, j = j0 + c / TX;
            if (i > g.mx || j > g.my) continue;
            cell_src2(prm[m], g, dt, work + M.qs_off, q_out + M.q_off, (size_t)(j - 1) * g.mx + (size_t)(i - 1));
        }
    }
}

// every member's tick, after its src2
__global__ void __launch_bounds__(TPB) k_tick_batch(int nmem, const dclaw_params* __restrict__ prm,
                                                    dclaw_clock* clocks) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m < nmem) tick_device(prm[m], clocks + m);
}

template <int TX, int TY>
inline int batch_tile_attr() {
    static std::atomic<bool> done[MAX_DEVICES];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) return DCLAW_ERR_CUDA;
    if (!done[dev].load(std::memory_order_acquire)) {
        std::lock_guard<std::mutex> lock(g_setup_mu);
        if (!done[dev].load(std::memory_order_relaxed)) {
            if (cudaFuncSetAttribute(k_tile_batch<TX, TY>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)TileGeom<TX, TY>::SMEM_BYTES) != cudaSuccess)
                return DCLAW_ERR_CUDA;
            done[dev].store(true, std::memory_order_release);
        }
    }
    return DCLAW_OK;
}

template <int TX, int TY>
inline int launch_tile_batch(const dclaw_batch* B, const dclaw_member* mem, const dclaw_params* prm, dclaw_clock* clocks,
                             const double* b, double* work, unsigned int* counters, const uint32_t* list_act, int nsm,
                             cudaStream_t s, double* q_out = nullptr) {
    if (batch_tile_attr<TX, TY>() != DCLAW_OK) return DCLAW_ERR_CUDA;
    unsigned grid = (unsigned)(nsm * (B->tile_ctas_per_sm > 0 ? B->tile_ctas_per_sm : 2));
    if (grid > B->ntiles) grid = B->ntiles > 0 ? B->ntiles : 1;
    k_tile_batch<TX, TY><<<grid, TPB, TileGeom<TX, TY>::SMEM_BYTES, s>>>(B->nmembers, B->ntiles, mem, prm, clocks, b,
                                                                        work, counters, list_act, q_out);
    return DCLAW_OK;
}

// the records the active tiles read, the tiles, src2 (after the scan and
// the lists)
template <int TX, int TY>
inline int launch_batch_tiles(const dclaw_batch* B, const dclaw_member* mem, const dclaw_params* prm,
                              dclaw_clock* clocks, const double* q_in, double* q_out, const double* b, double* w,
                              unsigned int* counters, const uint32_t* tflag, const uint32_t* list_act,
                              const uint32_t* list_rec, int nsm, int cpsm, cudaStream_t s) {
    unsigned g1 = (unsigned)(nsm * cpsm);
    if (g1 > B->ntiles) g1 = B->ntiles > 0 ? B->ntiles : 1;
    k_records_tiles_batch<TX, TY><<<g1, BATCH_CELL_TPB, 0, s>>>(B->nmembers, B->ntiles, mem, prm, q_in, b, w, counters,
                                                                 list_rec);
    int rc = launch_tile_batch<TX, TY>(B, mem, prm, clocks, b, w, counters, list_act, nsm, s, q_out);
    if (rc != DCLAW_OK) return rc;
    if (!DCLAW_BATCH_SRC2_KERNEL) return DCLAW_OK;
    unsigned g3 = (unsigned)(nsm * cpsm);
    if (g3 > B->ntiles) g3 = B->ntiles > 0 ? B->ntiles : 1;
    k_src2_batch<TX, TY><<<g3, BATCH_CELL_TPB, 0, s>>>(B->nmembers, B->ntiles, mem, prm, clocks, q_out, w, counters,
                                                        list_act);
    return DCLAW_OK;
}

inline int sm_count() {
    static std::atomic<int> n[MAX_DEVICES];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) return 0;
    int v = n[dev].load(std::memory_order_relaxed);
    if (!v) {
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
        n[dev].store(v, std::memory_order_relaxed);
    }
    return v;
}

// ---- patch calls (padded layout) ------------------------------------------
__global__ void __launch_bounds__(TPB) k_bc2amr(dclaw_params P, int mx, int my, double* q) {
    // one thread per padded cell; ghost cells read their source interior cell
    const int PX = mx + 4, PY = my + 4;
    const size_t npad = (size_t)PX * PY;
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)npad) return;
    int i = (int)(idx % PX) - 1, j = (int)(idx / PX) - 1;
    if (i >= 1 && i <= mx && j >= 1 && j <= my) return;
    int si = i, sj = j;
    bool fu = false, fv = false;
    if (i < 1) { if (P.bc_lower[0] == DCLAW_BC_WALL) { si = 1 - i; fu = true; } else si = 1; }
    else if (i > mx) { if (P.bc_upper[0] == DCLAW_BC_WALL) { si = 2 * mx + 1 - i; fu = true; } else si = mx; }
    if (j < 1) { if (P.bc_lower[1] == DCLAW_BC_WALL) { sj = 1 - j; fv = true; } else sj = 1; }
    else if (j > my) { if (P.bc_upper[1] == DCLAW_BC_WALL) { sj = 2 * my + 1 - j; fv = true; } else sj = my; }
    const size_t d = (size_t)(j + 1) * PX + (size_t)(i + 1);
    const size_t s = (size_t)(sj + 1) * PX + (size_t)(si + 1);
    for (int m = 0; m < 5; ++m) {
        double v = q[(size_t)m * npad + s];
        if ((m == 1 && fu) || (m == 2 && fv)) v = -v;
        q[(size_t)m * npad + d] = v;
    }
}

__global__ void __launch_bounds__(TPB) k_setaux(dclaw_params P, int mx, int my, double* aux) {
    const int PX = mx + 4, PY = my + 4;
    const size_t npad = (size_t)PX * PY;
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)npad) return;
    int i = (int)(idx % PX) - 1, j = (int)(idx / PX) - 1;
    int ii = i < 1 ? 1 : (i > mx ? mx : i);
    int jj = j < 1 ? 1 : (j > my ? my : j);
    aux[idx] = aux[(size_t)(jj + 1) * PX + (size_t)(ii + 1)];
    aux[npad + idx] = P.phi;
    aux[2 * npad + idx] = P.theta_input;
    aux[3 * npad + idx] = 0.0;
    aux[4 * npad + idx] = 0.0;
    aux[5 * npad + idx] = 0.0;
}

__global__ void __launch_bounds__(TPB) k_b4_padded(dclaw_params P, int mx, int my, double* q, dclaw_clock* clk) {
    const int PX = mx + 4, PY = my + 4;
    const size_t npad = (size_t)PX * PY;
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)npad) return;
    double h = q[idx], hu = q[npad + idx], hv = q[2 * npad + idx], hm = q[3 * npad + idx], p = q[4 * npad + idx];
    if (clk && ((h != h) || (hu != hu) || (hv != hv) || (hm != hm) || (p != p))) flag_status(clk, DCLAW_ERR_NAN);
    double u, v, m;
    qfix(P, h, hu, hv, hm, p, u, v, m, P.grav);
    if (h > 0.0) {
        double s = sqrt((sq(hu) + sq(hv))) / h;
        if (s > P.speed_limit) {
            double sratio = P.speed_limit / s;
            hu = hu * sratio;
            hv = hv * sratio;
        }
    }
    q[idx] = h; q[npad + idx] = hu; q[2 * npad + idx] = hv; q[3 * npad + idx] = hm; q[4 * npad + idx] = p;
}

__global__ void __launch_bounds__(TPB) k_update_padded(Geom g, Work W, double dt, double* q, double* fluxes,
                                                       dclaw_clock* clk) {
    const long long n = (long long)g.mx * g.my;
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n) return;
    int i = (int)(idx % g.mx) + 1, j = (int)(idx / g.mx) + 1;
    double qn[5], fl[20];
    bool nan = stage_update(g, W, i, j, dt, qn, fluxes ? fl : nullptr);
    if (nan && clk) flag_status(clk, DCLAW_ERR_NAN);
    const size_t pc = pidx(g, i, j);
    for (int m = 0; m < 5; ++m) q[(size_t)m * W.npad + pc] = qn[m];
    if (fluxes) {
        const size_t np = W.npad;
        for (int m = 0; m < 5; ++m) {
            fluxes[(size_t)(0 + m) * np + pidx(g, i + 1, j)] = fl[m];
            fluxes[(size_t)(5 + m) * np + pc] = fl[5 + m];
            fluxes[(size_t)(10 + m) * np + pidx(g, i, j + 1)] = fl[10 + m];
            fluxes[(size_t)(15 + m) * np + pc] = fl[15 + m];
        }
    }
}

__global__ void __launch_bounds__(TPB) k_src2_padded(dclaw_params P, int mx, int my, double dt, double* q) {
    const long long n = (long long)mx * my;
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n) return;
    const int PX = mx + 4, PY = my + 4;
    const size_t npad = (size_t)PX * PY;
    int i = (int)(idx % mx) + 1, j = (int)(idx / mx) + 1;
    const size_t pc = (size_t)(j + 1) * PX + (size_t)(i + 1);
    double a = q[pc], b = q[npad + pc], c = q[2 * npad + pc], d = q[3 * npad + pc], e = q[4 * npad + pc];
    src2_cell(P, P.phi, dt, a, b, c, d, e);
    q[pc] = a; q[npad + pc] = b; q[2 * npad + pc] = c; q[3 * npad + pc] = d; q[4 * npad + pc] = e;
}

// running peak of a plane and the step that set it; the adjoint adds the
// peak's adjoint at that step
__global__ void __launch_bounds__(TPB) k_peak_update(const double* __restrict__ h, double* __restrict__ hmax,
                                                     int32_t* __restrict__ arg, long long n, int step) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double v = h[i];
        if (v > hmax[i]) {
            hmax[i] = v;
            arg[i] = step;
        }
    }
}

__global__ void __launch_bounds__(TPB) k_peak_adjoint(const double* __restrict__ g, const int32_t* __restrict__ arg,
                                                      long long n, int step, double* __restrict__ lam) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        if (arg[i] == step) lam[i] += g[i];
}

// Fortran cell-major arrays (nfa fields per cell) <-> field planes: one
// thread per cell; a warp's reads cover its cells' contiguous records, its
// writes are contiguous within each plane
__global__ void __launch_bounds__(TPB) k_fields_soa(const double* __restrict__ a, int nfa, int nf, long long ncell,
                                                    double* __restrict__ planes) {
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < ncell;
         c += (long long)gridDim.x * blockDim.x)
        for (int f = 0; f < nf; ++f) planes[(long long)f * ncell + c] = a[c * nfa + f];
}

__global__ void __launch_bounds__(TPB) k_fields_aos(const double* __restrict__ planes, int nf, int nfa, long long ncell,
                                                    double* __restrict__ a) {
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < ncell;
         c += (long long)gridDim.x * blockDim.x)
        for (int f = 0; f < nf; ++f) a[c * nfa + f] = planes[(long long)f * ncell + c];
}

// observation slot of clock c after its step, or -1: the flume loop's
// k = round(t / dt_obs) - 1 (round half to even) and its hit test
// |t - (k+1) dt_obs| < 1e-9 with dt > 0 (pf_flume/flume_model.py:155-157)
__device__ __forceinline__ long long obs_slot(const dclaw_clock* c, int n_obs) {
    const double to = c->t_obs;
    if (!(to > 0.0) || !(c->dt_last > 0.0)) return -1;
    const double kr = rint(c->t / to) - 1.0;
    if (!(kr >= 0.0) || !(kr < (double)n_obs)) return -1;
    const long long k = (long long)kr;
    return fabs(c->t - (double)(k + 1) * to) < 1.0e-9 ? k : -1;
}

__global__ void __launch_bounds__(TPB) k_obs_record(const dclaw_clock* __restrict__ clocks, int n_clocks,
                                                    const int32_t* __restrict__ member, const double* __restrict__ q,
                                                    const int64_t* __restrict__ sel, long long nsel, int n_obs,
                                                    int step, double* __restrict__ out, int32_t* __restrict__ out_step) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < nsel; e += stride) {
        const long long k = obs_slot(clocks + (member ? member[e] : 0), n_obs);
        if (k >= 0) out[k * nsel + e] = q[sel ? sel[e] : e];
    }
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n_clocks; c += stride) {
        const long long k = obs_slot(clocks + c, n_obs);
        if (k >= 0) out_step[k * n_clocks + c] = step;
    }
}

__global__ void __launch_bounds__(TPB) k_wave_speed(dclaw_params P, int mx, int my, const double* __restrict__ q,
                                                   unsigned long long* acc) {
    const long long n = (long long)mx * my;
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double v = 0.0;
    if (idx < n) {
        double h = q[idx];
        if (h > P.dry_tolerance) {
            double u = q[n + idx] / h, w = q[2 * n + idx] / h;
            v = sqrt(sq(u) + sq(w)) + sqrt(P.grav * h);
        }
        if (!(v == v)) v = 0.0;
    }
    block_max_to(v, acc);
}

__global__ void k_cfl_from_bits(dclaw_clock* clk) {
    if (threadIdx.x == 0 && blockIdx.x == 0) clk->cfl = __longlong_as_double((long long)clk->cfl_bits);
}

// ---- host helpers ----------------------------------------------------------
inline unsigned nblocks(long long n) { return (unsigned)((n + TPB - 1) / TPB); }
inline unsigned src2_blocks(long long n) { return (unsigned)((n + SRC2_TPB - 1) / SRC2_TPB); }

struct Layout : StagedLayout {
    size_t total_staged;
    size_t off_rec, off_qstar, off_tflag, off_list_act, off_list_rec, off_counters, total_fused;
};

inline Layout layout(int mx, int my) {
    Layout L;
    static_cast<StagedLayout&>(L) = staged_layout(mx, my);
    L.total_staged = L.StagedLayout::total;
    // the fused step needs the cell records and the updated state before src2
    L.off_rec = 0;
    L.off_qstar = align256((size_t)NREC * L.npad * 8);
    L.off_tflag = L.off_qstar + align256((size_t)5 * mx * my * 8);
    const size_t ntiles = (size_t)((mx + TILE_X - 1) / TILE_X) * (size_t)((my + TILE_Y - 1) / TILE_Y);
    // the tile lists of the step without a branch log, then the queue and
    // list counters
    L.off_list_act = L.off_tflag + align256(ntiles * 4);
    L.off_list_rec = L.off_list_act + align256(ntiles * 4);
    L.off_counters = L.off_list_rec + align256(ntiles * 4);
    L.total_fused = L.off_counters + 256;
    L.total = L.total_staged > L.total_fused ? L.total_staged : L.total_fused;
    return L;
}

inline int cuda_status() {
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? DCLAW_OK : DCLAW_ERR_CUDA;
}

// the tile kernel's dynamic shared memory above 48 KB must be opted into
// once per device (function attributes belong to the device's context)
inline int ensure_tile_smem_attr() {
    static std::atomic<bool> done[MAX_DEVICES];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) return DCLAW_ERR_CUDA;
    if (!done[dev].load(std::memory_order_acquire)) {
        std::lock_guard<std::mutex> lock(g_setup_mu);
        if (!done[dev].load(std::memory_order_relaxed)) {
            const int bytes = (int)TileGeom<TILE_X, TILE_Y>::SMEM_BYTES;
            if (cudaFuncSetAttribute(k_tile<TILE_X, TILE_Y, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     bytes) != cudaSuccess ||
                cudaFuncSetAttribute(k_tile<TILE_X, TILE_Y, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     bytes) != cudaSuccess ||
                cudaFuncSetAttribute(k_tile_list<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) !=
                    cudaSuccess ||
                cudaFuncSetAttribute(k_tile_list<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) != cudaSuccess)
                return DCLAW_ERR_CUDA;
            done[dev].store(true, std::memory_order_release);
        }
    }
    return DCLAW_OK;
}

inline bool sizes_ok(int mx, int my) {
    return mx >= 2 && my >= 2 && (long long)(mx + 4) * (my + 4) < (1LL << 40);
}

// ---- the host-buffer step: bands of tile rows ------------------------------
// Band g holds tile rows T[g] .. T[g+1]-1 (cell rows 1 + T[g] TY .. T[g+1] TY).
// Its tiles read the records of rows up to T[g+1] TY + 2 (and only those
// records mark their flags); the record of row j reads the input rows
// j - 1 .. j + 1. So once the input rows up to T[g+1] TY + 3 are on the
// device, the band's records, tiles and src2 can run while later rows are
// still uploading, and its rows can download while later bands compute.
constexpr int MAX_HOST_BANDS = 64;

inline int host_auto_bands(int mx, int my) {
    const int nty = (my + TILE_Y - 1) / TILE_Y;
    // about 28 MB of state per band: enough work per band to fill the GPU
    // and few enough launches and copies, fine enough that the first upload
    // and the last download (the parts that do not overlap) stay short. On
    // the 4096^2 state (24 bands) the step then takes 15.2 ms, 1.03x the
    // bare copies both ways at once (14.7 ms); 12, 17, 20, 28 and 32 bands
    // took 15.7, 15.5, 15.2, 15.5 and 15.6 ms, 4 bands 1.25x, 64 bands 1.22x.
    const double state = 40.0 * mx * (double)my;
    int nb = (int)(state / 28.0e6) + 1;
    if (nb > MAX_HOST_BANDS) nb = MAX_HOST_BANDS;
    if (nb > nty) nb = nty;
    return nb < 1 ? 1 : nb;
}

// first tile row of each band (first[0..nb], first[nb] = tile rows)
inline void host_band_plan(int my, int nb, int* first) {
    const int nty = (my + TILE_Y - 1) / TILE_Y;
    for (int g = 0; g <= nb; ++g) first[g] = (int)((long long)g * nty / nb);
}

struct HostPipe {
    cudaStream_t up = nullptr, down = nullptr;
    cudaEvent_t ev_start = nullptr, ev_end = nullptr;
    cudaEvent_t ev_up[MAX_HOST_BANDS] = {}, ev_cmp[MAX_HOST_BANDS] = {};
    bool ready = false;
};
static HostPipe g_pipe[MAX_DEVICES];
static std::mutex g_pipe_mu;

// the two copy streams and the events of the current device, created on
// first use and kept for the process
inline HostPipe* host_pipe() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) return nullptr;
    HostPipe& hp = g_pipe[dev];
    if (!hp.ready) {
        const unsigned fl = cudaEventDisableTiming;
        bool ok = cudaStreamCreateWithFlags(&hp.up, cudaStreamNonBlocking) == cudaSuccess &&
                  cudaStreamCreateWithFlags(&hp.down, cudaStreamNonBlocking) == cudaSuccess &&
                  cudaEventCreateWithFlags(&hp.ev_start, fl) == cudaSuccess &&
                  cudaEventCreateWithFlags(&hp.ev_end, fl) == cudaSuccess;
        for (int k = 0; ok && k < MAX_HOST_BANDS; ++k)
            ok = cudaEventCreateWithFlags(&hp.ev_up[k], fl) == cudaSuccess &&
                 cudaEventCreateWithFlags(&hp.ev_cmp[k], fl) == cudaSuccess;
        if (!ok) return nullptr;
        hp.ready = true;
    }
    return &hp;
}

inline size_t host_state_bytes(int mx, int my) { return align256((size_t)5 * mx * my * 8); }

// rows lo .. hi (1-based, inclusive) of the five planes of a state
inline cudaError_t copy_rows(double* dst, const double* src, int mx, int my, int lo, int hi, cudaMemcpyKind kind,
                             cudaStream_t s) {
    if (lo > hi) return cudaSuccess;
    const size_t plane = (size_t)mx * my, off = (size_t)(lo - 1) * mx, n = (size_t)(hi - lo + 1) * mx;
    for (int m = 0; m < 5; ++m) {
        cudaError_t e = cudaMemcpyAsync(dst + m * plane + off, src + m * plane + off, n * 8, kind, s);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace dclaw

using namespace dclaw;

extern "C" {

int dclaw_abi_version(void) { return DCLAW_ABI_VERSION; }

const char* dclaw_error_string(int code) {
    switch (code) {
        case DCLAW_OK: return "ok";
        case DCLAW_ERR_ARG: return "invalid argument";
        case DCLAW_ERR_UNSUPPORTED: return "unsupported option";
        case DCLAW_ERR_NAN: return "NaN in the state";
        case DCLAW_ERR_CUDA: return "CUDA error";
        case DCLAW_ERR_WORKSPACE: return "workspace too small";
        case DCLAW_ERR_TOO_LARGE: return "size beyond the fixed limit";
        default: return "unknown error";
    }
}

void dclaw_params_default(dclaw_params* p) {
    if (!p) return;
    memset(p, 0, sizeof(*p));
    p->grav = 9.81;
    p->dry_tolerance = 1.0e-3;
    p->speed_limit = 1.0e6;
    p->friction_forcing = 0;
    p->dd_manning = 0;
    p->manning_coefficient = 0.0;
    p->friction_depth = 1.0e6;
    p->manning_max = 0.06;
    p->rho_s = 2700.0;
    p->rho_f = 1000.0;
    p->m_crit = 0.64;
    p->m0 = 0.62;
    p->mref = 0.60;
    p->kref = 1.0e-10;
    p->phi = 32.0 * 3.14159265358979323846 / 180.0;
    p->delta = 0.01;
    p->mu = 0.005;
    p->alpha_c = 0.01;
    p->c1 = 1.0;
    p->sigma_0 = 1.0e3;
    p->theta_input = 0.0;
    p->src2method = 0;
    p->alphamethod = 0;
    p->rarecorrectortest = 0;
    p->order = 2;
    p->transverse_waves = 2;
    p->limiter = 4;
    p->bc_lower[0] = p->bc_lower[1] = DCLAW_BC_WALL;
    p->bc_upper[0] = p->bc_upper[1] = DCLAW_BC_WALL;
    p->cfl_desired = 0.9;
    p->cfl_max = 1.0;
    p->dt_max = 1.0e99;
    p->beta_seg = 0.0;
    p->delta_kr_order = 2.0;
    p->chie = 0.5;
    p->me = 0.65;
    p->entrainment_rate = 0.2;
    p->entrainment_method = 1;
}

int dclaw_params_check(const dclaw_params* p) {
    if (!p) return DCLAW_ERR_ARG;
    if (p->bed_normal != 0 || p->curvature != 0) return DCLAW_ERR_UNSUPPORTED;
    if ((p->entrainment != 0 && p->entrainment != 1) || (p->segregation != 0 && p->segregation != 1))
        return DCLAW_ERR_ARG;
    if (p->entrainment_method != 0 && p->entrainment_method != 1) return DCLAW_ERR_ARG;
    if (p->src2method < -1 || p->src2method > 2) return DCLAW_ERR_UNSUPPORTED;
    if (p->alphamethod != 0 && p->alphamethod != 1) return DCLAW_ERR_ARG;
    // the setrun writer's parameter conflict check (src/python/dclaw/data.py:362-365)
    if (p->src2method == 2 && p->alphamethod < 1) return DCLAW_ERR_ARG;
    if (p->order != 1 && p->order != 2) return DCLAW_ERR_ARG;
    if (p->transverse_waves < 0 || p->transverse_waves > 2) return DCLAW_ERR_ARG;
    if (p->limiter < 0 || p->limiter > 5) return DCLAW_ERR_ARG;
    for (int k = 0; k < 2; ++k) {
        if (p->bc_lower[k] != DCLAW_BC_WALL && p->bc_lower[k] != DCLAW_BC_EXTRAP) return DCLAW_ERR_ARG;
        if (p->bc_upper[k] != DCLAW_BC_WALL && p->bc_upper[k] != DCLAW_BC_EXTRAP) return DCLAW_ERR_ARG;
    }
    if (!(p->grav > 0.0) || !(p->dry_tolerance > 0.0) || !(p->rho_f > 0.0) || !(p->rho_s > 0.0)) return DCLAW_ERR_ARG;
    if (!(p->alpha_c > 0.0) || !(p->cfl_desired > 0.0) || !(p->dt_max > 0.0)) return DCLAW_ERR_ARG;
    return DCLAW_OK;
}

int dclaw_params_check_5(const dclaw_params* p) {
    const int rc = dclaw_params_check(p);
    if (rc) return rc;
    if (p->entrainment != 0 || p->segregation != 0) return DCLAW_ERR_UNSUPPORTED;
    return DCLAW_OK;
}

size_t dclaw_workspace_bytes(int mx, int my) {
    if (!sizes_ok(mx, my)) return 0;
    return layout(mx, my).total;
}

int dclaw_clock_init(dclaw_clock* clock, double t, double dt, double t_final, int fixed_dt, void* stream) {
    if (!clock) return DCLAW_ERR_ARG;
    k_clock_init<<<1, 32, 0, (cudaStream_t)stream>>>(clock, t, dt, t_final, fixed_dt);
    return cuda_status();
}

int dclaw_clock_set_obs(dclaw_clock* clock, double t_obs, void* stream) {
    if (!clock || !(t_obs >= 0.0)) return DCLAW_ERR_ARG;
    k_clock_set_obs<<<1, 32, 0, (cudaStream_t)stream>>>(clock, t_obs);
    return cuda_status();
}

int dclaw_step(const double* q_in, double* q_out, const double* b, int mx, int my, double dx, double dy,
               const dclaw_params* p, dclaw_clock* clock, void* work, size_t work_bytes, uint32_t* branch_log,
               void* stream) {
    if (!q_in || !q_out || !b || !p || !clock || !work || q_in == q_out) return DCLAW_ERR_ARG;
    if (!sizes_ok(mx, my) || !(dx > 0.0) || !(dy > 0.0)) return DCLAW_ERR_ARG;
    int rc = dclaw_params_check_5(p);
    if (rc) return rc;
    Layout L = layout(mx, my);
    if (work_bytes < L.total_fused) return DCLAW_ERR_WORKSPACE;
    cudaStream_t s = (cudaStream_t)stream;
    Geom g{mx, my, mx + 4, my + 4, dx, dy};
    Rec R{(double*)((char*)work + L.off_rec), L.npad};
    const dclaw_params P = *p;
    using TG = TileGeom<TILE_X, TILE_Y>;
    if (ensure_tile_smem_attr() != DCLAW_OK) return DCLAW_ERR_CUDA;
    if (branch_log) {
        size_t nlog = (size_t)(my + 2) * (mx + 1) + (size_t)(mx + 2) * (my + 1);
        cudaMemsetAsync(branch_log, 0, nlog * sizeof(uint32_t), s);
    }
    uint32_t* tflag = (uint32_t*)((char*)work + L.off_tflag);
    const int ntx = (mx + TILE_X - 1) / TILE_X, nty = (my + TILE_Y - 1) / TILE_Y;
    if (!branch_log) {
        // over the tile lists (the branch log needs every interface's bits,
        // so it keeps the full-grid kernels below)
        const int nsm = sm_count();
        if (nsm <= 0) return DCLAW_ERR_CUDA;
        unsigned int* counters = (unsigned int*)((char*)work + L.off_counters);
        uint32_t* list_act = (uint32_t*)((char*)work + L.off_list_act);
        uint32_t* list_rec = (uint32_t*)((char*)work + L.off_list_rec);
        double* qstar = (double*)((char*)work + L.off_qstar);
        const long long ncell = (long long)mx * my;
        const unsigned ntiles = (unsigned)ntx * (unsigned)nty;
        unsigned g0 = (unsigned)(nsm * DCLAW_SCAN_MINB * 2);
        if ((long long)g0 * TPB > ncell) g0 = nblocks(ncell);
        k_scan_patch<<<g0, TPB, 0, s>>>(P, mx, my, q_in, q_out, clock, counters, tflag, 0, (size_t)ncell, 0,
                                        (size_t)ncell);
        k_list_patch<<<(ntiles + TPB - 1) / TPB, TPB, 0, s>>>(ntx, nty, clock, tflag, counters, list_act, list_rec, 0,
                                                             nty - 1);
        unsigned g1 = (unsigned)(nsm * RECORDS_MINB);
        if (g1 > ntiles) g1 = ntiles;
        k_records_list<<<g1, RECORDS_TPB, 0, s>>>(P, g, q_in, b, R, counters, list_rec);
        unsigned g2 = (unsigned)(nsm * DCLAW_TILE_MINBLOCKS);
        if (g2 > ntiles) g2 = ntiles;
        if (!DCLAW_LIST_SRC2_KERNEL) {
            k_tile_list<true><<<g2, TILE_TPB, TG::SMEM_BYTES, s>>>(P, g, R, b, q_out, clock, counters, list_act);
            return cuda_status();
        }
        k_tile_list<false><<<g2, TILE_TPB, TG::SMEM_BYTES, s>>>(P, g, R, b, qstar, clock, counters, list_act);
        unsigned g3 = (unsigned)(nsm * SRC2_MINB);
        if (g3 > ntiles) g3 = ntiles;
        k_src2_list<<<g3, SRC2_TPB, 0, s>>>(P, g, qstar, q_out, clock, counters, list_act);
        return cuda_status();
    }
    k_records<<<nblocks((long long)L.npad), TPB, 0, s>>>(P, g, q_in, b, R, clock, tflag);
    dim3 grid(ntx, nty);
    if (DCLAW_SRC2_KERNEL) {
        double* qstar = (double*)((char*)work + L.off_qstar);
        k_tile<TILE_X, TILE_Y, false><<<grid, TILE_TPB, TG::SMEM_BYTES, s>>>(P, g, R, b, qstar, clock, branch_log,
                                                                             tflag);
        k_src2_cells<<<src2_blocks((long long)mx * my), SRC2_TPB, 0, s>>>(P, g, qstar, q_out, clock, tflag);
    } else {
        k_tile<TILE_X, TILE_Y, true><<<grid, TILE_TPB, TG::SMEM_BYTES, s>>>(P, g, R, b, q_out, clock, branch_log,
                                                                            tflag);
    }
    return cuda_status();
}

size_t dclaw_step_host_workspace_bytes(int mx, int my) {
    if (!sizes_ok(mx, my)) return 0;
    return align256(layout(mx, my).total_fused) + 2 * host_state_bytes(mx, my);
}

int dclaw_step_host_bands(int mx, int my, int nbands, int32_t* first, int max) {
    if (!sizes_ok(mx, my) || nbands < 0) return 0;
    const int nty = (my + TILE_Y - 1) / TILE_Y;
    int nb = nbands == 0 ? host_auto_bands(mx, my) : (nbands > nty ? nty : nbands);
    if (nb > MAX_HOST_BANDS) nb = MAX_HOST_BANDS;
    int f[MAX_HOST_BANDS + 1];
    host_band_plan(my, nb, f);
    for (int g = 0; first && g <= nb && g < max; ++g) first[g] = f[g];
    return nb;
}

int dclaw_step_host(const double* q_in, double* q_out, const double* b, int mx, int my, double dx, double dy,
                    const dclaw_params* p, dclaw_clock* clock, void* work, size_t work_bytes, int nbands,
                    void* stream) {
    if (!q_in || !q_out || !b || !p || !clock || !work || nbands < 0) return DCLAW_ERR_ARG;
    if (!sizes_ok(mx, my) || !(dx > 0.0) || !(dy > 0.0)) return DCLAW_ERR_ARG;
    int rc = dclaw_params_check_5(p);
    if (rc) return rc;
    if (work_bytes < dclaw_step_host_workspace_bytes(mx, my)) return DCLAW_ERR_WORKSPACE;
    if (ensure_tile_smem_attr() != DCLAW_OK) return DCLAW_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_pipe_mu);
    HostPipe* hp = host_pipe();
    if (!hp) return DCLAW_ERR_CUDA;
    int first[MAX_HOST_BANDS + 1];
    const int nb = dclaw_step_host_bands(mx, my, nbands, first, MAX_HOST_BANDS + 1);
    Layout L = layout(mx, my);
    cudaStream_t s = (cudaStream_t)stream;
    Geom g{mx, my, mx + 4, my + 4, dx, dy};
    Rec R{(double*)((char*)work + L.off_rec), L.npad};
    const dclaw_params P = *p;
    using TG = TileGeom<TILE_X, TILE_Y>;
    uint32_t* tflag = (uint32_t*)((char*)work + L.off_tflag);
    double* qstar = (double*)((char*)work + L.off_qstar);
    double* dq_in = (double*)((char*)work + align256(L.total_fused));
    double* dq_out = (double*)((char*)dq_in + host_state_bytes(mx, my));
    const int ntx = (mx + TILE_X - 1) / TILE_X;
    cudaError_t e = cudaSuccess;
    // the copy streams start after the work queued on the caller's stream
    // (the previous step still reads the device copies)
    if (e == cudaSuccess) e = cudaEventRecord(hp->ev_start, s);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(hp->up, hp->ev_start, 0);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(hp->down, hp->ev_start, 0);
    // uploads: band g brings the input rows its compute needs
    int lo = 1;
    for (int k = 0; k < nb && e == cudaSuccess; ++k) {
        const int hi = k == nb - 1 ? my : (first[k + 1] * TILE_Y + 3 < my ? first[k + 1] * TILE_Y + 3 : my);
        e = copy_rows(dq_in, q_in, mx, my, lo, hi, cudaMemcpyHostToDevice, hp->up);
        if (e == cudaSuccess) e = cudaEventRecord(hp->ev_up[k], hp->up);
        lo = hi + 1 > lo ? hi + 1 : lo;
    }
    // compute on the caller's stream, downloads behind it
    int ja = -1;
    for (int k = 0; k < nb && e == cudaSuccess; ++k) {
        e = cudaStreamWaitEvent(s, hp->ev_up[k], 0);
        if (e != cudaSuccess) break;
        const int jb = k == nb - 1 ? my + 2 : (first[k + 1] * TILE_Y + 2 < my + 2 ? first[k + 1] * TILE_Y + 2 : my + 2);
        if (jb >= ja) {
            const int nrow = jb - ja + 1;
            k_records<<<nblocks((long long)g.PX * nrow), TPB, 0, s>>>(P, g, dq_in, b, R, clock, tflag, ja + 1, nrow);
            ja = jb + 1;
        }
        const int nty = first[k + 1] - first[k];
        const int r0 = 1 + first[k] * TILE_Y, r1 = first[k + 1] * TILE_Y < my ? first[k + 1] * TILE_Y : my;
        if (nty > 0) {
            dim3 grid(ntx, nty);
            k_tile<TILE_X, TILE_Y, false><<<grid, TILE_TPB, TG::SMEM_BYTES, s>>>(P, g, R, b, qstar, clock, nullptr,
                                                                                 tflag, first[k]);
            const long long nc = (long long)(r1 - r0 + 1) * mx;
            k_src2_cells<<<src2_blocks(nc), SRC2_TPB, 0, s>>>(P, g, qstar, dq_out, clock, tflag, (long long)(r0 - 1) * mx, nc,
                                                     0);
        }
        if (k == nb - 1) k_tick<<<1, 32, 0, s>>>(P, clock);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaEventRecord(hp->ev_cmp[k], s);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(hp->down, hp->ev_cmp[k], 0);
        if (e == cudaSuccess && nty > 0) e = copy_rows(q_out, dq_out, mx, my, r0, r1, cudaMemcpyDeviceToHost, hp->down);
    }
    // the caller's stream resumes after the last download
    if (e == cudaSuccess) e = cudaEventRecord(hp->ev_end, hp->down);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s, hp->ev_end, 0);
    return e == cudaSuccess ? cuda_status() : DCLAW_ERR_CUDA;
}

int dclaw_rows_granule(void) { return TILE_Y; }

int dclaw_step_rows(const double* q_in, double* q_out, const double* b, int mx, int my, double dx, double dy,
                    const dclaw_params* p, dclaw_clock* clock, void* work, size_t work_bytes, int row_first,
                    int row_count, void* stream) {
    if (!q_in || !q_out || !b || !p || !clock || !work || q_in == q_out) return DCLAW_ERR_ARG;
    if (!sizes_ok(mx, my) || !(dx > 0.0) || !(dy > 0.0)) return DCLAW_ERR_ARG;
    // whole tile rows: the first row starts a tile row and the range ends on
    // a tile-row boundary or at the patch's last row
    const int last = row_first + row_count - 1;
    if (row_first < 1 || row_count < 1 || last > my || (row_first - 1) % TILE_Y != 0 ||
        (last != my && last % TILE_Y != 0))
        return DCLAW_ERR_ARG;
    int rc = dclaw_params_check_5(p);
    if (rc) return rc;
    Layout L = layout(mx, my);
    if (work_bytes < L.total_fused) return DCLAW_ERR_WORKSPACE;
    if (ensure_tile_smem_attr() != DCLAW_OK) return DCLAW_ERR_CUDA;
    cudaStream_t s = (cudaStream_t)stream;
    Geom g{mx, my, mx + 4, my + 4, dx, dy};
    Rec R{(double*)((char*)work + L.off_rec), L.npad};
    const dclaw_params P = *p;
    using TG = TileGeom<TILE_X, TILE_Y>;
    uint32_t* tflag = (uint32_t*)((char*)work + L.off_tflag);
    double* qstar = (double*)((char*)work + L.off_qstar);
    // dclaw_step's kernels over tile lists, restricted to the range: the scan
    // of its rows and the 3 either side (the cells its tiles' marks depend
    // on; the range's rows of q_out are zeroed), the active tiles of its
    // tile rows, the records of those and their neighbours (one tile row
    // beyond, 13 >= 3 rows), the tiles, their cells' src2; no tick
    const int sm = sm_count();
    if (sm <= 0) return DCLAW_ERR_CUDA;
    unsigned int* counters = (unsigned int*)((char*)work + L.off_counters);
    uint32_t* list_act = (uint32_t*)((char*)work + L.off_list_act);
    uint32_t* list_rec = (uint32_t*)((char*)work + L.off_list_rec);
    const int ntx = (mx + TILE_X - 1) / TILE_X, ntyp = (my + TILE_Y - 1) / TILE_Y;
    const unsigned ntiles = (unsigned)ntx * (unsigned)ntyp;
    const int ty0 = (row_first - 1) / TILE_Y, ty1 = (last - 1) / TILE_Y;
    const int sa = row_first - 3 > 1 ? row_first - 3 : 1, sb = last + 3 < my ? last + 3 : my;
    const long long nscan = (long long)(sb - sa + 1) * mx;
    unsigned g0 = (unsigned)(sm * DCLAW_SCAN_MINB * 2);
    if ((long long)g0 * TPB > nscan) g0 = nblocks(nscan);
    k_scan_patch<<<g0, TPB, 0, s>>>(P, mx, my, q_in, q_out, clock, counters, tflag, (size_t)(sa - 1) * mx,
                                    (size_t)sb * mx, (size_t)(row_first - 1) * mx, (size_t)last * mx);
    k_list_patch<<<(ntiles + TPB - 1) / TPB, TPB, 0, s>>>(ntx, ntyp, clock, tflag, counters, list_act, list_rec, ty0,
                                                         ty1);
    unsigned g1 = (unsigned)(sm * RECORDS_MINB);
    if (g1 > ntiles) g1 = ntiles;
    k_records_list<<<g1, RECORDS_TPB, 0, s>>>(P, g, q_in, b, R, counters, list_rec);
    unsigned g2 = (unsigned)(sm * DCLAW_TILE_MINBLOCKS);
    if (g2 > ntiles) g2 = ntiles;
    k_tile_list<false><<<g2, TILE_TPB, TG::SMEM_BYTES, s>>>(P, g, R, b, qstar, clock, counters, list_act);
    unsigned g3 = (unsigned)(sm * SRC2_MINB);
    if (g3 > ntiles) g3 = ntiles;
    k_src2_list<<<g3, SRC2_TPB, 0, s>>>(P, g, qstar, q_out, clock, counters, list_act, 0);
    return cuda_status();
}

int dclaw_clock_tick(dclaw_clock* clock, const dclaw_params* p, void* stream) {
    if (!clock || !p) return DCLAW_ERR_ARG;
    int rc = dclaw_params_check_5(p);
    if (rc) return rc;
    k_tick<<<1, 32, 0, (cudaStream_t)stream>>>(*p, clock);
    return cuda_status();
}

int dclaw_bc2amr(double* q, int mx, int my, int mbc, const dclaw_params* p, void* stream) {
    if (!q || !p || mbc != 2 || !sizes_ok(mx, my)) return DCLAW_ERR_ARG;
    int rc = dclaw_params_check_5(p);
    if (rc) return rc;
    k_bc2amr<<<nblocks((long long)(mx + 4) * (my + 4)), TPB, 0, (cudaStream_t)stream>>>(*p, mx, my, q);
    return cuda_status();
}

int dclaw_setaux(double* aux, int mx, int my, int mbc, const dclaw_params* p, void* stream) {
    if (!aux || !p || mbc != 2 || !sizes_ok(mx, my)) return DCLAW_ERR_ARG;
    k_setaux<<<nblocks((long long)(mx + 4) * (my + 4)), TPB, 0, (cudaStream_t)stream>>>(*p, mx, my, aux);
    return cuda_status();
}

int dclaw_b4step2(double* q, double* aux, int mx, int my, int mbc, double dx, double dy, double t, double dt,
                  const dclaw_params* p, dclaw_clock* clock, void* stream) {
    (void)t; (void)dt;
    if (!q || !aux || !p || mbc != 2 || !sizes_ok(mx, my) || !(dx > 0.0) || !(dy > 0.0)) return DCLAW_ERR_ARG;
    int rc = dclaw_params_check_5(p);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    const size_t npad = (size_t)(mx + 4) * (my + 4);
    k_b4_padded<<<nblocks((long long)npad), TPB, 0, s>>>(*p, mx, my, q, clock);
    Geom g{mx, my, mx + 4, my + 4, dx, dy};
    Work W{};
    W.qB = q;
    W.bP = aux;
    W.td = aux + 3 * npad;
    W.npad = npad;
    k_taudir<<<nblocks((long long)npad), TPB, 0, s>>>(*p, g, W, 1);
    return cuda_status();
}

int dclaw_step2(double* q, const double* aux, int mx, int my, int mbc, double dx, double dy, double dt,
                const dclaw_params* p, dclaw_clock* clock, double* fluxes, void* work, size_t work_bytes,
                void* stream) {
    if (!q || !aux || !p || !clock || !work || mbc != 2 || !sizes_ok(mx, my) || !(dx > 0.0) || !(dy > 0.0))
        return DCLAW_ERR_ARG;
    int rc = dclaw_params_check_5(p);
    if (rc) return rc;
    Layout L = layout(mx, my);
    if (work_bytes < L.total_staged) return DCLAW_ERR_WORKSPACE;
    cudaStream_t s = (cudaStream_t)stream;
    Geom g{mx, my, mx + 4, my + 4, dx, dy};
    Work W = make_work(work, L);
    W.qB = q;
    W.bP = const_cast<double*>(aux);
    W.td = const_cast<double*>(aux) + 3 * L.npad;
    // the kernels read dt from the clock: use a clock set to this dt
    k_clock_init<<<1, 32, 0, s>>>(clock, 0.0, dt, 0.0, 1);
    const dclaw_params P = *p;
    k_riemann<0><<<nblocks((long long)L.nxi), TPB, 0, s>>>(P, g, W, clock, nullptr);
    k_riemann<1><<<nblocks((long long)(mx + 2) * (my + 3)), TPB, 0, s>>>(P, g, W, clock, nullptr);
    k_flux<0><<<nblocks((long long)(mx + 1) * (my + 2)), TPB, 0, s>>>(P, g, W, clock, nullptr);
    k_flux<1><<<nblocks((long long)(mx + 2) * (my + 1)), TPB, 0, s>>>(P, g, W, clock, nullptr);
    k_update_padded<<<nblocks((long long)mx * my), TPB, 0, s>>>(g, W, dt, q, fluxes, clock);
    k_cfl_from_bits<<<1, 32, 0, s>>>(clock);
    return cuda_status();
}

int dclaw_src2(double* q, const double* aux, int mx, int my, int mbc, double dx, double dy, double t, double dt,
               const dclaw_params* p, void* stream) {
    (void)aux; (void)dx; (void)dy; (void)t;
    if (!q || !p || mbc != 2 || !sizes_ok(mx, my)) return DCLAW_ERR_ARG;
    int rc = dclaw_params_check_5(p);
    if (rc) return rc;
    k_src2_padded<<<nblocks((long long)mx * my), TPB, 0, (cudaStream_t)stream>>>(*p, mx, my, dt, q);
    return cuda_status();
}

int dclaw_obs_record(const dclaw_clock* clocks, int n_clocks, const int32_t* member, const double* q,
                     const int64_t* select, int64_t n_select, int n_obs, int step, double* out,
                     int32_t* out_step, void* stream) {
    if (!clocks || n_clocks <= 0 || !q || n_select <= 0 || n_obs <= 0 || !out || !out_step) return DCLAW_ERR_ARG;
    if (n_clocks > 1 && !member) return DCLAW_ERR_ARG;
    const long long work = n_select > n_clocks ? (long long)n_select : (long long)n_clocks;
    long long nb = (work + TPB - 1) / TPB;
    if (nb > 4096) nb = 4096;
    k_obs_record<<<(unsigned)nb, TPB, 0, (cudaStream_t)stream>>>(clocks, n_clocks, member, q, select,
                                                                 (long long)n_select, n_obs, step, out, out_step);
    return cuda_status();
}

int dclaw_peak_update(const double* h, double* hmax, int32_t* argstep, int64_t n, int step, void* stream) {
    if (!h || !hmax || !argstep || n <= 0) return DCLAW_ERR_ARG;
    long long nb = ((long long)n + TPB - 1) / TPB;
    if (nb > 65535) nb = 65535;
    k_peak_update<<<(unsigned)nb, TPB, 0, (cudaStream_t)stream>>>(h, hmax, argstep, (long long)n, step);
    return cuda_status();
}

int dclaw_peak_adjoint(const double* g, const int32_t* argstep, int64_t n, int step, double* lam_h,
                       void* stream) {
    if (!g || !argstep || !lam_h || n <= 0) return DCLAW_ERR_ARG;
    long long nb = ((long long)n + TPB - 1) / TPB;
    if (nb > 65535) nb = 65535;
    k_peak_adjoint<<<(unsigned)nb, TPB, 0, (cudaStream_t)stream>>>(g, argstep, (long long)n, step, lam_h);
    return cuda_status();
}

int dclaw_fields_from_fortran(const double* fortran, int nf_fortran, int nf, int mx, int my, int mbc,
                              double* planes, void* stream) {
    if (!fortran || !planes || nf < 1 || nf > nf_fortran || mx < 1 || my < 1 || mbc < 0) return DCLAW_ERR_ARG;
    const long long ncell = (long long)(mx + 2 * mbc) * (my + 2 * mbc);
    long long nb = (ncell + TPB - 1) / TPB;
    if (nb > 65535) nb = 65535;
    k_fields_soa<<<(unsigned)nb, TPB, 0, (cudaStream_t)stream>>>(fortran, nf_fortran, nf, ncell, planes);
    return cuda_status();
}

int dclaw_fields_to_fortran(const double* planes, int nf, int nf_fortran, int mx, int my, int mbc,
                            double* fortran, void* stream) {
    if (!fortran || !planes || nf < 1 || nf > nf_fortran || mx < 1 || my < 1 || mbc < 0) return DCLAW_ERR_ARG;
    const long long ncell = (long long)(mx + 2 * mbc) * (my + 2 * mbc);
    long long nb = (ncell + TPB - 1) / TPB;
    if (nb > 65535) nb = 65535;
    k_fields_aos<<<(unsigned)nb, TPB, 0, (cudaStream_t)stream>>>(planes, nf, nf_fortran, ncell, fortran);
    return cuda_status();
}

int dclaw_max_wave_speed(const double* q, int mx, int my, const dclaw_params* p, double* smax, void* stream) {
    if (!q || !p || !smax || !sizes_ok(mx, my)) return DCLAW_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    cudaMemsetAsync(smax, 0, sizeof(double), s);
    k_wave_speed<<<nblocks((long long)mx * my), TPB, 0, s>>>(*p, mx, my, q, (unsigned long long*)smax);
    return cuda_status();
}

}  // extern "C"

extern "C" {

// the full-state workspace: the staged planes (full_layout), then the tile
// flags of the skip
inline size_t full_tflag_bytes(int mx, int my) {
    return align256((size_t)((mx + TILE_X - 1) / TILE_X) * (size_t)((my + TILE_Y - 1) / TILE_Y) * 4);
}

size_t dclaw_step_full_workspace_bytes(int mx, int my) {
    if (!sizes_ok(mx, my)) return 0;
    return full_layout(mx, my).total + full_tflag_bytes(mx, my);
}

int dclaw_step_full(const double* q_in, double* q_out, const double* b, const double* h_e, int mx, int my,
                    double dx, double dy, const dclaw_params* p, dclaw_clock* clock, void* work, size_t work_bytes,
                    uint32_t* branch_log, void* stream) {
    if (!q_in || !q_out || !b || !p || !clock || !work || q_in == q_out) return DCLAW_ERR_ARG;
    if (!sizes_ok(mx, my) || !(dx > 0.0) || !(dy > 0.0)) return DCLAW_ERR_ARG;
    int rc = dclaw_params_check(p);
    if (rc) return rc;
    if (p->entrainment == 1 && p->entrainment_method == 0 && !h_e) return DCLAW_ERR_ARG;
    const FullLayout L = full_layout(mx, my);
    if (work_bytes < L.total + full_tflag_bytes(mx, my)) return DCLAW_ERR_WORKSPACE;
    cudaStream_t s = (cudaStream_t)stream;
    Geom g{mx, my, mx + 4, my + 4, dx, dy};
    WorkF W = make_work_full(work, L);
    // with a branch log every interface is computed (its bits are logged)
    uint32_t* tflag = branch_log ? nullptr : (uint32_t*)((char*)work + L.total);
    const dclaw_params P = *p;
    if (branch_log) {
        size_t nlog = (size_t)(my + 2) * (mx + 1) + (size_t)(mx + 2) * (my + 1);
        cudaMemsetAsync(branch_log, 0, nlog * sizeof(uint32_t), s);
    }
    const long long npad = (long long)g.PX * g.PY;
    k_full_b4<<<nblocks(npad), TPB, 0, s>>>(P, g, q_in, b, W, clock, tflag);
    k_full_taudir<<<nblocks(npad), TPB, 0, s>>>(P, g, W);
    k_full_riemann<0><<<nblocks((long long)(mx + 3) * (my + 2)), TPB, 0, s>>>(P, g, W, clock, branch_log, tflag);
    k_full_riemann<1><<<nblocks((long long)(mx + 2) * (my + 3)), TPB, 0, s>>>(P, g, W, clock, branch_log, tflag);
    k_full_flux<0><<<nblocks((long long)(mx + 1) * (my + 2)), TPB, 0, s>>>(P, g, W, clock, branch_log, tflag);
    k_full_flux<1><<<nblocks((long long)(mx + 2) * (my + 1)), TPB, 0, s>>>(P, g, W, clock, branch_log, tflag);
    k_full_final<<<nblocks((long long)mx * my), TPB, 0, s>>>(P, g, W, h_e, q_out, clock, tflag);
    return cuda_status();
}

}  // extern "C"

// ---- allocation-free variant of the fused step ------------------------------
// Scratch for the per-cell records of one patch of at most
// NOALLOC_MAX_CELLS padded cells, in a fixed device array of this library
// (NREC * 2^18 doubles = 28 MiB per device). Host code must not use the
// symbol as an address: it is a host-side stand-in; the device address is
// looked up once per device with cudaGetSymbolAddress.
namespace dclaw {
constexpr size_t NOALLOC_MAX_CELLS = (size_t)1 << 18;
static __device__ __align__(256) double g_noalloc_scratch[(size_t)NREC * NOALLOC_MAX_CELLS];
static std::atomic<double*> g_noalloc_addr[MAX_DEVICES];
}  // namespace dclaw

extern "C" {

size_t dclaw_step_noalloc_max_cells(void) { return dclaw::NOALLOC_MAX_CELLS; }

int dclaw_step_noalloc(const double* q_in, double* q_out, const double* b, int mx, int my, double dx, double dy,
                       const dclaw_params* p, dclaw_clock* clock, void* stream) {
    if (!q_in || !q_out || !b || !p || !clock || q_in == q_out) return DCLAW_ERR_ARG;
    if (!sizes_ok(mx, my) || !(dx > 0.0) || !(dy > 0.0)) return DCLAW_ERR_ARG;
    if ((size_t)(mx + 4) * (size_t)(my + 4) > NOALLOC_MAX_CELLS) return DCLAW_ERR_TOO_LARGE;
    int rc = dclaw_params_check_5(p);
    if (rc) return rc;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) return DCLAW_ERR_CUDA;
    double* scratch = g_noalloc_addr[dev].load(std::memory_order_acquire);
    if (!scratch) {
        // set-up on first use on this device (this device is current here),
        // under the set-up lock so that concurrent first calls agree
        std::lock_guard<std::mutex> lock(g_setup_mu);
        scratch = g_noalloc_addr[dev].load(std::memory_order_relaxed);
        if (!scratch) {
            void* addr = nullptr;
            if (cudaGetSymbolAddress(&addr, g_noalloc_scratch) != cudaSuccess || !addr) return DCLAW_ERR_CUDA;
            scratch = static_cast<double*>(addr);
            g_noalloc_addr[dev].store(scratch, std::memory_order_release);
        }
    }
    if (ensure_tile_smem_attr() != DCLAW_OK) return DCLAW_ERR_CUDA;
    // every record plane a tile reads is written by k_records in the same
    // call (h, fsphi and taudir for every padded cell, the other planes for
    // every wet cell, the only cells whose other planes are read), so the
    // previous call's contents need no clearing
    cudaStream_t s = (cudaStream_t)stream;
    Geom g{mx, my, mx + 4, my + 4, dx, dy};
    const size_t npad = (size_t)(mx + 4) * (my + 4);
    Rec R{scratch, npad};
    const dclaw_params P = *p;
    k_records<<<nblocks((long long)npad), TPB, 0, s>>>(P, g, q_in, b, R, clock, nullptr);
    dim3 grid((mx + TILE_X - 1) / TILE_X, (my + TILE_Y - 1) / TILE_Y);
    k_tile<TILE_X, TILE_Y, true><<<grid, TILE_TPB, TileGeom<TILE_X, TILE_Y>::SMEM_BYTES, s>>>(P, g, R, b, q_out, clock,
                                                                                     nullptr, nullptr);
    return cuda_status();
}

}  // extern "C"

extern "C" {

int dclaw_batch_tile_shapes(int32_t* tx, int32_t* ty, int max) {
    int n = 0;
    for (int k = 0; k < NBATCH_SHAPES && k < max; ++k, ++n) {
        if (tx) tx[k] = batch_tx(k);
        if (ty) ty[k] = batch_ty(k);
    }
    return n;
}

int dclaw_batch_layout(int n, const int32_t* mx, const int32_t* my, const double* dx, const double* dy,
                       int tile_shape, dclaw_member* members, dclaw_batch* batch) {
    if (n <= 0 || !mx || !my || !dx || !dy || !members || !batch) return DCLAW_ERR_ARG;
    if (tile_shape < 0 || tile_shape >= NBATCH_SHAPES) return DCLAW_ERR_ARG;
    const int TX = batch_tx(tile_shape), TY = batch_ty(tile_shape);
    uint64_t q = 0, bb = 0, w = 0;
    uint32_t tiles = 0, rch = 0, sch = 0;
    for (int k = 0; k < n; ++k) {
        if (!sizes_ok(mx[k], my[k]) || !(dx[k] > 0.0) || !(dy[k] > 0.0)) return DCLAW_ERR_ARG;
        dclaw_member& M = members[k];
        memset(&M, 0, sizeof(M));
        M.mx = mx[k];
        M.my = my[k];
        M.dx = dx[k];
        M.dy = dy[k];
        const uint64_t cells = (uint64_t)mx[k] * my[k];
        const uint64_t npad = (uint64_t)(mx[k] + 4) * (my[k] + 4);
        M.q_off = q;
        q += 5 * cells;
        M.b_off = bb;
        bb += cells;
        M.rec_off = w;
        w += (uint64_t)NREC * npad;
        M.qs_off = w;
        w += 5 * cells;
        w = (w + 31) & ~(uint64_t)31;  // 256-byte alignment of every member's block
        M.ntiles_x = (uint32_t)((mx[k] + TX - 1) / TX);
        M.ntiles = M.ntiles_x * (uint32_t)((my[k] + TY - 1) / TY);
        M.tile0 = tiles;
        tiles += M.ntiles;
        M.nrchunks = (uint32_t)((npad + TPB - 1) / TPB);
        M.rchunk0 = rch;
        rch += M.nrchunks;
        M.nschunks = (uint32_t)((cells + TPB - 1) / TPB);
        M.schunk0 = sch;
        sch += M.nschunks;
    }
    memset(batch, 0, sizeof(*batch));
    batch->nmembers = n;
    batch->tile_shape = tile_shape;
    batch->tile_ctas_per_sm = 2;
    batch->cell_ctas_per_sm = 8;
    batch->ntiles = tiles;
    batch->nrchunks = rch;
    batch->nschunks = sch;
    batch->q_doubles = q;
    batch->b_doubles = bb;
    // + the active-tile and record-tile lists, the tile activity flags, then
    // the work-queue counters and list lengths
    batch->work_bytes = w * 8 + 3 * align256((size_t)tiles * 4) + 256;
    return DCLAW_OK;
}

int dclaw_batch_reset(const dclaw_batch* batch, void* work, void* stream) {
    if (!batch || !work) return DCLAW_ERR_ARG;
    unsigned int* counters = (unsigned int*)((char*)work + (batch->work_bytes - 256));
    cudaMemsetAsync(counters, 0, 256, (cudaStream_t)stream);
    return cuda_status();
}

int dclaw_step_batched(const dclaw_batch* batch, const dclaw_member* members, const dclaw_params* params,
                       dclaw_clock* clocks, const double* q_in, double* q_out, const double* b, void* work,
                       void* stream) {
    if (!batch || !members || !params || !clocks || !q_in || !q_out || !b || !work || q_in == q_out)
        return DCLAW_ERR_ARG;
    if (batch->nmembers <= 0 || batch->tile_shape < 0 || batch->tile_shape >= NBATCH_SHAPES) return DCLAW_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    const int nsm = sm_count();
    if (nsm <= 0) return DCLAW_ERR_CUDA;
    double* w = (double*)work;
    unsigned int* counters = (unsigned int*)((char*)work + (batch->work_bytes - 256));
    const size_t tbytes = align256((size_t)batch->ntiles * 4);
    uint32_t* tflag = (uint32_t*)((char*)counters - tbytes);
    uint32_t* list_rec = (uint32_t*)((char*)tflag - tbytes);
    uint32_t* list_act = (uint32_t*)((char*)list_rec - tbytes);
    const int cpsm = batch->cell_ctas_per_sm > 0 ? batch->cell_ctas_per_sm : 8;
    const int TX = batch_tx(batch->tile_shape), TY = batch_ty(batch->tile_shape);
    unsigned g0 = (unsigned)(nsm * cpsm);
    if (g0 > batch->nschunks) g0 = batch->nschunks;
    k_scan_batch<<<g0, TPB, 0, s>>>(batch->nmembers, batch->nschunks, members, params, clocks, q_in, q_out, counters,
                                    tflag, TX, TY);
    k_list_batch<<<(unsigned)((batch->ntiles + TPB - 1) / TPB), TPB, 0, s>>>(batch->nmembers, batch->ntiles, members,
                                                                            clocks, tflag, counters, list_act, list_rec);
    int rc = DCLAW_OK;
    switch (batch->tile_shape) {
        case 0: rc = launch_batch_tiles<batch_tx(0), batch_ty(0)>(batch, members, params, clocks, q_in, q_out, b, w, counters, tflag, list_act, list_rec, nsm, cpsm, s); break;
        case 1: rc = launch_batch_tiles<batch_tx(1), batch_ty(1)>(batch, members, params, clocks, q_in, q_out, b, w, counters, tflag, list_act, list_rec, nsm, cpsm, s); break;
        default: rc = launch_batch_tiles<batch_tx(2), batch_ty(2)>(batch, members, params, clocks, q_in, q_out, b, w, counters, tflag, list_act, list_rec, nsm, cpsm, s); break;
    }
    if (rc != DCLAW_OK) return rc;
    k_tick_batch<<<(unsigned)((batch->nmembers + TPB - 1) / TPB), TPB, 0, s>>>(batch->nmembers, params, clocks);
    return cuda_status();
}

}  // extern "C"
