// adjoint.cu -- CUDA kernels and C ABI of the adjoint (vector-Jacobian
// product) of one uniform-patch step, sm_100a, FP64.
//
// dclaw_step_adjoint maps the adjoint of a step's output state, lam_out, to
// the adjoint of its input state, lam_in = (dS/dq)^T lam_out, and adds
// (dS/dtheta)^T lam_out to the adjoints of the material parameters
// theta = (phi [rad], kref, alpha_c, mu). The step's dt is data.
//
// One call (a single patch, or every member of an ensemble) is 20
// launches that work only where the flow is (see "ensembles" below: a
// single patch runs as a one-member ensemble):
//   forward recompute  b4step2, calc_taudir, setvars records of the rpn2
//                      states (tau and its partial derivatives, once per
//                      cell state instead of once per interface side),
//                      x/y solves, x/y fluxes
//                      (the staged step's stages, bit-identical to the fused
//                      step, so every branch is the one the forward took)
//   reverse            src2+update, x/y fluxes, x/y solves, calc_taudir,
//                      b4step2, ghost gather, parameter sum
// Every reverse stage gathers what later stages wrote (no atomics), and the
// parameter adjoints are summed per block and then across blocks in a fixed
// order, so results are bit-reproducible run to run.
#include <cuda_runtime.h>
#include <string.h>

#include "adjoint.cuh"
#include "workspace.cuh"

namespace dclaw {
namespace adj {

// the reverse item functions are register-heavy: small blocks
#ifndef DCLAW_ADJ_TPB
#define DCLAW_ADJ_TPB 128
#endif
// resident blocks per SM the heavy reverse kernels' registers are sized for
#ifndef DCLAW_ADJ_MINB
#define DCLAW_ADJ_MINB 4
#endif
constexpr int ATPB = DCLAW_ADJ_TPB;
// threads of the block-list kernels: one per item of a 16 x 16 block
constexpr int BTPB = 256;

__host__ __device__ inline unsigned nblk(long long n) { return (unsigned)((n + ATPB - 1) / ATPB); }

// Programmatic dependent launch: a kernel launched with the
// programmatic-serialization attribute may start while the kernel before
// it on the stream drains; it waits here, before reading anything, until
// that kernel has completed and its writes are visible (a no-op for a
// kernel launched without the attribute). A CTA that has no work left
// lets the next kernel start launching.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <typename... KArgs, typename... Args>
inline void launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, cudaStream_t s, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, args...);
}

// Sum of the block's per-thread parameter adjoints, in a fixed order, into
// dst[0..NPB). Every thread of the block (NW warps) must call it.
template <int NW>
__device__ __forceinline__ void block_pbar(const double* pb, double* __restrict__ dst) {
    __shared__ double red[NPB][NW];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NPB; ++k) {
        double v = pb[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[k][wid] = v;
    }
    __syncthreads();
    if (threadIdx.x < NPB) {
        double s = 0.0;
        for (int w = 0; w < NW; ++w) s += red[threadIdx.x][w];
        dst[threadIdx.x] = s;
    }
}

struct AdjLayout {
    StagedLayout S;
    size_t off_lamq, off_xfb, off_yfb, off_xcb, off_ycb, off_tdq, off_qsb, off_sv, off_part, off_act;
    int act_nx, act_ny;
    long long nb_src2, nb_rx, nb_ry, nb_td, nparts;
    size_t total;
};

__host__ __device__ inline AdjLayout adj_layout(int mx, int my) {
    AdjLayout L;
    L.S = staged_layout(mx, my);
    L.nb_src2 = nblk((long long)mx * my);
    L.nb_rx = nblk((long long)(mx + 3) * (my + 2));
    L.nb_ry = nblk((long long)(mx + 2) * (my + 3));
    L.nb_td = nblk((long long)L.S.npad);
    L.nparts = L.nb_src2 + L.nb_rx + L.nb_ry + L.nb_td;
    size_t o = L.S.total;
    L.off_lamq = o; o += align256((size_t)5 * mx * my * 8);
    L.off_xfb = o; o += align256((size_t)NFB * L.S.nxi * 8);
    L.off_yfb = o; o += align256((size_t)NFB * L.S.nyi * 8);
    L.off_xcb = o; o += align256((size_t)NCB * L.S.nxi * 8);
    L.off_ycb = o; o += align256((size_t)NCB * L.S.nyi * 8);
    L.off_tdq = o; o += align256((size_t)NTD * L.S.npad * 8);
    L.off_qsb = o; o += align256((size_t)NQSB * L.S.npad * 8);
    L.off_sv = o; o += align256((size_t)NSV * L.S.npad * 8);
    L.act_nx = (mx + 4 + ACT_TILE - 1) / ACT_TILE;
    L.act_ny = (my + 4 + ACT_TILE - 1) / ACT_TILE;
    // block partials: per 128-item chunk (single patch) or per activity
    // block and reverse stage (ensembles), whichever needs more
    const long long nbp = 4LL * L.act_nx * L.act_ny;
    L.off_part = o; o += align256((size_t)(L.nparts > nbp ? L.nparts : nbp) * NPB * 8);
    L.off_act = o; o += align256((size_t)L.act_nx * L.act_ny * 4);
    L.total = o;
    return L;
}

inline bool adj_sizes_ok(int mx, int my) {
    return mx >= 2 && my >= 2 && (long long)(mx + 4) * (my + 4) < (1LL << 40);
}

// ---- ensembles: the same stages over the chunks of every member -------------
enum { SP_PAD = 0, SP_INT, SP_RX, SP_RY, SP_FX, SP_FY, NSPACE };
enum {
    OP_FW_B4, OP_FW_TAUDIR, OP_FW_SVREC, OP_FW_RX, OP_FW_RY, OP_FW_FX, OP_FW_FY,
    OP_RV_SRC2, OP_RV_FX, OP_RV_FY, OP_RV_RX, OP_RV_RY, OP_RV_TAUDIR, OP_RV_B4, OP_RV_GATHER
};

template <int OP>
struct OpTraits;
#define DC_OP(op, space, pb) \
    template <>              \
    struct OpTraits<op> {    \
        static constexpr int SPACE = space; \
        static constexpr bool PBAR = pb;    \
    };
DC_OP(OP_FW_B4, SP_PAD, false)
DC_OP(OP_FW_TAUDIR, SP_PAD, false)
DC_OP(OP_FW_SVREC, SP_PAD, false)
DC_OP(OP_FW_RX, SP_RX, false)
DC_OP(OP_FW_RY, SP_RY, false)
DC_OP(OP_FW_FX, SP_FX, false)
DC_OP(OP_FW_FY, SP_FY, false)
DC_OP(OP_RV_SRC2, SP_INT, true)
DC_OP(OP_RV_FX, SP_FX, false)
DC_OP(OP_RV_FY, SP_FY, false)
DC_OP(OP_RV_RX, SP_RX, true)
DC_OP(OP_RV_RY, SP_RY, true)
DC_OP(OP_RV_TAUDIR, SP_PAD, true)
DC_OP(OP_RV_B4, SP_PAD, false)
DC_OP(OP_RV_GATHER, SP_INT, false)
#undef DC_OP

__host__ __device__ inline long long space_items(int sp, int mx, int my) {
    switch (sp) {
        case SP_PAD: return (long long)(mx + 4) * (my + 4);
        case SP_INT: return (long long)mx * my;
        case SP_RX: return (long long)(mx + 3) * (my + 2);
        case SP_RY: return (long long)(mx + 2) * (my + 3);
        case SP_FX: return (long long)(mx + 1) * (my + 2);
        default: return (long long)(mx + 2) * (my + 1);
    }
}

struct BatchArgs {
    int nmem;
    const dclaw_adj_member* mem;
    const dclaw_params* prm;
    const double* dt;
    const double* q;
    const double* b;
    const double* lam_out;
    double* lam_in;
    double* bbar;   // += the beds' adjoints (bed layout), or null
    char* work;
    int32_t* status;
};

// ---- ensembles: the stages over lists of 16 x 16 activity blocks ------------
// A batch step of mostly dry members works only where a member is wet:
//   1. k_adj_batch_zero   each member's activity map, lam_in, list lengths
//   2. k_adj_batch_scan   every interior cell; a wet one marks the blocks
//                         within ACT_REACH (a wet ghost copies a wet interior
//                         cell within 2 of the edge, whose marks cover the
//                         ghost's: the padded grid ends 2 cells out)
//   3. k_adj_batch_list   per member block: the active blocks, and the
//                         blocks that are active or have an active neighbour
//   4. the forward recompute and the zeroing of the reverse planes over the
//      second list, the reverse stages over the first: every item an active
//      item reads lies within 6 cells of it, inside the second list's
//      blocks (16 wide), and its own inputs there come from those blocks
//   5. k_adj_batch_pbar   each member's block partials, in block order.
// Items are the ones the single-patch stages run; each writes its own slots,
// so lam_in equals dclaw_step_adjoint member by member, bit for bit, and the
// parameter adjoints agree to rounding (summed per block, not per chunk).
constexpr int BLK_PBAR_OPS = 4;   // src2, x solves, y solves, calc_taudir

__device__ __forceinline__ void batch_member_work(const BatchArgs& a, const dclaw_adj_member& M, AdjLayout& L, Work& W,
                                                  AdjWork& A, uint32_t*& act) {
    L = adj_layout(M.mx, M.my);
    char* base = a.work + M.work_off;
    W = make_work(base, L.S);
    act = (uint32_t*)(base + L.off_act);
    A = AdjWork{(double*)(base + L.off_lamq), (double*)(base + L.off_xfb), (double*)(base + L.off_yfb),
                (double*)(base + L.off_xcb), (double*)(base + L.off_ycb), (double*)(base + L.off_tdq),
                (double*)(base + L.off_qsb), (double*)(base + L.off_sv), act, L.act_nx, a.bbar != nullptr};
}

// one item of stage OP at activity cell (ci, cj) (the padded cell whose
// block decides the item's activity); false outside the item space
template <int OP>
__device__ __forceinline__ void block_item(const BatchArgs& a, int m, const dclaw_adj_member& M, const dclaw_params& P,
                                           const Geom& g, const Work& W, const AdjWork& A, const AdjLayout& L,
                                           int ci, int cj, double* pb) {
    constexpr int SP = OpTraits<OP>::SPACE;
    const int mx = g.mx, my = g.my;
    const double* q_in = a.q + M.q_off;
    const double dt = a.dt[m];
    if (SP == SP_PAD) {
        if (ci < -1 || cj < -1 || ci > mx + 2 || cj > my + 2) return;
        if (OP == OP_FW_B4) {
            if (stage_b4(P, g, q_in, a.b + M.b_off, W, ci, cj) && a.status) atomicCAS(a.status + m, 0, DCLAW_ERR_NAN);
        } else if (OP == OP_FW_TAUDIR) {
            stage_taudir(P, g, W, ci, cj);
        } else if (OP == OP_FW_SVREC) {
            adj_item_svrec(P, g, W, A, ci, cj);
        } else if (OP == OP_RV_TAUDIR) {
            adj_item_taudir(P, g, W, A, ci, cj, pb);
        } else if (OP == OP_RV_B4) {
            adj_item_b4(P, g, W, A, q_in, ci, cj);
        }
    } else if (SP == SP_INT) {
        if (ci < 1 || cj < 1 || ci > mx || cj > my) return;
        if (OP == OP_RV_SRC2) adj_item_src2(P, g, W, A, a.lam_out + M.q_off, ci, cj, dt, pb);
        else if (OP == OP_RV_GATHER) {
            adj_item_gather(P, g, A, W, a.lam_in + M.q_off, ci, cj);
            if (a.bbar) adj_item_gather_bed(g, A, W, a.bbar + M.b_off, ci, cj);
        }
    } else if (SP == SP_RX) {
        if (ci < 0 || cj < 0 || ci > mx + 2 || cj > my + 1) return;
        if (OP == OP_FW_RX) stage_riemann<0>(P, g, W, cj, ci, nullptr, A.sv);
        else if (!adj_item_riemann<0>(P, g, W, A, cj, ci, pb) && a.status) atomicCAS(a.status + m, 0, DCLAW_ERR_UNSUPPORTED);
    } else if (SP == SP_RY) {
        if (ci < 0 || cj < 0 || ci > mx + 1 || cj > my + 2) return;
        if (OP == OP_FW_RY) stage_riemann<1>(P, g, W, ci, cj, nullptr, A.sv);
        else if (!adj_item_riemann<1>(P, g, W, A, ci, cj, pb) && a.status) atomicCAS(a.status + m, 0, DCLAW_ERR_UNSUPPORTED);
    } else if (SP == SP_FX) {
        if (ci < 1 || cj < 0 || ci > mx + 1 || cj > my + 1) return;
        if (OP == OP_FW_FX) stage_flux<0>(P, g, W, cj, ci, dt / g.dx, nullptr);
        else adj_item_flux<0>(P, g, W, A, cj, ci, dt);
    } else {
        if (ci < 0 || cj < 1 || ci > mx + 1 || cj > my + 1) return;
        if (OP == OP_FW_FY) stage_flux<1>(P, g, W, ci, cj, dt / g.dy, nullptr);
        else adj_item_flux<1>(P, g, W, A, ci, cj, dt);
    }
}

// In a listed block that is not active (a neighbour of active blocks) only
// the items near an active block matter: whether activity cell (ci, cj) lies
// within `margin` cells (Chebyshev) of one of the eight blocks around its
// block that is active. Active items read at most 3 cells away; each
// forward stage reads its inputs at most 2 cells further, so the margins
// grow along the forward chain (all below the block width).
__device__ __forceinline__ bool near_active_block(const uint32_t* __restrict__ act, int nx, int ny, int bx, int by,
                                                  int ci, int cj, int margin) {
    const int px = ci + 1, py = cj + 1;
    for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
            const int x = bx + dx, y = by + dy;
            if ((dx == 0 && dy == 0) || x < 0 || y < 0 || x >= nx || y >= ny || !act[y * nx + x]) continue;
            const int ex = dx < 0 ? px - (bx * ACT_TILE - 1) : dx > 0 ? (bx + 1) * ACT_TILE - px : 0;
            const int ey = dy < 0 ? py - (by * ACT_TILE - 1) : dy > 0 ? (by + 1) * ACT_TILE - py : 0;
            if ((ex > ey ? ex : ey) <= margin) return true;
        }
    return false;
}

template <int OP>
struct FwMargin {
    static constexpr int value = OP == OP_FW_B4 ? 10 : (OP == OP_FW_TAUDIR || OP == OP_FW_SVREC) ? 8
                                 : (OP == OP_FW_RX || OP == OP_FW_RY) ? 6 : 4;
};
constexpr int ZERO_MARGIN = 4;

// resident CTAs per SM of the block kernels; the stages of the set
// DCLAW_ADJ_HEAVY_SET (1: reverse solves, 2: and reverse fluxes, 3: and
// reverse src2) take DCLAW_ADJ_HEAVY_MINB instead
#ifndef DCLAW_ADJ_HEAVY_MINB
#define DCLAW_ADJ_HEAVY_MINB (DCLAW_ADJ_MINB / 2)
#endif
#ifndef DCLAW_ADJ_HEAVY_SET
#define DCLAW_ADJ_HEAVY_SET 0
#endif
template <int OP>
struct BlkMinB {
    static constexpr bool heavy = (DCLAW_ADJ_HEAVY_SET >= 1 && (OP == OP_RV_RX || OP == OP_RV_RY)) ||
                                  (DCLAW_ADJ_HEAVY_SET >= 2 && (OP == OP_RV_FX || OP == OP_RV_FY)) ||
                                  (DCLAW_ADJ_HEAVY_SET >= 3 && OP == OP_RV_SRC2);
    static constexpr int value = heavy ? DCLAW_ADJ_HEAVY_MINB : DCLAW_ADJ_MINB / 2;
};

// One stage over a list of (member, block) entries (grid-stride; every
// thread of a CTA runs the same iterations, so the barriers are uniform).
// A CTA has one thread per item of a 16 x 16 block; two CTAs per SM at up
// to 128 registers a thread.
template <int OP>
__global__ void __launch_bounds__(BTPB, BlkMinB<OP>::value) k_adj_blocks(BatchArgs a, const uint64_t* __restrict__ list,
                                                                     const unsigned int* __restrict__ count) {
    __shared__ dclaw_adj_member sM;
    __shared__ dclaw_params sP;
    __shared__ uint64_t s_e;
    __shared__ int s_list[BTPB];
    __shared__ int s_wcnt[BTPB / 32];
    pdl_wait();
    const unsigned int n = *count;
    int cur = -1;
    for (unsigned int k = blockIdx.x; k < n; k += gridDim.x) {
        if (threadIdx.x == 0) s_e = list[k];
        __syncthreads();
        const int m = (int)(s_e >> 32);
        const int blk = (int)(s_e & 0xffffffffu);
        if (m != cur) {
            const int nM = (int)(sizeof(dclaw_adj_member) / 4), nP = (int)(sizeof(dclaw_params) / 4);
            for (int j = threadIdx.x; j < nM + nP; j += blockDim.x) {
                if (j < nM) reinterpret_cast<int*>(&sM)[j] = reinterpret_cast<const int*>(a.mem + m)[j];
                else reinterpret_cast<int*>(&sP)[j - nM] = reinterpret_cast<const int*>(a.prm + m)[j - nM];
            }
            __syncthreads();
            cur = m;
        }
        const Geom g{sM.mx, sM.my, sM.mx + 4, sM.my + 4, sM.dx, sM.dy};
        AdjLayout L;
        Work W;
        AdjWork A;
        uint32_t* act;
        batch_member_work(a, sM, L, W, A, act);
        const int bx = blk % L.act_nx, by = blk / L.act_nx;
        const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
        const int ci = bx * ACT_TILE + tx - 1, cj = by * ACT_TILE + ty - 1;
        double pb[NPB] = {0.0, 0.0, 0.0, 0.0};
        if (OP == OP_RV_RX || OP == OP_RV_RY) {
            // the reverse of a dry-dry solve writes zeros (the forward
            // skipped it): those items store their zeros here, the others
            // are gathered into a dense list so that the warps running the
            // reverse solver are full of them
            constexpr int DIR = OP == OP_RV_RX ? 0 : 1;
            const int mx = g.mx, my = g.my;
            const bool valid = DIR == 0 ? (ci >= 0 && cj >= 0 && ci <= mx + 2 && cj <= my + 1)
                                        : (ci >= 0 && cj >= 0 && ci <= mx + 1 && cj <= my + 2);
            bool need = false;
            if (valid) {
                // x: row r = cj, interface i = ci (cells i-1, i); y: column r = ci, interface i = cj
                const size_t pL = DIR == 0 ? pidx(g, ci - 1, cj) : pidx(g, ci, cj - 1);
                const size_t pR = pidx(g, ci, cj);
                need = !(W.qB[pL] <= sP.dry_tolerance && W.qB[pR] <= sP.dry_tolerance);
                if (!need) {
                    double* dst = DIR == 0 ? A.xcb : A.ycb;
                    const size_t np = DIR == 0 ? W.nxi : W.nyi;
                    const size_t oi = DIR == 0 ? xidx(g, cj, ci) : yidx(g, cj, ci);
                    const int nz = A.bed ? NCB : NCB_Q;
                    for (int k = 0; k < nz; ++k) dst[(size_t)k * np + oi] = 0.0;
                }
            }
            // the list is in thread order (warp counts summed in warp
            // order), so each item lands on the same thread every run and
            // the block's parameter partial is bit-reproducible
            const unsigned bal = __ballot_sync(0xffffffffu, need);
            const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
            if (lane == 0) s_wcnt[wid] = __popc(bal);
            __syncthreads();
            int base = 0, tot = 0;
            for (int w = 0; w < BTPB / 32; ++w) {
                base += w < wid ? s_wcnt[w] : 0;
                tot += s_wcnt[w];
            }
            if (need) s_list[base + __popc(bal & ((1u << lane) - 1u))] = threadIdx.x;
            __syncthreads();
            if ((int)threadIdx.x < tot) {
                const int t = s_list[threadIdx.x];
                block_item<OP>(a, m, sM, sP, g, W, A, L, bx * ACT_TILE + (t & 15) - 1, by * ACT_TILE + (t >> 4) - 1,
                               pb);
            }
        } else if (OpTraits<OP>::PBAR || OP >= OP_RV_SRC2 || act[blk] ||
                   near_active_block(act, L.act_nx, L.act_ny, bx, by, ci, cj, FwMargin<OP>::value)) {
            // forward stages run over active blocks and their neighbours; in
            // a neighbour, only near the active ones
            block_item<OP>(a, m, sM, sP, g, W, A, L, ci, cj, pb);
        }
        if (OpTraits<OP>::PBAR) {
            const int pidx = OP == OP_RV_SRC2 ? 0 : OP == OP_RV_RX ? 1 : OP == OP_RV_RY ? 2 : 3;
            double* part = (double*)(a.work + sM.work_off + L.off_part);
            block_pbar<BTPB / 32>(pb, part + ((size_t)pidx * L.act_nx * L.act_ny + blk) * NPB);
        }
        __syncthreads();
    }
    pdl_trigger();
}

// zero the reverse planes of the listed blocks that are not active: an
// active block's items write every slot of theirs (each reverse item writes
// all of its outputs) before a later stage reads them, so only the slots of
// the inactive neighbours, which active items read near the block edges,
// need zeros; the rest of the planes is never read
__global__ void __launch_bounds__(BTPB) k_adj_blocks_zero(BatchArgs a, const uint64_t* __restrict__ list,
                                                          const unsigned int* __restrict__ count) {
    const unsigned int n = *count;
    for (unsigned int k = blockIdx.x; k < n; k += gridDim.x) {
        const uint64_t e = list[k];
        const int m = (int)(e >> 32), blk = (int)(e & 0xffffffffu);
        const dclaw_adj_member& M = a.mem[m];
        const Geom g{M.mx, M.my, M.mx + 4, M.my + 4, M.dx, M.dy};
        AdjLayout L;
        Work W;
        AdjWork A;
        uint32_t* act;
        batch_member_work(a, M, L, W, A, act);
        if (act[blk]) continue;
        const int bx = blk % L.act_nx, by = blk / L.act_nx;
        const int mx = g.mx, my = g.my;
        const size_t nint = (size_t)mx * my, nxi = L.S.nxi, nyi = L.S.nyi, npad = L.S.npad;
        const int ci = bx * ACT_TILE + (threadIdx.x & 15) - 1, cj = by * ACT_TILE + (threadIdx.x >> 4) - 1;
        if (near_active_block(act, L.act_nx, L.act_ny, bx, by, ci, cj, ZERO_MARGIN)) {
            if (ci >= 1 && cj >= 1 && ci <= mx && cj <= my) {
                const size_t c = (size_t)(cj - 1) * mx + (size_t)(ci - 1);
                for (int f = 0; f < 5; ++f) A.lamq[f * nint + c] = 0.0;
            }
            if (ci >= 0 && cj >= 0 && ci <= mx + 2 && cj <= my + 1) {
                const size_t x = xidx(g, cj, ci);
                for (int f = 0; f < NFB; ++f) A.xfb[f * nxi + x] = 0.0;
                for (int f = 0; f < NCB_Q; ++f) A.xcb[f * nxi + x] = 0.0;
            }
            if (ci >= 0 && cj >= 0 && ci <= mx + 1 && cj <= my + 2) {
                const size_t y = yidx(g, cj, ci);
                for (int f = 0; f < NFB; ++f) A.yfb[f * nyi + y] = 0.0;
                for (int f = 0; f < NCB_Q; ++f) A.ycb[f * nyi + y] = 0.0;
            }
            if (ci >= -1 && cj >= -1 && ci <= mx + 2 && cj <= my + 2) {
                const size_t pp = pidx(g, ci, cj);
                for (int f = 0; f < NTD_Q; ++f) A.tdq[f * npad + pp] = 0.0;
                for (int f = 0; f < NQSB_Q; ++f) A.qsb[f * npad + pp] = 0.0;
            }
        }
    }
}

// member m (blockIdx.y): activity map and lam_in to zero; block 0 of member
// 0 clears the list lengths
// (what & 1: the activity map and the list lengths; what & 2: lam_in)
__global__ void __launch_bounds__(256) k_adj_batch_zero(BatchArgs a, unsigned int* counts, int what) {
    pdl_wait();
    const dclaw_adj_member M = a.mem[blockIdx.y];
    const AdjLayout L = adj_layout(M.mx, M.my);
    const size_t t0 = (size_t)blockIdx.x * blockDim.x + threadIdx.x, st = (size_t)gridDim.x * blockDim.x;
    if (what & 1) {
        uint32_t* act = (uint32_t*)(a.work + M.work_off + L.off_act);
        const size_t nact = (size_t)L.act_nx * L.act_ny;
        for (size_t x = t0; x < nact; x += st) act[x] = 0u;
        if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x < 2) counts[threadIdx.x] = 0u;
    }
    if (what & 2) {
        double* lam = a.lam_in + M.q_off;
        const size_t nl = (size_t)5 * M.mx * M.my;
        for (size_t x = t0; x < nl; x += st) lam[x] = 0.0;
    }
    pdl_trigger();
}

// member m (blockIdx.y): a wet interior cell marks the blocks within
// ACT_REACH; every field of every cell is tested for NaN (status)
__global__ void __launch_bounds__(256) k_adj_batch_scan(BatchArgs a) {
    const int m = blockIdx.y;
    const dclaw_adj_member M = a.mem[m];
    const double dry = a.prm[m].dry_tolerance;
    const AdjLayout L = adj_layout(M.mx, M.my);
    uint32_t* act = (uint32_t*)(a.work + M.work_off + L.off_act);
    const double* h = a.q + M.q_off;
    const size_t n = (size_t)M.mx * M.my;
    const int act_ny = (M.my + 4 + ACT_TILE - 1) / ACT_TILE;
    bool nan = false;
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
        const double hc = h[c], f1 = h[n + c], f2 = h[2 * n + c], f3 = h[3 * n + c], f4 = h[4 * n + c];
        nan |= (hc != hc) || (f1 != f1) || (f2 != f2) || (f3 != f3) || (f4 != f4);
        if (!(hc > dry)) continue;
        const int px = (int)(c % (size_t)M.mx) + 1 + 1, py = (int)(c / (size_t)M.mx) + 1 + 1;   // padded index i + 1
        int x0 = px - ACT_REACH < 0 ? 0 : (px - ACT_REACH) / ACT_TILE, x1 = (px + ACT_REACH) / ACT_TILE;
        int y0 = py - ACT_REACH < 0 ? 0 : (py - ACT_REACH) / ACT_TILE, y1 = (py + ACT_REACH) / ACT_TILE;
        if (x1 > L.act_nx - 1) x1 = L.act_nx - 1;
        if (y1 > act_ny - 1) y1 = act_ny - 1;
        for (int y = y0; y <= y1; ++y)
            for (int x = x0; x <= x1; ++x) act[y * L.act_nx + x] = 1u;
    }
    if (nan && a.status) atomicCAS(a.status + m, 0, DCLAW_ERR_NAN);
}

// member m (blockIdx.y): its active blocks into list_act and its blocks with
// an active block among the 3 x 3 around them into list_dil (one
// warp-aggregated atomic per warp and list)
__global__ void __launch_bounds__(256) k_adj_batch_list(BatchArgs a, unsigned int* counts, uint64_t* list_act,
                                                        uint64_t* list_dil) {
    const int m = blockIdx.y;
    const dclaw_adj_member M = a.mem[m];
    const AdjLayout L = adj_layout(M.mx, M.my);
    const uint32_t* act = (const uint32_t*)(a.work + M.work_off + L.off_act);
    const int nx = L.act_nx, ny = L.act_ny, nb = nx * ny;
    const int lane = threadIdx.x & 31;
    for (int b0 = blockIdx.x * blockDim.x; b0 < nb; b0 += gridDim.x * blockDim.x) {
        const int b = b0 + threadIdx.x;
        bool on = false, dil = false;
        if (b < nb) {
            const int bx = b % nx, by = b / nx;
            on = act[b] != 0u;
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    const int x = bx + dx, y = by + dy;
                    if (x >= 0 && y >= 0 && x < nx && y < ny) dil |= act[y * nx + x] != 0u;
                }
        }
        const unsigned ba = __ballot_sync(0xffffffffu, on), bd = __ballot_sync(0xffffffffu, dil);
        unsigned base_a = 0, base_d = 0;
        if (lane == 0) {
            if (ba) base_a = atomicAdd(counts, (unsigned)__popc(ba));
            if (bd) base_d = atomicAdd(counts + 1, (unsigned)__popc(bd));
        }
        base_a = __shfl_sync(0xffffffffu, base_a, 0);
        base_d = __shfl_sync(0xffffffffu, base_d, 0);
        const unsigned below = (1u << lane) - 1u;
        const uint64_t e = ((uint64_t)m << 32) | (uint32_t)b;
        if (on) list_act[base_a + __popc(ba & below)] = e;
        if (dil) list_dil[base_d + __popc(bd & below)] = e;
    }
}

// pbar[4 m + k] += member m's block partials of its active blocks, summed in
// a fixed order: thread t takes blocks t, t + BTPB, ... of each stage in
// turn, all four parameters at once; then the threads in order
__global__ void __launch_bounds__(BTPB) k_adj_batch_pbar(BatchArgs a, double* __restrict__ pbar) {
    __shared__ double red[NPB][BTPB];
    pdl_wait();
    const int m = blockIdx.x;
    const dclaw_adj_member M = a.mem[m];
    const AdjLayout L = adj_layout(M.mx, M.my);
    const double* part = (const double*)(a.work + M.work_off + L.off_part);
    const uint32_t* act = (const uint32_t*)(a.work + M.work_off + L.off_act);
    const int nb = L.act_nx * L.act_ny;
    double sum[NPB] = {0.0, 0.0, 0.0, 0.0};
    for (int p = 0; p < BLK_PBAR_OPS; ++p)
        for (int b = threadIdx.x; b < nb; b += BTPB)
            if (act[b]) {
                const double* v = part + ((size_t)p * nb + b) * NPB;
#pragma unroll
                for (int k = 0; k < NPB; ++k) sum[k] += v[k];
            }
#pragma unroll
    for (int k = 0; k < NPB; ++k) red[k][threadIdx.x] = sum[k];
    __syncthreads();
    if (threadIdx.x < NPB) {
        double s = 0.0;
        for (int t = 0; t < BTPB; ++t) s += red[threadIdx.x][t];
        pbar[(size_t)m * NPB + threadIdx.x] += s;
    }
}

// the step adjoint of nmem members over the block lists (all launches)
// phase & 1: prepare (activity, lists, zeroing, forward recompute: none of
// it reads lam_out); phase & 2: reverse (lam_in, the reverse stages)
enum { PHASE_PREPARE = 1, PHASE_REVERSE = 2 };
inline void launch_block_adjoint(const BatchArgs& a, uint32_t nblocks, char* lists, unsigned int* counts, int nsm,
                                 cudaStream_t s, int phase) {
    uint64_t* list_act = (uint64_t*)lists;
    uint64_t* list_dil = (uint64_t*)(lists + align256((size_t)nblocks * 8));
    // the per-member kernels fill the GPU whether there is one member or many
    int gx = 4 * nsm / (a.nmem > 0 ? a.nmem : 1);
    gx = gx < 16 ? 16 : (gx > 512 ? 512 : gx);
    const dim3 per_member((unsigned)gx, (unsigned)a.nmem);
    // persistent grids over the lists
    const unsigned grid = (unsigned)nsm * 2u;
#define DC_FW(op) k_adj_blocks<op><<<grid, BTPB, 0, s>>>(a, list_dil, counts + 1)
#define DC_RV(op) k_adj_blocks<op><<<grid, BTPB, 0, s>>>(a, list_act, counts)
    if (phase & PHASE_PREPARE) {
        k_adj_batch_zero<<<per_member, 256, 0, s>>>(a, counts, 1);
        k_adj_batch_scan<<<per_member, 256, 0, s>>>(a);
        k_adj_batch_list<<<dim3(8, (unsigned)a.nmem), 256, 0, s>>>(a, counts, list_act, list_dil);
        k_adj_blocks_zero<<<grid * 2u, BTPB, 0, s>>>(a, list_dil, counts + 1);
        DC_FW(OP_FW_B4);
        DC_FW(OP_FW_TAUDIR);
        DC_FW(OP_FW_SVREC);
        DC_FW(OP_FW_RX);
        DC_FW(OP_FW_RY);
        DC_FW(OP_FW_FX);
        DC_FW(OP_FW_FY);
    }
    if (!(phase & PHASE_REVERSE)) return;
    // the reverse chain: each kernel launched as the one before it drains
#undef DC_RV
#define DC_RV(op) launch_pdl(k_adj_blocks<op>, dim3(grid), dim3(BTPB), s, a, (const uint64_t*)list_act, \
                             (const unsigned int*)counts)
    launch_pdl(k_adj_batch_zero, per_member, dim3(256), s, a, counts, 2);
    DC_RV(OP_RV_SRC2);
    DC_RV(OP_RV_FX);
    DC_RV(OP_RV_FY);
    DC_RV(OP_RV_RX);
    DC_RV(OP_RV_RY);
    DC_RV(OP_RV_TAUDIR);
    DC_RV(OP_RV_B4);
    DC_RV(OP_RV_GATHER);
#undef DC_FW
#undef DC_RV
}

// the single patch as a one-member batch: its table entry and parameters,
// written into the workspace tail by one thread
__global__ void k_adj_single_setup(dclaw_adj_member M, dclaw_params P, dclaw_adj_member* mem, dclaw_params* prm) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        *mem = M;
        *prm = P;
    }
}

// tail of the single-patch workspace: member entry, parameters, two block
// lists, list lengths
struct SingleTail {
    size_t off_mem, off_prm, off_lists, off_counts, total;
};

inline SingleTail single_tail(const AdjLayout& L) {
    SingleTail T;
    const size_t nb = (size_t)L.act_nx * L.act_ny;
    size_t o = L.total;
    T.off_mem = o; o += align256(sizeof(dclaw_adj_member));
    T.off_prm = o; o += align256(sizeof(dclaw_params));
    T.off_lists = o; o += 2 * align256(nb * 8);
    T.off_counts = o; o += 256;
    T.total = o;
    return T;
}

inline int sm_count_adj() {
    int dev = 0, nsm = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    return nsm;
}

}  // namespace adj
}  // namespace dclaw

using namespace dclaw;
using namespace dclaw::adj;

extern "C" {

size_t dclaw_adjoint_workspace_bytes(int mx, int my) {
    if (!adj_sizes_ok(mx, my)) return 0;
    return single_tail(adj_layout(mx, my)).total;
}

int dclaw_adjoint_supported(const dclaw_params* p) {
    if (!p) return DCLAW_ERR_ARG;
    int rc = dclaw_params_check_5(p);
    if (rc) return rc;
    // no adjoint form: the rare-wave corrector's branch structure and
    // src2method 2's data-dependent substeps
    if (p->src2method == 2) return DCLAW_ERR_UNSUPPORTED;
    return DCLAW_OK;
}

// the single patch as a one-member batch over its workspace (phase: which
// part of the step adjoint to queue)
static int single_adjoint(const double* q_in, const double* b, int mx, int my, double dx, double dy,
                          const double* dt, const dclaw_params* p, const double* lam_out, double* lam_in,
                          double* pbar, double* bbar, void* work, size_t work_bytes, int32_t* status, void* stream,
                          int phase) {
    if (!q_in || !b || !dt || !work) return DCLAW_ERR_ARG;
    if ((phase & PHASE_REVERSE) && (!lam_out || !lam_in || !pbar || lam_in == lam_out)) return DCLAW_ERR_ARG;
    if (!adj_sizes_ok(mx, my) || !(dx > 0.0) || !(dy > 0.0)) return DCLAW_ERR_ARG;
    int rc = dclaw_adjoint_supported(p);
    if (rc) return rc;
    AdjLayout L = adj_layout(mx, my);
    const SingleTail T = single_tail(L);
    if (work_bytes < T.total) return DCLAW_ERR_WORKSPACE;
    cudaStream_t s = (cudaStream_t)stream;
    char* base = (char*)work;
    dclaw_adj_member* mem = (dclaw_adj_member*)(base + T.off_mem);
    dclaw_params* prm = (dclaw_params*)(base + T.off_prm);
    if (phase & PHASE_PREPARE) {
        dclaw_adj_member M;
        memset(&M, 0, sizeof(M));
        M.mx = mx;
        M.my = my;
        M.dx = dx;
        M.dy = dy;
        k_adj_single_setup<<<1, 32, 0, s>>>(M, *p, mem, prm);
    }
    BatchArgs a{1, mem, prm, dt, q_in, b, lam_out, lam_in, bbar, base, status};
    launch_block_adjoint(a, (uint32_t)((size_t)L.act_nx * L.act_ny), base + T.off_lists,
                         (unsigned int*)(base + T.off_counts), sm_count_adj(), s, phase);
    if (phase & PHASE_REVERSE) launch_pdl(k_adj_batch_pbar, dim3(1), dim3(BTPB), s, a, pbar);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? DCLAW_OK : DCLAW_ERR_CUDA;
}

int dclaw_step_adjoint(const double* q_in, const double* b, int mx, int my, double dx, double dy,
                       const double* dt, const dclaw_params* p, const double* lam_out, double* lam_in,
                       double* pbar, double* bbar, void* work, size_t work_bytes, int32_t* status, void* stream) {
    return single_adjoint(q_in, b, mx, my, dx, dy, dt, p, lam_out, lam_in, pbar, bbar, work, work_bytes, status,
                          stream, PHASE_PREPARE | PHASE_REVERSE);
}

int dclaw_step_adjoint_prepare(const double* q_in, const double* b, int mx, int my, double dx, double dy,
                               const double* dt, const dclaw_params* p, void* work, size_t work_bytes,
                               int32_t* status, void* stream) {
    return single_adjoint(q_in, b, mx, my, dx, dy, dt, p, nullptr, nullptr, nullptr, nullptr, work, work_bytes,
                          status, stream, PHASE_PREPARE);
}

int dclaw_step_adjoint_reverse(const double* q_in, const double* b, int mx, int my, double dx, double dy,
                               const double* dt, const dclaw_params* p, const double* lam_out, double* lam_in,
                               double* pbar, double* bbar, void* work, size_t work_bytes, int32_t* status,
                               void* stream) {
    return single_adjoint(q_in, b, mx, my, dx, dy, dt, p, lam_out, lam_in, pbar, bbar, work, work_bytes, status,
                          stream, PHASE_REVERSE);
}

int dclaw_adjoint_batch_layout(int n, const int32_t* mx, const int32_t* my, const double* dx, const double* dy,
                               const uint64_t* q_off, const uint64_t* b_off, dclaw_adj_member* members,
                               dclaw_adj_batch* batch) {
    if (n <= 0 || !mx || !my || !dx || !dy || !q_off || !b_off || !members || !batch) return DCLAW_ERR_ARG;
    uint64_t w = 0, nblocks = 0;
    uint64_t nch[NSPACE] = {0, 0, 0, 0, 0, 0};
    for (int k = 0; k < n; ++k) {
        if (!adj_sizes_ok(mx[k], my[k]) || !(dx[k] > 0.0) || !(dy[k] > 0.0)) return DCLAW_ERR_ARG;
        dclaw_adj_member& M = members[k];
        M.mx = mx[k];
        M.my = my[k];
        M.dx = dx[k];
        M.dy = dy[k];
        M.q_off = q_off[k];
        M.b_off = b_off[k];
        M.work_off = w;
        const AdjLayout Lk = adj_layout(mx[k], my[k]);
        w += align256(Lk.total);
        nblocks += (uint64_t)Lk.act_nx * Lk.act_ny;
        for (int sp = 0; sp < NSPACE; ++sp) {
            const uint64_t c = nblk(space_items(sp, mx[k], my[k]));
            if (nch[sp] + c > 0xffffffffull) return DCLAW_ERR_TOO_LARGE;
            M.chunk0[sp] = (uint32_t)nch[sp];
            M.nchunk[sp] = (uint32_t)c;
            nch[sp] += c;
        }
    }
    if (nblocks > 0xffffffffull) return DCLAW_ERR_TOO_LARGE;
    batch->nmembers = n;
    batch->chunk_items = ATPB;
    for (int sp = 0; sp < NSPACE; ++sp) batch->nchunks[sp] = (uint32_t)nch[sp];
    batch->nblocks = (uint32_t)nblocks;
    batch->pad_ = 0;
    // + the two block lists and their lengths
    batch->work_bytes = w + 2 * align256(nblocks * 8) + 256;
    return DCLAW_OK;
}

static int batched_adjoint(const dclaw_adj_batch* batch, const dclaw_adj_member* members,
                           const dclaw_params* params, const double* dt, const double* q_in, const double* b,
                           const double* lam_out, double* lam_in, double* pbar, double* bbar, void* work,
                           int32_t* status, void* stream, int phase) {
    if (!batch || !members || !params || !dt || !q_in || !b || !work) return DCLAW_ERR_ARG;
    if ((phase & PHASE_REVERSE) && (!lam_out || !lam_in || !pbar || lam_in == lam_out)) return DCLAW_ERR_ARG;
    if (batch->nmembers <= 0 || batch->chunk_items != (uint32_t)ATPB) return DCLAW_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    BatchArgs a{batch->nmembers, members, params, dt, q_in, b, lam_out, lam_in, bbar, (char*)work, status};
    char* lists = (char*)work + (batch->work_bytes - 256 - 2 * align256((size_t)batch->nblocks * 8));
    unsigned int* counts = (unsigned int*)((char*)work + (batch->work_bytes - 256));
    launch_block_adjoint(a, batch->nblocks, lists, counts, sm_count_adj(), s, phase);
    if (phase & PHASE_REVERSE) launch_pdl(k_adj_batch_pbar, dim3((unsigned)batch->nmembers), dim3(BTPB), s, a, pbar);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? DCLAW_OK : DCLAW_ERR_CUDA;
}

int dclaw_step_adjoint_batched(const dclaw_adj_batch* batch, const dclaw_adj_member* members,
                               const dclaw_params* params, const double* dt, const double* q_in, const double* b,
                               const double* lam_out, double* lam_in, double* pbar, double* bbar, void* work,
                               int32_t* status, void* stream) {
    return batched_adjoint(batch, members, params, dt, q_in, b, lam_out, lam_in, pbar, bbar, work, status, stream,
                           PHASE_PREPARE | PHASE_REVERSE);
}

int dclaw_step_adjoint_batched_prepare(const dclaw_adj_batch* batch, const dclaw_adj_member* members,
                                       const dclaw_params* params, const double* dt, const double* q_in,
                                       const double* b, void* work, int32_t* status, void* stream) {
    return batched_adjoint(batch, members, params, dt, q_in, b, nullptr, nullptr, nullptr, nullptr, work, status,
                           stream, PHASE_PREPARE);
}

int dclaw_step_adjoint_batched_reverse(const dclaw_adj_batch* batch, const dclaw_adj_member* members,
                                       const dclaw_params* params, const double* dt, const double* q_in,
                                       const double* b, const double* lam_out, double* lam_in, double* pbar,
                                       double* bbar, void* work, int32_t* status, void* stream) {
    return batched_adjoint(batch, members, params, dt, q_in, b, lam_out, lam_in, pbar, bbar, work, status, stream,
                           PHASE_REVERSE);
}

}  // extern "C"
