// adjoint.cu -- CUDA kernels and C ABI of the adjoint (vector-Jacobian
// product) of one uniform-patch step, sm_100a, FP64.
//
// dclaw_step_adjoint maps the adjoint of a step's output state, lam_out, to
// the adjoint of its input state, lam_in = (dS/dq)^T lam_out, and adds
// (dS/dtheta)^T lam_out to the adjoints of the material parameters
// theta = (phi [rad], kref, alpha_c, mu). The step's dt is data.
//
// One call is 16 data-parallel launches:
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
constexpr int NWARP = ATPB / 32;

inline unsigned nblk(long long n) { return (unsigned)((n + ATPB - 1) / ATPB); }

__device__ __forceinline__ void flag(int32_t* st, int code) {
    if (st) atomicCAS(st, 0, code);
}

// Sum of the block's per-thread parameter adjoints, in a fixed order, into
// part[blockIdx.x * NPB + k]. Every thread of the block must call it.
__device__ __forceinline__ void block_pbar(const double* pb, double* __restrict__ part) {
    __shared__ double red[NPB][NWARP];
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
        for (int w = 0; w < NWARP; ++w) s += red[threadIdx.x][w];
        part[(size_t)blockIdx.x * NPB + threadIdx.x] = s;
    }
}

// ---- forward recompute (the staged step's stages A-D) ---------------------
__global__ void __launch_bounds__(ATPB) k_fw_b4(dclaw_params P, Geom g, const double* __restrict__ q_in,
                                                const double* __restrict__ b, Work W, int32_t* status) {
    const long long n = (long long)g.PX * g.PY;
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n) return;
    int i = (int)(idx % g.PX) - 1, j = (int)(idx / g.PX) - 1;
    if (stage_b4(P, g, q_in, b, W, i, j)) flag(status, DCLAW_ERR_NAN);
}

__global__ void __launch_bounds__(ATPB) k_fw_taudir(dclaw_params P, Geom g, Work W) {
    const long long n = (long long)g.PX * g.PY;
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n) return;
    int i = (int)(idx % g.PX) - 1, j = (int)(idx / g.PX) - 1;
    stage_taudir(P, g, W, i, j);
}

// DIR 0: rows r = 0..my+1, interfaces i = 0..mx+2; DIR 1: interfaces
// k = 0..my+2, columns c = 0..mx+1 (the fast index is along x)
__global__ void __launch_bounds__(ATPB) k_fw_svrec(dclaw_params P, Geom g, Work W, AdjWork A) {
    const long long n = (long long)g.PX * g.PY;
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n) return;
    int i = (int)(idx % g.PX) - 1, j = (int)(idx / g.PX) - 1;
    adj_item_svrec(P, g, W, A, i, j);
}

template <int DIR>
__global__ void __launch_bounds__(ATPB) k_fw_riemann(dclaw_params P, Geom g, Work W, const double* __restrict__ sv) {
    const int nfast = DIR == 0 ? g.mx + 3 : g.mx + 2;
    const int nslow = DIR == 0 ? g.my + 2 : g.my + 3;
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)nfast * nslow) return;
    int a = (int)(idx % nfast), s = (int)(idx / nfast);
    int r = DIR == 0 ? s : a, i = DIR == 0 ? a : s;
    stage_riemann<DIR>(P, g, W, r, i, nullptr, sv);
}

// DIR 0: rows 0..my+1, interfaces 1..mx+1; DIR 1: interfaces 1..my+1, columns 0..mx+1
template <int DIR>
__global__ void __launch_bounds__(ATPB) k_fw_flux(dclaw_params P, Geom g, Work W, const double* __restrict__ dtp) {
    const int nfast = DIR == 0 ? g.mx + 1 : g.mx + 2;
    const int nslow = DIR == 0 ? g.my + 2 : g.my + 1;
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)nfast * nslow) return;
    int a = (int)(idx % nfast), s = (int)(idx / nfast);
    int r = DIR == 0 ? s : a, i = DIR == 0 ? a + 1 : s + 1;
    const double dt = *dtp;
    stage_flux<DIR>(P, g, W, r, i, DIR == 0 ? dt / g.dx : dt / g.dy, nullptr);
}

// ---- reverse stages -------------------------------------------------------
__global__ void __launch_bounds__(ATPB, DCLAW_ADJ_MINB) k_rv_src2(dclaw_params P, Geom g, Work W, AdjWork A,
                                                  const double* __restrict__ lam_out, const double* __restrict__ dtp,
                                                  double* __restrict__ part) {
    const long long n = (long long)g.mx * g.my;
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double pb[NPB] = {0.0, 0.0, 0.0, 0.0};
    if (idx < n) {
        int i = (int)(idx % g.mx) + 1, j = (int)(idx / g.mx) + 1;
        adj_item_src2(P, g, W, A, lam_out, i, j, *dtp, pb);
    }
    block_pbar(pb, part);
}

template <int DIR>
__global__ void __launch_bounds__(ATPB, DCLAW_ADJ_MINB) k_rv_flux(dclaw_params P, Geom g, Work W, AdjWork A,
                                                  const double* __restrict__ dtp) {
    const int nfast = DIR == 0 ? g.mx + 1 : g.mx + 2;
    const int nslow = DIR == 0 ? g.my + 2 : g.my + 1;
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)nfast * nslow) return;
    int a = (int)(idx % nfast), s = (int)(idx / nfast);
    int r = DIR == 0 ? s : a, i = DIR == 0 ? a + 1 : s + 1;
    adj_item_flux<DIR>(P, g, W, A, r, i, *dtp);
}

template <int DIR>
__global__ void __launch_bounds__(ATPB, DCLAW_ADJ_MINB) k_rv_riemann(dclaw_params P, Geom g, Work W, AdjWork A,
                                                     double* __restrict__ part, int32_t* status) {
    const int nfast = DIR == 0 ? g.mx + 3 : g.mx + 2;
    const int nslow = DIR == 0 ? g.my + 2 : g.my + 3;
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double pb[NPB] = {0.0, 0.0, 0.0, 0.0};
    if (idx < (long long)nfast * nslow) {
        int a = (int)(idx % nfast), s = (int)(idx / nfast);
        int r = DIR == 0 ? s : a, i = DIR == 0 ? a : s;
        if (!adj_item_riemann<DIR>(P, g, W, A, r, i, pb)) flag(status, DCLAW_ERR_UNSUPPORTED);
    }
    block_pbar(pb, part);
}

__global__ void __launch_bounds__(ATPB) k_rv_taudir(dclaw_params P, Geom g, Work W, AdjWork A,
                                                    double* __restrict__ part) {
    const long long n = (long long)g.PX * g.PY;
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double pb[NPB] = {0.0, 0.0, 0.0, 0.0};
    if (idx < n) {
        int i = (int)(idx % g.PX) - 1, j = (int)(idx / g.PX) - 1;
        adj_item_taudir(P, g, W, A, i, j, pb);
    }
    block_pbar(pb, part);
}

__global__ void __launch_bounds__(ATPB) k_rv_b4(dclaw_params P, Geom g, Work W, AdjWork A,
                                                const double* __restrict__ q_in) {
    const long long n = (long long)g.PX * g.PY;
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n) return;
    int i = (int)(idx % g.PX) - 1, j = (int)(idx / g.PX) - 1;
    adj_item_b4(P, g, W, A, q_in, i, j);
}

__global__ void __launch_bounds__(ATPB) k_rv_gather(dclaw_params P, Geom g, Work W, AdjWork A,
                                                    double* __restrict__ lam_in) {
    const long long n = (long long)g.mx * g.my;
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n) return;
    int i = (int)(idx % g.mx) + 1, j = (int)(idx / g.mx) + 1;
    adj_item_gather(P, g, A, W, lam_in, i, j);
}

// pbar[k] += sum over the nb block partials, in block order (one block)
__global__ void __launch_bounds__(ATPB) k_rv_pbar(const double* __restrict__ part, long long nb,
                                                  double* __restrict__ pbar) {
    __shared__ double red[NPB][ATPB];
    for (int k = 0; k < NPB; ++k) {
        double s = 0.0;
        for (long long b = threadIdx.x; b < nb; b += ATPB) s += part[b * NPB + k];
        red[k][threadIdx.x] = s;
    }
    __syncthreads();
    if (threadIdx.x < NPB) {
        double s = 0.0;
        for (int t = 0; t < ATPB; ++t) s += red[threadIdx.x][t];
        pbar[threadIdx.x] += s;
    }
}

struct AdjLayout {
    StagedLayout S;
    size_t off_lamq, off_xfb, off_yfb, off_xcb, off_ycb, off_tdq, off_qsb, off_sv, off_part;
    long long nb_src2, nb_rx, nb_ry, nb_td, nparts;
    size_t total;
};

inline AdjLayout adj_layout(int mx, int my) {
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
    L.off_qsb = o; o += align256((size_t)5 * L.S.npad * 8);
    L.off_sv = o; o += align256((size_t)NSV * L.S.npad * 8);
    L.off_part = o; o += align256((size_t)L.nparts * NPB * 8);
    L.total = o;
    return L;
}

inline bool adj_sizes_ok(int mx, int my) {
    return mx >= 2 && my >= 2 && (long long)(mx + 4) * (my + 4) < (1LL << 40);
}

}  // namespace adj
}  // namespace dclaw

using namespace dclaw;
using namespace dclaw::adj;

extern "C" {

size_t dclaw_adjoint_workspace_bytes(int mx, int my) {
    if (!adj_sizes_ok(mx, my)) return 0;
    return adj_layout(mx, my).total;
}

int dclaw_adjoint_supported(const dclaw_params* p) {
    if (!p) return DCLAW_ERR_ARG;
    int rc = dclaw_params_check(p);
    if (rc) return rc;
    // no adjoint form: the rare-wave corrector's branch structure, Manning
    // friction and src2method 2's data-dependent substeps
    if (p->rarecorrectortest || (p->friction_forcing && p->manning_coefficient > 0.0) || p->src2method == 2)
        return DCLAW_ERR_UNSUPPORTED;
    return DCLAW_OK;
}

int dclaw_step_adjoint(const double* q_in, const double* b, int mx, int my, double dx, double dy,
                       const double* dt, const dclaw_params* p, const double* lam_out, double* lam_in,
                       double* pbar, void* work, size_t work_bytes, int32_t* status, void* stream) {
    if (!q_in || !b || !dt || !lam_out || !lam_in || !pbar || !work) return DCLAW_ERR_ARG;
    if (lam_in == lam_out || !adj_sizes_ok(mx, my) || !(dx > 0.0) || !(dy > 0.0)) return DCLAW_ERR_ARG;
    int rc = dclaw_adjoint_supported(p);
    if (rc) return rc;
    AdjLayout L = adj_layout(mx, my);
    if (work_bytes < L.total) return DCLAW_ERR_WORKSPACE;
    cudaStream_t s = (cudaStream_t)stream;
    const dclaw_params P = *p;
    Geom g{mx, my, mx + 4, my + 4, dx, dy};
    Work W = make_work(work, L.S);
    char* base = (char*)work;
    AdjWork A{(double*)(base + L.off_lamq), (double*)(base + L.off_xfb), (double*)(base + L.off_yfb),
              (double*)(base + L.off_xcb), (double*)(base + L.off_ycb), (double*)(base + L.off_tdq),
              (double*)(base + L.off_qsb), (double*)(base + L.off_sv)};
    double* part = (double*)(base + L.off_part);
    const long long npad = (long long)L.S.npad, nint = (long long)mx * my;
    const long long nxf = (long long)(mx + 1) * (my + 2), nyf = (long long)(mx + 2) * (my + 1);
    // forward intermediates of this step
    k_fw_b4<<<nblk(npad), ATPB, 0, s>>>(P, g, q_in, b, W, status);
    k_fw_taudir<<<nblk(npad), ATPB, 0, s>>>(P, g, W);
    k_fw_svrec<<<nblk(npad), ATPB, 0, s>>>(P, g, W, A);
    k_fw_riemann<0><<<(unsigned)L.nb_rx, ATPB, 0, s>>>(P, g, W, A.sv);
    k_fw_riemann<1><<<(unsigned)L.nb_ry, ATPB, 0, s>>>(P, g, W, A.sv);
    k_fw_flux<0><<<nblk(nxf), ATPB, 0, s>>>(P, g, W, dt);
    k_fw_flux<1><<<nblk(nyf), ATPB, 0, s>>>(P, g, W, dt);
    // reverse
    double* part_src2 = part;
    double* part_rx = part_src2 + (size_t)L.nb_src2 * NPB;
    double* part_ry = part_rx + (size_t)L.nb_rx * NPB;
    double* part_td = part_ry + (size_t)L.nb_ry * NPB;
    k_rv_src2<<<(unsigned)L.nb_src2, ATPB, 0, s>>>(P, g, W, A, lam_out, dt, part_src2);
    k_rv_flux<0><<<nblk(nxf), ATPB, 0, s>>>(P, g, W, A, dt);
    k_rv_flux<1><<<nblk(nyf), ATPB, 0, s>>>(P, g, W, A, dt);
    k_rv_riemann<0><<<(unsigned)L.nb_rx, ATPB, 0, s>>>(P, g, W, A, part_rx, status);
    k_rv_riemann<1><<<(unsigned)L.nb_ry, ATPB, 0, s>>>(P, g, W, A, part_ry, status);
    k_rv_taudir<<<(unsigned)L.nb_td, ATPB, 0, s>>>(P, g, W, A, part_td);
    k_rv_b4<<<nblk(npad), ATPB, 0, s>>>(P, g, W, A, q_in);
    k_rv_gather<<<nblk(nint), ATPB, 0, s>>>(P, g, W, A, lam_in);
    k_rv_pbar<<<1, ATPB, 0, s>>>(part, L.nparts, pbar);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? DCLAW_OK : DCLAW_ERR_CUDA;
}

}  // extern "C"
