// workspace.cuh -- layout of the staged step's intermediates inside a
// caller-provided workspace (host-side arithmetic only).
//
// The staged step (one launch per stage, kernels.cu) keeps the b4step2 state,
// the padded bed, calc_taudir's three fields, the interface solves and the
// interface fluxes of one patch; the adjoint (adjoint.cu) recomputes exactly
// these intermediates from a step's input state before running the reverse
// stages, so both use this one layout.
#pragma once
#include <stddef.h>
#include "stages.cuh"

#if defined(__CUDACC__)
#define WS_HD __host__ __device__ inline
#else
#define WS_HD inline
#endif

namespace dclaw {

WS_HD size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

struct StagedLayout {
    size_t npad, nxi, nyi;
    size_t off_qB, off_bP, off_td, off_wx, off_wy, off_fx, off_fy, total;
};

WS_HD StagedLayout staged_layout(int mx, int my) {
    StagedLayout L;
    L.npad = (size_t)(mx + 4) * (my + 4);
    L.nxi = (size_t)(mx + 3) * (my + 2);
    L.nyi = (size_t)(my + 3) * (mx + 2);
    size_t o = 0;
    L.off_qB = o; o += align256(5 * L.npad * 8);
    L.off_bP = o; o += align256(L.npad * 8);
    L.off_td = o; o += align256(3 * L.npad * 8);
    L.off_wx = o; o += align256((size_t)NW * L.nxi * 8);
    L.off_wy = o; o += align256((size_t)NW * L.nyi * 8);
    L.off_fx = o; o += align256((size_t)NF * L.nxi * 8);
    L.off_fy = o; o += align256((size_t)NF * L.nyi * 8);
    L.total = o;
    return L;
}

WS_HD Work make_work(void* base, const StagedLayout& L) {
    char* b = (char*)base;
    Work W;
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

}  // namespace dclaw
