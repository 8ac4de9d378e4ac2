// Device-side decisions of the PCG state machine, shared by the solver
// kernels (pcg.cu) and the multigrid finish kernel (mg.cu).
#pragma once

#include "common.cuh"
#include "pcg.hpp"

namespace rb200 {

enum Mode : int { MODE_INIT = 0, MODE_ITER = 1, MODE_REPLACE = 2 };
constexpr int F_CANDIDATE = 32;  // RB-SGS: candidate decided in pass 2, acted on after z

__device__ __forceinline__ bool gate(int flags, int mode) {
    if (mode == MODE_INIT) return !(flags & F_DONE);
    if (mode == MODE_ITER) return !(flags & F_STOP);
    return (flags & F_NEED_REPLACE) != 0;
}

__device__ __forceinline__ int block_id3() { return blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z); }
__device__ __forceinline__ int nblocks3() { return gridDim.x * gridDim.y * gridDim.z; }
__device__ __forceinline__ int tid3() { return threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z); }

__device__ __forceinline__ void finish(SolveState* st, int status, int flags) {
    st->status = status;
    st->flags = flags | F_DONE | F_STOP;
}

__device__ __forceinline__ void breakdown(SolveState* st, int iteration, int flags) {
    st->breakdown_it = iteration;
    finish(st, RB200_BREAKDOWN, flags);
}

// Decision after a fresh r.z (precondition's return value).
__device__ __forceinline__ void decide_rz(SolveState* st, rb200_trace* trace, double rz, int mode) {
    int flags = st->flags;
    const int it = st->it;
    if (mode == MODE_INIT) {
        st->rz = rz;  // checked at iteration 1 (src/pressure.rs:662)
        st->flags = flags | F_REPLACED;
        return;
    }
    if (mode == MODE_REPLACE) {
        if (trace && it >= 1) {
            trace[it - 1].rz = rz;
            trace[it - 1].beta = 0.0;
            trace[it - 1].replaced = 1;
        }
        if (!isfinite(rz) || rz <= 0.0) {
            breakdown(st, it, flags);
            return;
        }
        st->rz = rz;
        st->flags = (flags & ~(F_STOP | F_NEED_TRUE | F_NEED_REPLACE | F_CANDIDATE)) | F_REPLACED;
        return;
    }
    // MODE_ITER
    if (flags & F_CANDIDATE) {
        st->rz_next = rz;
        st->flags = (flags & ~F_CANDIDATE) | F_STOP | F_NEED_TRUE;
        return;
    }
    if (!isfinite(rz) || rz <= 0.0) {
        breakdown(st, it, flags);
        return;
    }
    double beta = rz / st->rz;
    if (trace) {
        trace[it - 1].rz = rz;
        trace[it - 1].beta = beta;
    }
    st->beta = beta;
    st->rz = rz;
}

// Flexible-CG decision after the preconditioner (multigrid): r.z and z.q give
// beta = -z.q / d.q (Polak-Ribiere form); init and restart behave as
// decide_rz.
__device__ __forceinline__ void decide_flexible(SolveState* st, rb200_trace* trace, double rz, double zq, int mode) {
    if (mode != MODE_ITER) {
        decide_rz(st, trace, rz, mode);
        return;
    }
    const int flags = st->flags;
    const int it = st->it;
    const double beta = -zq / st->curvature;
    if (flags & F_CANDIDATE) {
        st->rz_next = rz;
        st->beta_next = beta;
        st->flags = (flags & ~F_CANDIDATE) | F_STOP | F_NEED_TRUE;
        return;
    }
    if (!isfinite(rz) || rz <= 0.0 || !isfinite(beta)) {
        breakdown(st, it, flags);
        return;
    }
    if (trace) {
        trace[it - 1].rz = rz;
        trace[it - 1].beta = beta;
    }
    st->beta = beta;
    st->rz = rz;
}

}  // namespace rb200
