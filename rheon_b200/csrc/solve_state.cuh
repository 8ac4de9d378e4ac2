// Device-side decisions of the PCG state machine, shared by the solver
// kernels (pcg.cu) and the multigrid finish kernel (mg.cu).
#pragma once

#include "common.cuh"
#include "pcg.hpp"

namespace rb200 {

enum Mode : int { MODE_INIT = 0, MODE_ITER = 1, MODE_REPLACE = 2 };
constexpr int F_CANDIDATE = 32;  // RB-SGS: candidate decided in pass 2, acted on after z

// Kernels of one mode run while the flags allow: the start of a cold solve
// (a seeded solve starts with its true-residual check instead), iterations
// until a stop, the restart when one is pending.
__device__ __forceinline__ bool gate(int flags, int mode) {
    if (mode == MODE_INIT) return !(flags & (F_DONE | F_WARM));
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

// Flexible-CG decision after the preconditioner (multigrid): r.z and
// z.r_old (the residual before this iteration's update) give the
// Polak-Ribiere beta = (z.r - z.r_old) / (z_old.r_old), which is
// -z.q / d.q with q = K d since r = r_old - alpha q and alpha d.q = z_old.r_old;
// init and restart behave as decide_rz.
__device__ __forceinline__ void decide_flexible(SolveState* st, rb200_trace* trace, double rz, double zr_old,
                                                int mode) {
    if (mode != MODE_ITER) {
        decide_rz(st, trace, rz, mode);
        return;
    }
    const int flags = st->flags;
    const int it = st->it;
    const double beta = (rz - zr_old) / st->rz;
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

// Pass 1 (src/pressure.rs:657-668): the curvature d.q of the new direction
// gives alpha = r.z / d.q, or a breakdown. `flags` and `dsel` are the values
// the pass started with; the direction buffers swap roles.
__device__ __forceinline__ void decide_pass1(SolveState* st, rb200_trace* trace, double curvature, int flags,
                                             int dsel) {
    st->curvature = curvature;
    st->dsel = dsel ^ 1;
    if (flags & F_PROFILE) return;
    const double rz = st->rz;
    const int it = st->it + 1;
    const int fl = flags & ~F_REPLACED;
    if (trace) {
        trace[it - 1].curvature = curvature;
        trace[it - 1].replaced = 0;
        trace[it - 1].checked = 0;
    }
    if (!isfinite(curvature) || curvature <= 0.0 || !isfinite(rz) || rz <= 0.0) {
        breakdown(st, it, fl);
        return;
    }
    const double alpha = rz / curvature;
    if (!isfinite(alpha)) {
        breakdown(st, it, fl);
        return;
    }
    if (trace) trace[it - 1].alpha = alpha;
    st->alpha = alpha;
    st->flags = fl;
}

// Pass 2 (src/pressure.rs:669-685): the iteration is complete; the recursive
// norm decides whether the true residual is checked (a candidate, or the last
// allowed iteration). With the Jacobi preconditioner r.z is already known
// (`has_rz`) and beta follows; the other preconditioners only mark the
// candidate and decide after forming z.
__device__ __forceinline__ void decide_pass2(SolveState* st, rb200_trace* trace, double rr, double rz, int flags,
                                             bool has_rz) {
    if (flags & F_PROFILE) {
        st->recursive_l2 = rr;
        st->rz_next = rz;
        return;
    }
    const int it = st->it + 1;
    st->it = it;
    const double recursive_l2 = sqrt(rr);
    st->recursive_l2 = recursive_l2;
    if (trace) trace[it - 1].recursive_l2 = recursive_l2;
    const bool candidate = recursive_l2 <= st->threshold || it == st->max_it;
    if (has_rz) {
        if (candidate) {
            st->rz_next = rz;
            st->flags = flags | F_STOP | F_NEED_TRUE;
        } else {
            decide_rz(st, trace, rz, MODE_ITER);
        }
    } else if (candidate) {
        st->flags = flags | F_CANDIDATE;
    }
}

// True-residual check (true_report, src/pressure.rs:432-456, and the
// acceptance/restart decisions of solve_loaded, :686-715): accept, stop at the
// iteration limit, restart from the true residual, or keep the recurrence.
// `squared` is |t|^2 over every row, `squared_tail` over the rows after the
// gauge row: a seeded solve judges the restart by the latter (:697-704). At
// iteration 0 (the seeded start, :634-650) an unaccepted residual becomes the
// first residual unless no iteration is allowed.
__device__ __forceinline__ void decide_true(SolveState* st, rb200_trace* trace, double squared, double squared_tail,
                                            double maximum, int flags, double volume) {
    const int it = st->it;
    const double div = maximum * st->dt / volume;
    if (trace && it >= 1) trace[it - 1].checked = 1;
    if (!isfinite(squared) || !isfinite(div)) {
        breakdown(st, it, flags);
        return;
    }
    const double l2 = sqrt(squared);
    st->true_l2 = l2;
    st->true_max = maximum;
    st->true_div = div;
    if (l2 <= st->threshold && div <= st->divergence_limit) {
        finish(st, RB200_OK, flags);
        return;
    }
    if (it == 0) {
        if (st->max_it == 0) {
            finish(st, RB200_ITERATION_LIMIT, flags);
            return;
        }
        st->flags = (flags & ~F_NEED_TRUE) | F_NEED_REPLACE;
        return;
    }
    // A seeded solve (src/pressure.rs:700-708) and the flexible method judge
    // the restart by the rows other than the eliminated gauge row: a true
    // residual that exceeds the target only in that row is not recurrence
    // drift, and restarting there discards the directions that reduce it. The
    // multigrid preconditioner sees the gauge row's residual (minus the sum of
    // the others) only weakly, so a restart after every candidate would repeat
    // forever where that sum converges last.
    const double replacement_l2 = ((flags & F_WARM) || st->flexible) ? sqrt(squared_tail) : l2;
    const bool replaced = replacement_l2 > st->threshold;
    if (it == st->max_it) {
        finish(st, RB200_ITERATION_LIMIT, flags);
        return;
    }
    if (replaced) {
        st->flags = (flags & ~F_NEED_TRUE) | F_NEED_REPLACE;
        return;
    }
    // Keep the recurrence: precondition the recursive residual.
    const double rz = st->rz_next;
    if (!isfinite(rz) || rz <= 0.0) {
        breakdown(st, it, flags);
        return;
    }
    const double beta = st->flexible ? st->beta_next : rz / st->rz;
    if (trace) {
        trace[it - 1].rz = rz;
        trace[it - 1].beta = beta;
    }
    st->beta = beta;
    st->rz = rz;
    st->flags = flags & ~(F_STOP | F_NEED_TRUE);
}

}  // namespace rb200
