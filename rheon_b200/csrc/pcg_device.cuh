// Device bodies of the start of a solve (src/pressure.rs:603-650): the
// compatibility sums and threshold, and the residual load with the first
// preconditioner application where it is elementwise. Shared by the
// single-grid kernels (pcg.cu) and the packed batch kernels (batch.cu); each
// body works on the blocks of one grid, given as a Span of the launch.
#pragma once

#include "pcg.hpp"
#include "slab.cuh"
#include "solve_state.cuh"

namespace rb200 {

constexpr double kEps = 2.220446049250313e-16;

// ------------------------------------------------------------------ init
// Compatibility sums, threshold and the true report of p = 0
// (src/pressure.rs:603-647); p is zeroed here. A seeded solve (F_WARM) keeps p,
// validates it after the compatibility check (finite, p[0] == 0,
// :615-624) and leaves its true report to the true-residual kernel.
__device__ __forceinline__ void init_sums_body(const GridDev& g, SolveState* st, const double* __restrict__ b,
                                               double* __restrict__ p, Partials part, Span sp) {
    __shared__ BlockReduce<3, 3> sm;
    const int flags0 = st->flags;
    if (flags0 & F_DONE) return;
    const bool warm = (flags0 & F_WARM) != 0;
    dd s[3] = {{0, 0}, {0, 0}, {0, 0}};
    double m[3] = {0.0, 0.0, 0.0};
    for (int c = sp.block * blockDim.x + threadIdx.x; c < g.cells; c += sp.blocks * blockDim.x) {
        double x = b[c];
        if (warm) {
            if (!isfinite(p[c])) m[2] = 1.0;
        } else {
            p[c] = 0.0;
        }
        if (!isfinite(x)) m[1] = 1.0;
        s[0] = dd_add1(s[0], x);
        s[1] = dd_add1(s[1], fabs(x));
        s[2] = dd_add1(s[2], x * x);
        m[0] = fmax(m[0], fabs(x));
    }
    block_reduce<3, 3>(sm, s, m);
    if (publish_and_check_last<3, 3>(part, sp.block, sp.blocks, s, m)) {
        fold_partials<3, 3>(part, sp.blocks, sm, s, m);
        if (threadIdx.x == 0) {
            int flags = st->flags;
            if (m[1] != 0.0) {
                finish(st, RB200_NONFINITE_INPUT, flags);
                return;
            }
            double sum = dd_value(s[0]), sum_abs = dd_value(s[1]), sq = dd_value(s[2]);
            double budget = (64.0 * kEps) * sum_abs;
            if (!isfinite(sum) || !isfinite(sum_abs)) {
                breakdown(st, 0, flags);
                return;
            }
            if (fabs(sum) > budget) {
                st->incompatible_sum = sum;
                st->incompatible_budget = budget;
                finish(st, RB200_INCOMPATIBLE_RHS, flags);
                return;
            }
            if (warm) {
                if (m[2] != 0.0) {
                    finish(st, RB200_NONFINITE_INPUT, flags);
                    return;
                }
                if (p[0] != 0.0) {
                    finish(st, RB200_INVALID_INITIAL_PRESSURE, flags);
                    return;
                }
            }
            double rhs_l2 = sqrt(sq);
            double threshold = fmax(st->absolute, st->relative * rhs_l2);
            if (!isfinite(rhs_l2) || !isfinite(threshold)) {
                breakdown(st, 0, flags);
                return;
            }
            st->threshold = threshold;
            if (warm) {
                // true_report(p0) runs next, in the true-residual kernel.
                st->flags = flags | F_STOP | F_NEED_TRUE;
                return;
            }
            // true_report(p = 0): the product is exactly b.
            double div = m[0] * st->dt / g.volume;
            if (!isfinite(sq) || !isfinite(div)) {
                breakdown(st, 0, flags);
                return;
            }
            st->true_l2 = rhs_l2;
            st->true_max = m[0];
            st->true_div = div;
            if (rhs_l2 <= threshold && div <= st->divergence_limit) {
                finish(st, RB200_OK, flags);
                return;
            }
            if (st->max_it == 0) {
                finish(st, RB200_ITERATION_LIMIT, flags);
                return;
            }
        }
    }
}

// r <- src (r[0] = 0) and the preconditioned start. Jacobi stores z = r/D and
// reduces r.z, then decides; the red-black SGS method stores y = r/D on the
// red cells (its forward red solve) and leaves the rest to its sweep kernels.
// Used for the initial residual (MODE_INIT, src = b) and for the restart
// (MODE_REPLACE, src = the true residual in the spare direction buffer).
// KIND: 0 Jacobi, 1 red-black SGS, 2 copy only (multigrid and lexicographic
// SGS form z in their own kernels).
enum : int { KIND_JACOBI = 0, KIND_RBSGS = 1, KIND_MG = 2 };
template <int KIND>
__device__ __forceinline__ void load_residual_body(const GridDev& g, SolveState* st, const double* b, double* d0,
                                                   double* d1, double* __restrict__ r, double* __restrict__ z,
                                                   int mode, Partials part, rb200_trace* trace, Span sp) {
    __shared__ BlockReduce<1, 0> sm;
    const int flags = st->flags;
    if (!gate(flags, mode)) return;
    const double* src = mode == MODE_INIT ? b : (st->dsel ? d0 : d1);
    // the flexible method alternates two residual buffers; a loaded residual
    // is in the first (the buffer the V-cycle's first half-sweep reads)
    if (KIND == KIND_MG && sp.block == 0 && threadIdx.x == 0) st->rsel = 0;
    Neu acc;
    for (int c = sp.block * blockDim.x + threadIdx.x; c < g.cells; c += sp.blocks * blockDim.x) {
        double rc = c == 0 ? 0.0 : src[c];
        r[c] = rc;
        if (c == 0) {
            if (z) z[0] = 0.0;  // the multigrid method forms z in its own kernels and passes none
            continue;
        }
        if (KIND == KIND_MG) continue;
        int i, j, k;
        cell_coords(g, c, i, j, k);
        if (KIND == KIND_JACOBI) {
            const int m = diag_mask(g, i, j, k);
            double zc = div_diag(rc, g.diag[m], g.rdiag[m]);
            z[c] = zc;
            acc.add(rc * zc);
        } else if (((i + j + k) & 1) == 0) {
            z[c] = rc / diag_at(g, i, j, k);
        }
    }
    if (KIND != KIND_JACOBI) return;
    dd sums[1] = {acc.as_dd()};
    double none[1];
    block_reduce<1, 0>(sm, sums, none);
    if (publish_and_check_last<1, 0>(part, sp.block, sp.blocks, sums, none)) {
        fold_partials<1, 0>(part, sp.blocks, sm, sums, none);
        if (threadIdx.x == 0) decide_rz(st, trace, dd_value(sums[0]), mode);
    }
}

}  // namespace rb200
