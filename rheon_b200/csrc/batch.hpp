// Packed batch of independent fixed-box carriers stepped together with the
// mixed-precision pressure method (new; the reference steps one box at a time,
// src/simulation.rs:812-1403).
//
// Every instance keeps its own accepted state, solver vectors and multigrid
// hierarchy in one device arena; a device table describes them. Each kernel of
// the step is ONE launch over all instances: a launch gives every instance a
// contiguous range of blocks (its span), found by a binary search over the
// ranges passed in the kernel's parameters, and every body works on its
// instance's span exactly as a single-grid launch works on all of its blocks.
// The span of an instance depends only on that instance's grid, and every
// reduction folds that instance's partials in block order under its own
// ticket, so an instance's results are bit for bit the same in a batch of one
// and in any mix. Solver decisions are per instance (solve_state.cuh); the
// kernels of an instance whose solve has stopped return at once. The whole
// batched step is one CUDA graph: the solve is a WHILE node over chunks of
// iterations that runs while any instance is unfinished.
#pragma once

#include <cstddef>

#include "mg.hpp"
#include "pcg.hpp"

namespace rb200 {

constexpr int kBatchMax = 128;  // instances of one batch

// Block ranges of one packed launch: entry e owns blocks [first[e], first[e+1]).
struct BatchSpans {
    int count;
    int first[kBatchMax + 1];
};

// Per-instance step state (dt policy, gates, commit), the batch counterpart of
// the single carrier's descriptor.
struct BatchStepDev {
    int acc;      // accepted face buffer
    int status;   // STEP_RUNNING while the step runs, then the step's status
    int skip;     // nonzero: the solve is skipped (the step already failed)
    int flags;    // validation flags of the step's kernels
    double requested_dt, cfl;
    int iteration_limit_ok, skip_gates;
    double max_courant, divergence_limit;
    double dt, rate, time;
    unsigned long long generation;
    double scalars[4];  // max|div|, max|u|, max|v|, max|w| of the corrected faces
    rb200_step_report report;
    int step_status;
    int trips;
};

// Per-instance device descriptor.
struct BatchInstDev {
    GridDev g;
    float* faces[3][3];  // [buffer][axis], f32 storage
    double *b, *p, *r, *r1, *d0, *d1;  // r, r1: the two residual buffers (the state's rsel picks r)
    SolveState* st;
    Partials part;       // this instance's reduction partials and ticket
    BatchStepDev* step;
    MgLevelDev fine;     // the finest level, with its own correction buffer
};

// One instance's part of a packed V-cycle launch.
struct BatchLevelOp {
    MgLevelDev L;          // the level; x is the buffer the operation reads
    MgLevelDev C;          // restriction/prolongation: the coarser level (x its final buffer)
    float* out;            // fused pairs and trains: the buffer written
    const double* r0;      // the finest level's first half-sweep: its FP64 residual
    const SolveState* st;  // the instance's solver state (gating)
    int color, first;      // half-sweeps; trains: colour of the first phase
    int start;             // sweep trains: the first phase's kind (TrainStart)
    int sj, sk;            // sweep trains: strip rows and chunk planes of a block
};

// One instance's levels below its grid-kernel levels (from its lower_first
// level on, the coarsest included) for the per-instance cluster kernel.
struct BatchLowerDev {
    MgLower P;             // the levels, their second buffers and pairing
    const double* G;       // the coarsest level's FP64 pseudo-inverse
    const SolveState* st;  // the instance's solver state (gating)
};

}  // namespace rb200
