// Device-driven PCG for the gauge-eliminated sealed-box pressure system
// (PressureWorkspace::solve_loaded, src/pressure.rs:577-740).
#pragma once

#include <cuda.h>

#include "internal.hpp"
#include "mg.hpp"

namespace rb200 {

// Device-resident solver state. Every control decision of solve_loaded is
// taken on the device by the last block of the kernel that produces the
// deciding scalar; the host only pumps chunks and polls `flags`.
struct SolveState {
    double rz;          // r.z of the current direction
    double rz_next;     // r.z of the recursive residual after the update
    double alpha, beta;
    double curvature, recursive_l2;
    double threshold, dt, divergence_limit, relative, absolute;
    double true_l2, true_max, true_div;
    double incompatible_sum, incompatible_budget;
    double beta_next;   // flexible method: beta pending a true-residual check
    int it;             // completed iterations
    int max_it;
    int dsel;           // which direction buffer holds the current direction
    int flags;
    int status;         // rb200_status, or ST_RUNNING
    int breakdown_it;
    int flexible;       // beta = z.(r - r_old) / rz_old (flexible CG) instead of rz'/rz
    int trips;          // loop-body passes of the graph-embedded solve
    int rsel;           // flexible method: which residual buffer holds r (the update writes the other)
};

enum : int {
    F_STOP = 1,          // iteration kernels are no-ops
    F_NEED_TRUE = 2,     // evaluate the true residual b - K p
    F_REPLACED = 4,      // the next direction is z (fresh start)
    F_DONE = 8,          // solve finished; status is final
    F_NEED_REPLACE = 16, // replace r by the true residual, re-precondition
    F_PROFILE = 64,      // timing mode: passes do their work, decisions are skipped
    F_WARM = 128         // seeded solve: p holds the caller's initial pressure
};
constexpr int ST_RUNNING = -1;

// Tensor maps of the solver's vectors for the TMA slab loads (unused when the
// grid takes the cp.async path).
// z, d0, d1, p: halo slabs ((TX+4) x (TY+2) x (ZC+2)); p_box, r_box: one
// brick without halo (TX x TY x ZC), for the persistent solver.
struct TmaMaps {
    CUtensorMap z, d0, d1, p;
    CUtensorMap p_box, r_box;
    int use;
};

// Grid barrier of the persistent solver kernel (zeroed before each solve).
// `count` only grows: barrier m of a solve is passed once it reaches
// m x (blocks of the grid), so no reset is needed between barriers.
struct GridBarrier {
    unsigned long long count;  // arrivals since the solve began
    unsigned abort;            // a block gave up: every waiting block leaves
    unsigned pad;
};

// Work queue of the lexicographic SGS preconditioner (one launch per
// application, forward and reverse sweep): the 8^3 tiles in wave order and
// one state word per tile. The word block is zeroed by the r.z kernel that
// follows every application.
struct SgsFlow {
    const int* order = nullptr;  // tile ids (tx + ntx (ty + nty tz)), waves tx + ty + tz ascending
    unsigned* ctl = nullptr;     // [0] next queue slot, [1] abort, [2 + tile] 1 forward done, 2 reverse done
    int ntiles = 0;
    int blocks = 0;              // resident blocks of the sweep kernel
};

// Persistent PCG kernel (persist.cu); pre: 0 Jacobi, 1 red-black SGS.
int persistent_setup(const GridDev& g, int* blocks);
size_t persistent_partial_doubles(int blocks);
cudaError_t launch_persistent(const GridDev& g, SolveState* st, const double* b, double* p, double* r, double* z,
                              double* d0, double* d1, double* part, GridBarrier* bar, rb200_trace* trace,
                              const TmaMaps& maps, int blocks, int budget, cudaStream_t s, int pre);

class PcgSolver {
public:
    PcgSolver() = default;
    ~PcgSolver();
    PcgSolver(const PcgSolver&) = delete;
    PcgSolver& operator=(const PcgSolver&) = delete;

    // Allocates b, p, r, two direction buffers, partials and the state.
    int init(const GridDev& g, int method, cudaStream_t stream);
    // Solve K p = b for the RHS already in b(). dt is the step's dt (for the
    // divergence gate). On return p() holds the iterate (also on
    // ITERATION_LIMIT). `status` receives the PressureError-style outcome.
    // `initial` (host or device memory, g.cells values, or nullptr) seeds the
    // solve: solve_*_with_initial_pressure (src/pressure.rs:395-430).
    int solve(double dt, const rb200_settings& s, rb200_report* report, rb200_cancel_fn cancelled,
              void* ctx, const double* initial = nullptr);
    double* b() { return b_; }
    double* p() { return p_; }
    double* scratch() { return d_[1]; }
    size_t bytes() const { return bytes_; }
    int set_trace(rb200_trace* host, size_t capacity);
    // Average device time of `launches` back-to-back launches of one PCG pass
    // (which = 0: direction+apply, 1: update), or (which = 2, persistent
    // solver only) of one iteration of the persistent kernel run for
    // `launches` iterations in one launch; timed with CUDA events on the
    // solver's stream, on the current vectors. Scalars are left in a timing
    // state; the next solve() resets them.
    int profile(int which, int launches, double* avg_ms);

    // Graph embedding (the resident carrier step is one CUDA graph):
    // enqueue_reset initialises the state on the device from `settings` and the
    // device dt (*dt_dev); when *skip != 0 the solve is marked done and every
    // solver kernel is a no-op. enqueue_loop adds a WHILE conditional node that
    // repeats the iteration chunk until the state is done, with the trip count
    // bounded so that the loop always ends. Both run during a stream capture.
    // With `warm` (device flag) set, the solve is seeded from `seed` (device,
    // g.cells values): the resident carrier's accepted previous pressure.
    int enqueue_reset(const double* dt_dev, const int* skip, const rb200_settings& settings, cudaStream_t s,
                      const int* warm = nullptr, const double* seed = nullptr);
    int enqueue_loop(cudaStream_t capture_stream, cudaStream_t body_stream, const rb200_settings& settings);
    int nodes_per_chunk() const { return nodes_per_chunk_ + 1; }
    // Blocks of the persistent solver kernel (0: the per-pass kernels run).
    int persistent_blocks() const { return persist_blocks_; }
    // One launch of the persistent kernel for at most `budget` iterations.
    cudaError_t launch_persistent_chunk(cudaStream_t s, int budget);
    int persist_pre_ = 0;  // preconditioner of the persistent kernel: 0 Jacobi, 1 red-black SGS
    SolveState* state() { return st_; }
    const GridDev& grid() const { return g_; }
    Partials partials() const { return part_; }
    int partial_blocks() const { return part_blocks_; }
    // Kernels launched by solve() so far (graph nodes included).
    uint64_t launches() const { return launches_; }

private:
    int capture_chunk();
    int sgs_setup();
    int launch_chunk(int slot);
    int record_flags(int slot);

    GridDev g_{};
    int method_ = RB200_JACOBI_PCG_V1;
    cudaStream_t stream_ = nullptr;
    double* b_ = nullptr;
    double* p_ = nullptr;
    double* r_ = nullptr;
    double* d_[2] = {nullptr, nullptr};
    double* z_ = nullptr;  // preconditioned residual
    double* r1_ = nullptr;  // the multigrid method's second residual buffer (r and r_old alternate)
    Multigrid mg_;
    TmaMaps maps_{};
    Partials part_{nullptr, nullptr};
    int part_blocks_ = 0;
    SolveState* st_ = nullptr;
    SolveState* h_st_ = nullptr;  // pinned, one slot per in-flight chunk
    cudaEvent_t ev_[2] = {nullptr, nullptr};
    cudaGraphExec_t chunk_exec_ = nullptr;
    int chunk_ = 16;
    rb200_trace* d_trace_ = nullptr;
    rb200_trace* h_trace_ = nullptr;
    size_t trace_cap_ = 0;
    size_t bytes_ = 0;
    int nodes_per_chunk_ = 0;
    uint64_t launches_ = 0;
    int persist_blocks_ = 0;
    GridBarrier* gbar_ = nullptr;
    SgsFlow sgs_{};
    double* ppart_ = nullptr;
};

// Blocks of the slab passes (reduction partials needed per pass).
int slab_blocks(const GridDev& g);

}  // namespace rb200
