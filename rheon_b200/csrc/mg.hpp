// Mixed-precision geometric multigrid preconditioner for the sealed-box
// pressure system (new; the reference has no multigrid).
//
// One V(2,2) cycle in FP32 on a hierarchy of cell-centred grids: symmetric
// red-black Gauss-Seidel smoothing (red then black before, black then red
// after), residual restriction by summing the children (integrated RHS),
// piecewise-constant prolongation (the transpose of the restriction), and
// rediscretised coarse operators. Every axis longer than 8 cells is halved
// (rounding up) until all are at most 8, so the coarsest grid has at most
// 8^3 cells; it is solved in FP64 by a dense, mean-projected pseudo-inverse of
// its (singular, Neumann) operator, computed once on the host. The cycle is a
// fixed symmetric operator up to FP32 rounding; the outer FP64 flexible CG
// absorbs the rest.
//
// Launch structure of one cycle: grid-wide kernels for the levels above 32^3
// cells; one kernel on a thread-block cluster (16 CTAs where the device
// schedules them) for every level of at most 32^3 cells, the dense coarsest
// solve included, whose half-sweeps meet at hardware cluster barriers. Where
// a level's rows are a multiple of 4 long, consecutive red and black
// half-sweeps run as one fused pass over row tiles (the level keeps a second
// correction buffer for it); the results are those of the single
// half-sweeps bit for bit. The last red half-sweep of the finest level is
// left to the caller, which fuses it with the outer method's dot products
// (k_mg_finish_red).
#pragma once

#include <vector>

#include "internal.hpp"

namespace rb200 {

// One level of the hierarchy, passed by value to the kernels.
struct MgLevelDev {
    int n[3];
    int cells;
    int cf[3];        // coarsening factor to the next level per axis (1 or 2)
    float w[3];       // rediscretised face weights
    float dinv[64];   // 1/diagonal by neighbour mask
    float* x;         // correction (FP32)
    float* b;         // right-hand side (FP32); level 0's is f32(r)
};

constexpr int kMgLowerCells = 32768;   // levels of at most 32^3 cells: one cluster kernel
constexpr int kMgMaxLower = 16;

// The levels handled by the cluster kernel, the coarsest last.
struct MgLower {
    // lv[0][q]: level q with its own correction buffer; lv[1][q]: the same
    // level with its second buffer (fused pairs), or lv[0][q] again
    MgLevelDev lv[2][kMgMaxLower];
    int paired[kMgMaxLower];
    int count;
};

// The hierarchy of a grid (geometry and tables; no buffers): every axis longer
// than 8 cells is halved, rounding up, until all are at most 8.
std::vector<MgLevelDev> mg_level_geometry(const GridDev& g);
// The FP64 pseudo-inverse of the coarsest level's operator (cells x cells,
// row-major); false when the level has more than 512 cells or is singular
// beyond its constant null space.
bool mg_coarse_pseudo_inverse(const MgLevelDev& C, std::vector<double>& G);
// Whether a level's red and black half-sweeps can run as one fused pair
// (rows a multiple of 4 long, tile rows within the shared-memory limit).
bool mg_level_pairable(const MgLevelDev& L);

class Multigrid {
public:
    Multigrid() = default;
    ~Multigrid();
    Multigrid(const Multigrid&) = delete;
    Multigrid& operator=(const Multigrid&) = delete;

    int init(const GridDev& g, cudaStream_t s);
    // Enqueue one V-cycle, b0 = f32(r) -> x0, except the final red half-sweep
    // of level 0 (k_mg_finish_red) when the hierarchy has more than one level.
    // Kernels are gated on the solver flags by `mode` (0 init, 1 iteration,
    // 2 restart). Returns the number of launches.
    // With first_done the finest level's first red half-sweep is taken as done
    // (by enqueue_update_first).
    int enqueue(const double* r, const void* state, int mode, cudaStream_t s, bool first_done = false) const;
    // Whether enqueue_update_first applies (the finest level is a grid-kernel
    // level), and the fused flexible-CG update + first red half-sweep.
    bool fuses_update() const { return lower_first_ > 0; }
    // r0 and r1 are the two residual buffers (the state's rsel tells which
    // holds r; the update writes the other).
    int enqueue_update_first(const GridDev& g, void* state, double* p, double* r0, double* r1, double* d0,
                             double* d1, Partials part, rb200_trace* trace, cudaStream_t s) const;
    // The finish: last red half-sweep of level 0 (when there is a hierarchy),
    // r.z and z.r_old with z = x (z[0] = 0), and the flexible-CG decision. z
    // stays in the finest level's x (FP32); enqueue_pass1 reads it there.
    int enqueue_finish(void* state, const double* r0, const double* r1, int mode, Partials part,
                       rb200_trace* trace, cudaStream_t s) const;
    // The flexible-CG direction pass reading z from the finest level's x.
    int enqueue_pass1(const GridDev& g, void* state, double* d0, double* d1, Partials part, rb200_trace* trace,
                      cudaStream_t s) const;
    const MgLevelDev& fine() const { return levels_[0]; }
    int levels() const { return int(levels_.size()); }
    size_t bytes() const { return bytes_; }

private:
    std::vector<MgLevelDev> levels_;
    double* dense_ = nullptr;   // coarsest-grid pseudo-inverse, cells x cells (FP64)
    int lower_first_ = 0;       // first level handled by the cluster kernel
    int cluster_ = 0;           // CTAs of that kernel's cluster
    size_t bytes_ = 0;
    // Second correction buffer of each level smoothed by fused red-black
    // pairs (nullptr: the level runs single half-sweeps).
    std::vector<float*> alt_;
};

}  // namespace rb200
