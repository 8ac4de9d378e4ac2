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
// Launch structure of one cycle: grid-wide kernels for the levels above 4096
// cells, one single-block kernel for the whole descent and one for the ascent
// through the levels of at most 4096 cells, a many-block dense coarse solve.
// The last red half-sweep of the finest level is left to the caller, which
// fuses it with the outer method's dot products (k_mg_finish_red).
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

constexpr int kMgBottomCells = 4096;   // levels handled by single-block kernels
constexpr int kMgMaxBottom = 6;

struct MgBottom {
    MgLevelDev lv[kMgMaxBottom + 1];   // bottom levels and the coarsest level
    int count;                         // bottom levels (excluding the coarsest)
};

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
    int enqueue(const double* r, const void* state, int mode, cudaStream_t s) const;
    // The finish: last red half-sweep of level 0 (when there is a hierarchy),
    // z = x with z[0] = 0, r.z and z.q, and the flexible-CG decision.
    int enqueue_finish(void* state, double* z, const double* r, const double* q, int mode, Partials part,
                       rb200_trace* trace, cudaStream_t s) const;
    const MgLevelDev& fine() const { return levels_[0]; }
    int levels() const { return int(levels_.size()); }
    size_t bytes() const { return bytes_; }

private:
    std::vector<MgLevelDev> levels_;
    double* dense_ = nullptr;   // coarsest-grid pseudo-inverse, cells x cells (FP64)
    int bottom_first_ = 0;      // first level handled by the single-block kernels
    size_t bytes_ = 0;
};

}  // namespace rb200
