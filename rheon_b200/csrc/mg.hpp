// Mixed-precision geometric multigrid preconditioner for the sealed-box
// pressure system (new; the reference has no multigrid).
//
// One V(2,2) cycle in FP32 on a hierarchy of cell-centred grids: symmetric
// red-black Gauss-Seidel smoothing (red then black before, black then red
// after), residual restriction by summing the children (integrated RHS),
// piecewise-constant prolongation (the transpose of the restriction), and
// rediscretised coarse operators. The coarsest grid (at most 4096 cells) is
// solved in FP64 by conjugate gradients in one thread block, on the
// mean-projected singular Neumann system. The cycle is a fixed symmetric
// operator up to FP32 rounding; the outer FP64 flexible CG absorbs the rest.
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
    float* b;         // right-hand side (FP32); level 0 reads the FP64 residual
};

constexpr int kMgMaxCoarseCells = 4096;

class Multigrid {
public:
    Multigrid() = default;
    ~Multigrid();
    Multigrid(const Multigrid&) = delete;
    Multigrid& operator=(const Multigrid&) = delete;

    // Builds the hierarchy for a fine grid; RB200_UNSUPPORTED if the coarsest
    // grid it can reach is larger than kMgMaxCoarseCells.
    int init(const GridDev& g, cudaStream_t s);
    // Enqueue one V-cycle on `stream`: b0 = residual r (FP64) -> x0 (FP32).
    // Every kernel is gated on the solver flags by `mode` (0 init, 1 iteration,
    // 2 restart), like the other preconditioner kernels. Returns launches.
    int enqueue(const double* r, const void* state, int mode, cudaStream_t s) const;
    const float* x0() const { return levels_.empty() ? nullptr : levels_[0].x; }
    size_t bytes() const { return bytes_; }
    int levels() const { return int(levels_.size()); }

private:
    std::vector<MgLevelDev> levels_;
    size_t bytes_ = 0;
    size_t coarse_smem_ = 0;
};

}  // namespace rb200
