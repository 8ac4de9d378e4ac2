// FP32 geometric multigrid V(2,2) with an FP64 coarsest-grid solve; the
// preconditioner of the mixed-precision pressure method (see mg.hpp).
#include <algorithm>
#include <cmath>
#include <utility>
#include <vector>

#include "mg_device.cuh"
#include "slab.cuh"

namespace rb200 {

// ------------------------------------------------------------ grid kernels (large levels)
__global__ void __launch_bounds__(MG_THREADS) k_mg_smooth(MgLevelDev L, const double* __restrict__ r0, int color,
                                                          int first, const SolveState* st, int mode) {
    pdl_wait();
    if (!mg_gate(st, mode)) return;
    smooth_rows<false>(L, r0, color, first != 0, grid_warps());
}



__global__ void __launch_bounds__(MG_THREADS) k_mg_smooth_pair(MgLevelDev L, float* __restrict__ x_out, int c1,
                                                               int first, const SolveState* st, int mode) {
    pdl_wait();
    extern __shared__ float4 srow[];  // PAIR_ROWS rows of n0/4 quads
    if (!mg_gate(st, mode)) return;
    const int tj = (L.n[1] + PJ - 1) / PJ;
    pair_tile<false, PJ, PK>(L, x_out, c1, first != 0, int(blockIdx.x % unsigned(tj)) * PJ,
                             int(blockIdx.x / unsigned(tj)) * PK, srow);
}

__global__ void __launch_bounds__(MG_THREADS) k_mg_restrict(MgLevelDev L, MgLevelDev C, const SolveState* st,
                                                            int mode) {
    pdl_wait();
    if (!mg_gate(st, mode)) return;
    restrict_rows<false>(L, C, grid_warps());
}

__global__ void __launch_bounds__(MG_THREADS) k_mg_prolong_black(MgLevelDev L, MgLevelDev C, const SolveState* st,
                                                                 int mode) {
    pdl_wait();
    if (!mg_gate(st, mode)) return;
    prolong_black_rows<false>(L, C, grid_warps());
}

__global__ void __launch_bounds__(MG_LOWER_THREADS, 1) k_mg_lower(MgLower P, const double* __restrict__ r0,
                                                               const double* __restrict__ G,
                                                               const SolveState* st, int mode, int skip_last_red) {
    pdl_wait();
    __shared__ double bs[512];
    __shared__ float4 prow[kLowerPairRows];
    if (!mg_gate(st, mode)) return;  // uniform: every CTA reads the same flags
    lower_body(P, r0, G, skip_last_red, bs, prow);
}

// ------------------------------------------------------------ host side
// Launch of a V-cycle kernel that may overlap the drain of the kernel before
// it on the stream (programmatic stream serialisation); the kernel waits for
// it in pdl_wait before its first memory access.
template <typename... KArgs, typename... Args>
static void pdl_launch(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args&&... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

Multigrid::~Multigrid() {
    for (auto& L : levels_) {
        cudaFree(L.x);
        cudaFree(L.b);
    }
    for (float* a : alt_) cudaFree(a);
    cudaFree(dense_);
}

static void level_tables(MgLevelDev& L, const double w[3]) {
    for (int d = 0; d < 3; ++d) L.w[d] = float(w[d]);
    for (int mask = 0; mask < 64; ++mask) {
        double D = 0.0;
        for (int side = 0; side < 6; ++side)
            if (mask & (1 << side)) D += double(L.w[side / 2]);
        L.dinv[mask] = D > 0.0 ? float(1.0 / D) : 0.0f;
    }
}

// Mean-projected pseudo-inverse of the coarsest operator K (singular Neumann,
// null space = constants): A = K + s/M * 1 1^T is SPD and agrees with K on
// mean-zero vectors, so G = P A^-1 P with P = I - 1 1^T / M. Cholesky in FP64.
static bool coarse_pseudo_inverse(const MgLevelDev& C, std::vector<double>& G) {
    const int M = C.cells;
    const int n0 = C.n[0], n1 = C.n[1], n2 = C.n[2];
    std::vector<double> A(size_t(M) * M, 0.0);
    const double w[3] = {double(C.w[0]), double(C.w[1]), double(C.w[2])};
    double trace = 0.0;
    for (int c = 0; c < M; ++c) {
        const int i = c % n0, j = (c / n0) % n1, k = c / (n0 * n1);
        const int nb[6] = {i > 0 ? c - 1 : -1, i + 1 < n0 ? c + 1 : -1, j > 0 ? c - n0 : -1,
                           j + 1 < n1 ? c + n0 : -1, k > 0 ? c - n0 * n1 : -1, k + 1 < n2 ? c + n0 * n1 : -1};
        for (int s = 0; s < 6; ++s)
            if (nb[s] >= 0) {
                A[size_t(c) * M + c] += w[s / 2];
                A[size_t(c) * M + nb[s]] -= w[s / 2];
            }
        trace += A[size_t(c) * M + c];
    }
    const double shift = (trace > 0.0 ? trace / M : 1.0) / M;
    for (size_t e = 0; e < A.size(); ++e) A[e] += shift;
    // Cholesky A = L L^T (lower triangle, in place)
    for (int j = 0; j < M; ++j) {
        double d = A[size_t(j) * M + j];
        for (int k = 0; k < j; ++k) d -= A[size_t(j) * M + k] * A[size_t(j) * M + k];
        if (!(d > 0.0)) return false;
        d = std::sqrt(d);
        A[size_t(j) * M + j] = d;
        for (int i = j + 1; i < M; ++i) {
            double s = A[size_t(i) * M + j];
            for (int k = 0; k < j; ++k) s -= A[size_t(i) * M + k] * A[size_t(j) * M + k];
            A[size_t(i) * M + j] = s / d;
        }
    }
    // X = A^-1 P column by column, then G = P X.
    G.assign(size_t(M) * M, 0.0);
    std::vector<double> y(M);
    for (int col = 0; col < M; ++col) {
        for (int i = 0; i < M; ++i) y[i] = (i == col ? 1.0 : 0.0) - 1.0 / M;
        for (int i = 0; i < M; ++i) {
            double s = y[i];
            for (int k = 0; k < i; ++k) s -= A[size_t(i) * M + k] * y[k];
            y[i] = s / A[size_t(i) * M + i];
        }
        for (int i = M - 1; i >= 0; --i) {
            double s = y[i];
            for (int k = i + 1; k < M; ++k) s -= A[size_t(k) * M + i] * y[k];
            y[i] = s / A[size_t(i) * M + i];
        }
        double mean = 0.0;
        for (int i = 0; i < M; ++i) mean += y[i];
        mean /= M;
        for (int i = 0; i < M; ++i) G[size_t(i) * M + col] = y[i] - mean;
    }
    return true;
}

std::vector<MgLevelDev> mg_level_geometry(const GridDev& g) {
    std::vector<MgLevelDev> out;
    double h[3] = {g.h[0], g.h[1], g.h[2]};
    const double rho = g.area[0] / (g.weight[0] * g.h[0]);  // w = area/(rho h)
    int n[3] = {g.n[0], g.n[1], g.n[2]};
    for (;;) {
        MgLevelDev L{};
        for (int d = 0; d < 3; ++d) L.n[d] = n[d];
        L.cells = n[0] * n[1] * n[2];
        const double area[3] = {h[1] * h[2], h[0] * h[2], h[0] * h[1]};
        double w[3];
        for (int d = 0; d < 3; ++d) w[d] = area[d] / (rho * h[d]);
        level_tables(L, w);
        bool coarser = false;
        for (int d = 0; d < 3; ++d) {
            L.cf[d] = n[d] > 8 ? 2 : 1;
            coarser = coarser || L.cf[d] == 2;
        }
        out.push_back(L);
        if (!coarser) break;
        for (int d = 0; d < 3; ++d) {
            h[d] *= L.cf[d];
            n[d] = (n[d] + L.cf[d] - 1) / L.cf[d];
        }
    }
    return out;
}

bool mg_coarse_pseudo_inverse(const MgLevelDev& C, std::vector<double>& G) {
    return C.cells <= 512 && coarse_pseudo_inverse(C, G);
}

bool mg_level_pairable(const MgLevelDev& L) {
    return (L.n[0] & 3) == 0 && size_t(PAIR_ROWS) * size_t(L.n[0]) * sizeof(float) <= kPairSmemMax;
}

int Multigrid::init(const GridDev& g, cudaStream_t s) {
    for (MgLevelDev L : mg_level_geometry(g)) {
        const bool ok_x = cudaMalloc(&L.x, size_t(L.cells) * sizeof(float)) == cudaSuccess;
        const bool ok_b = ok_x && cudaMalloc(&L.b, size_t(L.cells) * sizeof(float)) == cudaSuccess;
        levels_.push_back(L);
        if (!ok_b) return RB200_OUT_OF_MEMORY;
        bytes_ += 2 * size_t(L.cells) * sizeof(float);
    }
    const MgLevelDev& C = levels_.back();
    std::vector<double> G;
    if (!mg_coarse_pseudo_inverse(C, G)) {
        set_error("multigrid coarsest-level factorisation failed");
        return RB200_UNSUPPORTED;
    }
    RB200_CUDA(cudaMalloc(&dense_, G.size() * sizeof(double)));
    bytes_ += G.size() * sizeof(double);
    RB200_CUDA(cudaMemcpyAsync(dense_, G.data(), G.size() * sizeof(double), cudaMemcpyHostToDevice, s));
    RB200_CUDA(cudaStreamSynchronize(s));
    const int nl = int(levels_.size());
    lower_first_ = nl - 1;
    while (lower_first_ > 0 && levels_[lower_first_ - 1].cells <= kMgLowerCells) --lower_first_;
    if (nl - lower_first_ > kMgMaxLower) {
        set_error("multigrid hierarchy too deep for one cluster kernel");
        return RB200_UNSUPPORTED;
    }
    // Fused red-black pairs on the grid-kernel levels whose rows are a
    // multiple of 4 long and whose tile rows fit in shared memory.
    alt_.assign(levels_.size(), nullptr);
    size_t pair_smem = 0;
    for (int l = 0; l < lower_first_; ++l) {
        const MgLevelDev& L = levels_[l];
        const size_t smem = size_t(PAIR_ROWS) * size_t(L.n[0]) * sizeof(float);
        if (!mg_level_pairable(L)) continue;
        RB200_CUDA(cudaMalloc(&alt_[l], size_t(L.cells) * sizeof(float)));
        bytes_ += size_t(L.cells) * sizeof(float);
        pair_smem = std::max(pair_smem, smem);
    }
    if (pair_smem)
        RB200_CUDA(cudaFuncSetAttribute(k_mg_smooth_pair, cudaFuncAttributeMaxDynamicSharedMemorySize, int(pair_smem)));
    // and on the cluster kernel's levels above the dense one with short rows
    for (int l = lower_first_; l + 1 < nl; ++l) {
        const MgLevelDev& L = levels_[l];
        if ((L.n[0] & 3) != 0 || L.n[0] > LPAIR_N0) continue;
        RB200_CUDA(cudaMalloc(&alt_[l], size_t(L.cells) * sizeof(float)));
        bytes_ += size_t(L.cells) * sizeof(float);
    }
    // The largest cluster the device schedules for the lower-level kernel:
    // 16 CTAs (non-portable) where available, else 8.
    RB200_CUDA(cudaFuncSetAttribute(k_mg_lower, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    cluster_ = 0;
    for (int cl : {16, 8, 4, 2, 1}) {
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = dim3(unsigned(cl), 1, 1);
        cfg.blockDim = dim3(MG_LOWER_THREADS, 1, 1);
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = unsigned(cl);
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int clusters = 0;
        if (cudaOccupancyMaxActiveClusters(&clusters, k_mg_lower, &cfg) == cudaSuccess && clusters >= 1) {
            cluster_ = cl;
            break;
        }
        cudaGetLastError();
    }
    if (!cluster_) {
        set_error("no thread-block cluster fits the multigrid lower-level kernel");
        return RB200_UNSUPPORTED;
    }
    return RB200_OK;
}

// Blocks of a level loop: one warp per row (j, k) of the level, at most 16
// blocks per SM.
static int row_blocks(const MgLevelDev& L, int per = 32) {
    const long rows = long(L.n[1]) * L.n[2];
    const long rpw = 32 / lanes_for(per);  // rows per warp
    const long warps = (rows + rpw - 1) / rpw;
    const long per_block = MG_THREADS / 32;
    long b = (warps + per_block - 1) / per_block;
    if (b < 1) b = 1;
    return int(b < 148 * 16 ? b : 148 * 16);
}

int Multigrid::enqueue(const double* r, const void* state, int mode, cudaStream_t s, bool first_done) const {
    const SolveState* st = static_cast<const SolveState*>(state);
    const int nl = int(levels_.size());
    int launches = 0;
    // Level l with its correction in buffer `which` (0: its own x, 1: the
    // second buffer of the fused pairs).
    auto with_x = [&](int l, int which) {
        MgLevelDev L = levels_[l];
        if (which) L.x = alt_[l];
        return L;
    };
    // A fused pair (colour c1, then the other) from buffer `from` into the
    // other buffer; returns the buffer that holds the result.
    auto pair = [&](int l, int from, int c1, bool first) {
        const MgLevelDev L = with_x(l, from);
        const int tiles = ((L.n[1] + PJ - 1) / PJ) * ((L.n[2] + PK - 1) / PK);
        const size_t smem = size_t(PAIR_ROWS) * size_t(L.n[0]) * sizeof(float);
        pdl_launch(k_mg_smooth_pair, dim3(tiles), dim3(MG_THREADS), smem, s, L, from ? levels_[l].x : alt_[l], c1,
                   first ? 1 : 0, st, mode);
        launches += 1;
        return 1 - from;
    };
    std::vector<int> cur(levels_.size(), 0);  // buffer of each grid-kernel level's correction
    // Descent on the large levels.
    for (int l = 0; l < lower_first_; ++l) {
        const MgLevelDev& L = levels_[l];
        const int pb = row_blocks(L, sweep_items(L));
        if (alt_[l]) {
            // red, black, red, black as pairs; on the finest level the first
            // red is done by the update kernel or converts the residual here
            if (l == 0) {
                if (!first_done) {
                    pdl_launch(k_mg_smooth, dim3(pb), dim3(MG_THREADS), 0, s, L, r, 0, 1, st, mode);
                    launches += 1;
                }
                cur[0] = pair(0, 0, 1, false);
                pdl_launch(k_mg_smooth, dim3(pb), dim3(MG_THREADS), 0, s, with_x(0, cur[0]), nullptr, 1, 0, st, mode);
                launches += 1;
            } else {
                cur[l] = pair(l, 0, 0, true);
                cur[l] = pair(l, cur[l], 0, false);
            }
        } else {
            for (int sweep = 0; sweep < 2; ++sweep) {
                // the finest level's first red half-sweep may already be done
                // (k_mg_update_first)
                if (!(l == 0 && sweep == 0 && first_done)) {
                    pdl_launch(k_mg_smooth, dim3(pb), dim3(MG_THREADS), 0, s, L, (l == 0 && sweep == 0) ? r : nullptr,
                               0, sweep == 0, st, mode);
                    launches += 1;
                }
                pdl_launch(k_mg_smooth, dim3(pb), dim3(MG_THREADS), 0, s, L, nullptr, 1, 0, st, mode);
                launches += 1;
            }
        }
        pdl_launch(k_mg_restrict, dim3(row_blocks(levels_[l + 1], restrict_items(L, levels_[l + 1]))), dim3(MG_THREADS),
                   0, s, with_x(l, cur[l]), levels_[l + 1], st, mode);
        launches += 1;
    }
    // The lower levels, coarsest solve included, in one cluster.
    MgLower P{};
    P.count = nl - lower_first_;
    for (int q = 0; q < P.count; ++q) {
        P.lv[0][q] = levels_[lower_first_ + q];
        P.lv[1][q] = levels_[lower_first_ + q];
        P.paired[q] = alt_[lower_first_ + q] ? 1 : 0;
        if (P.paired[q]) P.lv[1][q].x = alt_[lower_first_ + q];
    }
    {
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = dim3(unsigned(cluster_), 1, 1);
        cfg.blockDim = dim3(MG_LOWER_THREADS, 1, 1);
        cfg.stream = s;
        cudaLaunchAttribute attr[2];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = unsigned(cluster_);
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[1].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 2;
        const double* r0 = lower_first_ == 0 ? r : nullptr;
        const double* G = dense_;
        const int skip = (lower_first_ == 0 && nl > 1) ? 1 : 0;
        cudaLaunchKernelEx(&cfg, k_mg_lower, P, r0, G, st, mode, skip);
        launches += 1;
    }
    // Ascent on the large levels; the finest level's last red half-sweep is
    // fused by the caller into its finish kernel. With fused pairs the finest
    // level ends in its own x, where the finish kernel and the direction pass
    // read it.
    for (int l = lower_first_ - 1; l >= 0; --l) {
        const MgLevelDev L = with_x(l, cur[l]);
        // the cluster kernel leaves its first level in the second buffer when
        // that level is a paired coarse level (two pairs down, one up)
        const MgLevelDev C = with_x(l + 1, l + 1 < lower_first_ ? cur[l + 1] : (alt_[l + 1] ? 1 : 0));
        const int pb = row_blocks(L, sweep_items(L));
        pdl_launch(k_mg_prolong_black, dim3(pb), dim3(MG_THREADS), 0, s, L, C, st, mode);
        launches += 1;
        if (alt_[l]) {
            cur[l] = pair(l, cur[l], 0, false);
            if (l > 0) {
                pdl_launch(k_mg_smooth, dim3(pb), dim3(MG_THREADS), 0, s, with_x(l, cur[l]), nullptr, 0, 0, st, mode);
                launches += 1;
            }
        } else {
            pdl_launch(k_mg_smooth, dim3(pb), dim3(MG_THREADS), 0, s, L, nullptr, 0, 0, st, mode);
            pdl_launch(k_mg_smooth, dim3(pb), dim3(MG_THREADS), 0, s, L, nullptr, 1, 0, st, mode);
            launches += 2;
            if (l > 0) {
                pdl_launch(k_mg_smooth, dim3(pb), dim3(MG_THREADS), 0, s, L, nullptr, 0, 0, st, mode);
                launches += 1;
            }
        }
    }
    return launches;
}

// ------------------------------------------------------------ flexible-CG kernels
__global__ void __launch_bounds__(MG_THREADS) k_mg_finish_red(MgLevelDev L, int smooth, SolveState* st,
                                                              const double* r0, const double* r1, int mode,
                                                              Partials part, rb200_trace* trace) {
    pdl_wait();
    finish_red_body(L, smooth, st, r0, r1, mode, part, trace, whole_launch());
}

__global__ void __launch_bounds__(MG_THREADS) k_mg_pass1(GridDev g, MgLevelDev L, SolveState* st, double* d0,
                                                         double* d1, Partials part, rb200_trace* trace, int kc_len) {
    pdl_wait();
    pass1_body(g, L, st, d0, d1, part, trace, kc_len, whole_launch());
}

__global__ void __launch_bounds__(MG_THREADS) k_mg_update_first(GridDev g, MgLevelDev L, SolveState* st,
                                                                double* __restrict__ p, double* r0, double* r1,
                                                                const double* d0, const double* d1, Partials part,
                                                                rb200_trace* trace) {
    pdl_wait();
    update_first_body(g, L, st, p, r0, r1, d0, d1, part, trace, whole_launch());
}


int Multigrid::enqueue_update_first(const GridDev& g, void* state, double* p, double* r0, double* r1, double* d0,
                                    double* d1, Partials part, rb200_trace* trace, cudaStream_t s) const {
    int pb = row_blocks(levels_[0]);
    if (pb > 148 * 8) pb = 148 * 8;  // reduction partials capacity
    pdl_launch(k_mg_update_first, dim3(pb), dim3(MG_THREADS), 0, s, g, levels_[0], static_cast<SolveState*>(state), p,
               r0, r1, d0, d1, part, trace);
    return 1;
}

int Multigrid::enqueue_pass1(const GridDev& g, void* state, double* d0, double* d1, Partials part,
                             rb200_trace* trace, cudaStream_t s) const {
    int pb = row_blocks(levels_[0]);
    if (pb > 148 * 8) pb = 148 * 8;  // reduction partials capacity
    // the z-march length of the quad path: long where there are enough lines
    // for every warp of the grid, short otherwise
    const int quads = g.n[0] / 4, qsegs = (quads + 31) / 32;
    const int warps = pb * (MG_THREADS / 32);
    int kc_len = 16;
    while (kc_len > 2 && qsegs * g.n[1] * ((g.n[2] + kc_len - 1) / kc_len) < warps) kc_len /= 2;
    pdl_launch(k_mg_pass1, dim3(pb), dim3(MG_THREADS), 0, s, g, levels_[0], static_cast<SolveState*>(state), d0, d1,
               part, trace, kc_len);
    return 1;
}

int Multigrid::enqueue_finish(void* state, const double* r0, const double* r1, int mode, Partials part,
                              rb200_trace* trace, cudaStream_t s) const {
    const MgLevelDev& L = levels_[0];
    int pb = row_blocks(L);
    if (pb > 148 * 8) pb = 148 * 8;  // reduction partials capacity
    pdl_launch(k_mg_finish_red, dim3(pb), dim3(MG_THREADS), 0, s, L, levels_.size() > 1 ? 1 : 0,
               static_cast<SolveState*>(state), r0, r1, mode, part, trace);
    return 1;
}

}  // namespace rb200
