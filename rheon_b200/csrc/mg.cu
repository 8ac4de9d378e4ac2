// FP32 geometric multigrid V(2,2) with an FP64 coarsest-grid solve; the
// preconditioner of the mixed-precision pressure method (see mg.hpp).
#include <cmath>
#include <vector>

#include "mg.hpp"
#include "pcg.hpp"
#include "slab.cuh"
#include "solve_state.cuh"

namespace rb200 {

constexpr int MG_THREADS = 256;
constexpr int MG_BOTTOM_THREADS = 1024;

__device__ __forceinline__ bool mg_gate(const SolveState* st, int mode) { return gate(st->flags, mode); }

__device__ __forceinline__ int mask_of(const int n[3], int i, int j, int k) {
    return int(i > 0) | (int(i + 1 < n[0]) << 1) | (int(j > 0) << 2) | (int(j + 1 < n[1]) << 3) |
           (int(k > 0) << 4) | (int(k + 1 < n[2]) << 5);
}

__host__ __device__ __forceinline__ long mg_pairs(const MgLevelDev& L) {
    return long((L.n[0] + 1) >> 1) * L.n[1] * L.n[2];
}

// Pair mapping of a red-black half-sweep: pair t covers cells 2m and 2m+1 of
// row (j, k); (i, j, k) is the cell of colour `color` in it (i may be n0).
__device__ __forceinline__ void pair_cell(const MgLevelDev& L, long t, int color, int& i, int& j, int& k) {
    const int hx = (L.n[0] + 1) >> 1;
    const int m = int(t % hx);
    const long row = t / hx;
    j = int(row % L.n[1]);
    k = int(row / L.n[1]);
    i = 2 * m + ((color + j + k) & 1);
}

// Gauss-Seidel value x = (b + sum_nb w x_nb) / D, summed x-, x+, y-, y+, z-, z+.
__device__ __forceinline__ float gs_value(const MgLevelDev& L, float b, int i, int j, int k, int c) {
    const int sy = L.n[0], sz = L.n[0] * L.n[1];
    const float* __restrict__ x = L.x;
    float s = b;
    if (i > 0) s += L.w[0] * x[c - 1];
    if (i + 1 < L.n[0]) s += L.w[0] * x[c + 1];
    if (j > 0) s += L.w[1] * x[c - sy];
    if (j + 1 < L.n[1]) s += L.w[1] * x[c + sy];
    if (k > 0) s += L.w[2] * x[c - sz];
    if (k + 1 < L.n[2]) s += L.w[2] * x[c + sz];
    return s * L.dinv[mask_of(L.n, i, j, k)];
}

// Half-sweep of colour `color` over pairs [t0, pairs) step dt. With `first`
// the correction starts from zero (red = b/D, black cleared); with r0 the FP32
// right-hand side of the finest level is converted from the FP64 residual on
// the way (both cells of the pair).
__device__ __forceinline__ void smooth_pairs(const MgLevelDev& L, const double* __restrict__ r0, int color,
                                             bool first, long t0, long dt) {
    const long pairs = mg_pairs(L);
    for (long t = t0; t < pairs; t += dt) {
        int i, j, k;
        pair_cell(L, t, color, i, j, k);
        const int io = i ^ 1;
        const int row = L.n[0] * (j + L.n[1] * k);
        if (first && io < L.n[0]) {
            if (r0) L.b[io + row] = float(r0[io + row]);
            L.x[io + row] = 0.0f;
        }
        if (i >= L.n[0]) continue;
        const int c = i + row;
        float b;
        if (r0) {
            b = float(r0[c]);
            L.b[c] = b;
        } else {
            b = L.b[c];
        }
        L.x[c] = first ? b * L.dinv[mask_of(L.n, i, j, k)] : gs_value(L, b, i, j, k, c);
    }
}

// Residual b - K x on the fine cells summed over each coarse cell's children
// (restriction = transpose of the piecewise-constant prolongation).
__device__ __forceinline__ void restrict_cells(const MgLevelDev& L, const MgLevelDev& C, int c0, int dc) {
    const int sy = L.n[0], sz = L.n[0] * L.n[1];
    for (int cc = c0; cc < C.cells; cc += dc) {
        const int I = cc % C.n[0], J = (cc / C.n[0]) % C.n[1], K = cc / (C.n[0] * C.n[1]);
        float sum = 0.0f;
        for (int dk = 0; dk < L.cf[2]; ++dk)
            for (int dj = 0; dj < L.cf[1]; ++dj)
                for (int di = 0; di < L.cf[0]; ++di) {
                    const int i = I * L.cf[0] + di, j = J * L.cf[1] + dj, k = K * L.cf[2] + dk;
                    if (i >= L.n[0] || j >= L.n[1] || k >= L.n[2]) continue;
                    const int c = i + L.n[0] * (j + L.n[1] * k);
                    const float xc = L.x[c];
                    float kx = 0.0f;
                    if (i > 0) kx += L.w[0] * (xc - L.x[c - 1]);
                    if (i + 1 < L.n[0]) kx += L.w[0] * (xc - L.x[c + 1]);
                    if (j > 0) kx += L.w[1] * (xc - L.x[c - sy]);
                    if (j + 1 < L.n[1]) kx += L.w[1] * (xc - L.x[c + sy]);
                    if (k > 0) kx += L.w[2] * (xc - L.x[c - sz]);
                    if (k + 1 < L.n[2]) kx += L.w[2] * (xc - L.x[c + sz]);
                    sum += L.b[c] - kx;
                }
        C.b[cc] = sum;
    }
}

__device__ __forceinline__ float coarse_at(const MgLevelDev& L, const MgLevelDev& C, int i, int j, int k) {
    return C.x[(i >> (L.cf[0] - 1)) + C.n[0] * ((j >> (L.cf[1] - 1)) + C.n[1] * (k >> (L.cf[2] - 1)))];
}

// Prolongation fused with the first post-smoothing half-sweep (black): black
// cells are relaxed against their red neighbours' corrected values x + P xc,
// formed on the fly. Red cells are not written: the red half-sweep that
// follows replaces every red value without reading it. Nothing this pass reads
// is written by it.
__device__ __forceinline__ void prolong_black_pairs(const MgLevelDev& L, const MgLevelDev& C, long t0, long dt) {
    const long pairs = mg_pairs(L);
    const int sy = L.n[0], sz = L.n[0] * L.n[1];
    for (long t = t0; t < pairs; t += dt) {
        int i, j, k;
        pair_cell(L, t, 1, i, j, k);
        if (i >= L.n[0]) continue;
        const int c = i + L.n[0] * (j + L.n[1] * k);
        float s = L.b[c];
        if (i > 0) s += L.w[0] * (L.x[c - 1] + coarse_at(L, C, i - 1, j, k));
        if (i + 1 < L.n[0]) s += L.w[0] * (L.x[c + 1] + coarse_at(L, C, i + 1, j, k));
        if (j > 0) s += L.w[1] * (L.x[c - sy] + coarse_at(L, C, i, j - 1, k));
        if (j + 1 < L.n[1]) s += L.w[1] * (L.x[c + sy] + coarse_at(L, C, i, j + 1, k));
        if (k > 0) s += L.w[2] * (L.x[c - sz] + coarse_at(L, C, i, j, k - 1));
        if (k + 1 < L.n[2]) s += L.w[2] * (L.x[c + sz] + coarse_at(L, C, i, j, k + 1));
        L.x[c] = s * L.dinv[mask_of(L.n, i, j, k)];
    }
}

// ------------------------------------------------------------ grid kernels
__global__ void __launch_bounds__(MG_THREADS) k_mg_smooth(MgLevelDev L, const double* __restrict__ r0, int color,
                                                          int first, const SolveState* st, int mode) {
    if (!mg_gate(st, mode)) return;
    smooth_pairs(L, r0, color, first != 0, blockIdx.x * long(blockDim.x) + threadIdx.x, long(gridDim.x) * blockDim.x);
}

__global__ void __launch_bounds__(MG_THREADS) k_mg_restrict(MgLevelDev L, MgLevelDev C, const SolveState* st,
                                                            int mode) {
    if (!mg_gate(st, mode)) return;
    restrict_cells(L, C, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

__global__ void __launch_bounds__(MG_THREADS) k_mg_prolong_black(MgLevelDev L, MgLevelDev C, const SolveState* st,
                                                                 int mode) {
    if (!mg_gate(st, mode)) return;
    prolong_black_pairs(L, C, blockIdx.x * long(blockDim.x) + threadIdx.x, long(gridDim.x) * blockDim.x);
}

// ------------------------------------------------------------ bottom levels
// The descent through the small levels in one block: two red-black sweeps,
// restriction, next level; barriers between the half-sweeps. r0 is non-null
// when the first bottom level is the finest level.
__global__ void __launch_bounds__(MG_BOTTOM_THREADS) k_mg_bottom_down(MgBottom B, const double* __restrict__ r0,
                                                                      const SolveState* st, int mode) {
    if (!mg_gate(st, mode)) return;
    for (int l = 0; l < B.count; ++l) {
        const MgLevelDev& L = B.lv[l];
        const double* src = l == 0 ? r0 : nullptr;
        for (int sweep = 0; sweep < 2; ++sweep) {
            smooth_pairs(L, sweep == 0 ? src : nullptr, 0, sweep == 0, threadIdx.x, blockDim.x);
            __syncthreads();
            smooth_pairs(L, nullptr, 1, false, threadIdx.x, blockDim.x);
            __syncthreads();
        }
        restrict_cells(L, B.lv[l + 1], threadIdx.x, blockDim.x);
        __syncthreads();
    }
}

// The ascent: prolongation + black, red, black, red per level; the final red
// half-sweep of the finest level is skipped when skip_last_red is set (the
// caller fuses it with its dot products).
__global__ void __launch_bounds__(MG_BOTTOM_THREADS) k_mg_bottom_up(MgBottom B, int skip_last_red,
                                                                    const SolveState* st, int mode) {
    if (!mg_gate(st, mode)) return;
    for (int l = B.count - 1; l >= 0; --l) {
        const MgLevelDev& L = B.lv[l];
        prolong_black_pairs(L, B.lv[l + 1], threadIdx.x, blockDim.x);
        __syncthreads();
        smooth_pairs(L, nullptr, 0, false, threadIdx.x, blockDim.x);
        __syncthreads();
        smooth_pairs(L, nullptr, 1, false, threadIdx.x, blockDim.x);
        __syncthreads();
        if (!(l == 0 && skip_last_red)) {
            smooth_pairs(L, nullptr, 0, false, threadIdx.x, blockDim.x);
            __syncthreads();
        }
    }
}

// ------------------------------------------------------------ coarsest level
// x = G b in FP64, G the mean-projected pseudo-inverse of the coarsest
// operator; one warp per row, lanes over columns, a fixed shuffle tree.
// r0 is the right-hand side when the whole grid is the coarsest level.
__global__ void __launch_bounds__(256) k_mg_dense(MgLevelDev C, const double* __restrict__ G,
                                                  const double* __restrict__ r0, const SolveState* st, int mode) {
    if (!mg_gate(st, mode)) return;
    __shared__ double bs[512];
    const int M = C.cells;
    for (int c = threadIdx.x; c < M; c += blockDim.x) bs[c] = r0 ? r0[c] : double(C.b[c]);
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (row >= M) return;
    const double* g = G + size_t(row) * M;
    double s = 0.0;
    for (int c = lane; c < M; c += 32) s += g[c] * bs[c];
    for (int m = 16; m >= 1; m >>= 1) s += __shfl_xor_sync(0xffffffffu, s, m);
    if (lane == 0) C.x[row] = float(s);
}

// ------------------------------------------------------------ host side
Multigrid::~Multigrid() {
    for (auto& L : levels_) {
        cudaFree(L.x);
        cudaFree(L.b);
    }
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

int Multigrid::init(const GridDev& g, cudaStream_t s) {
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
        const bool ok_x = cudaMalloc(&L.x, size_t(L.cells) * sizeof(float)) == cudaSuccess;
        const bool ok_b = ok_x && cudaMalloc(&L.b, size_t(L.cells) * sizeof(float)) == cudaSuccess;
        levels_.push_back(L);
        if (!ok_b) return RB200_OUT_OF_MEMORY;
        bytes_ += 2 * size_t(L.cells) * sizeof(float);
        if (!coarser) break;
        for (int d = 0; d < 3; ++d) {
            h[d] *= L.cf[d];
            n[d] = (n[d] + L.cf[d] - 1) / L.cf[d];
        }
    }
    const MgLevelDev& C = levels_.back();
    std::vector<double> G;
    if (C.cells > 512 || !coarse_pseudo_inverse(C, G)) {
        set_error("multigrid coarsest-level factorisation failed");
        return RB200_UNSUPPORTED;
    }
    RB200_CUDA(cudaMalloc(&dense_, G.size() * sizeof(double)));
    bytes_ += G.size() * sizeof(double);
    RB200_CUDA(cudaMemcpyAsync(dense_, G.data(), G.size() * sizeof(double), cudaMemcpyHostToDevice, s));
    RB200_CUDA(cudaStreamSynchronize(s));
    const int nl = int(levels_.size());
    bottom_first_ = nl - 1;
    while (bottom_first_ > 0 && levels_[bottom_first_ - 1].cells <= kMgBottomCells &&
           (nl - 1) - (bottom_first_ - 1) <= kMgMaxBottom)
        --bottom_first_;
    return RB200_OK;
}

static int mg_blocks(long work) {
    long b = (work + MG_THREADS - 1) / MG_THREADS;
    if (b < 1) b = 1;
    return int(b < 148 * 16 ? b : 148 * 16);
}

int Multigrid::enqueue(const double* r, const void* state, int mode, cudaStream_t s) const {
    const SolveState* st = static_cast<const SolveState*>(state);
    const int nl = int(levels_.size());
    const MgLevelDev& C = levels_[nl - 1];
    const int dense_blocks = (C.cells + 7) / 8;
    if (nl == 1) {
        k_mg_dense<<<dense_blocks, 256, 0, s>>>(C, dense_, r, st, mode);
        return 1;
    }
    int launches = 0;
    // Descent on the large levels.
    for (int l = 0; l < bottom_first_; ++l) {
        const MgLevelDev& L = levels_[l];
        const int pb = mg_blocks(mg_pairs(L));
        for (int sweep = 0; sweep < 2; ++sweep) {
            k_mg_smooth<<<pb, MG_THREADS, 0, s>>>(L, (l == 0 && sweep == 0) ? r : nullptr, 0, sweep == 0, st, mode);
            k_mg_smooth<<<pb, MG_THREADS, 0, s>>>(L, nullptr, 1, 0, st, mode);
        }
        k_mg_restrict<<<mg_blocks(levels_[l + 1].cells), MG_THREADS, 0, s>>>(L, levels_[l + 1], st, mode);
        launches += 5;
    }
    MgBottom B{};
    B.count = (nl - 1) - bottom_first_;
    for (int q = 0; q <= B.count; ++q) B.lv[q] = levels_[bottom_first_ + q];
    if (B.count > 0) {
        k_mg_bottom_down<<<1, MG_BOTTOM_THREADS, 0, s>>>(B, bottom_first_ == 0 ? r : nullptr, st, mode);
        launches += 1;
    }
    k_mg_dense<<<dense_blocks, 256, 0, s>>>(C, dense_, nullptr, st, mode);
    launches += 1;
    if (B.count > 0) {
        k_mg_bottom_up<<<1, MG_BOTTOM_THREADS, 0, s>>>(B, bottom_first_ == 0 ? 1 : 0, st, mode);
        launches += 1;
    }
    // Ascent on the large levels; the finest level's last red half-sweep is
    // fused by the caller into its finish kernel.
    for (int l = bottom_first_ - 1; l >= 0; --l) {
        const MgLevelDev& L = levels_[l];
        const int pb = mg_blocks(mg_pairs(L));
        k_mg_prolong_black<<<pb, MG_THREADS, 0, s>>>(L, levels_[l + 1], st, mode);
        k_mg_smooth<<<pb, MG_THREADS, 0, s>>>(L, nullptr, 0, 0, st, mode);
        k_mg_smooth<<<pb, MG_THREADS, 0, s>>>(L, nullptr, 1, 0, st, mode);
        launches += 3;
        if (l > 0) {
            k_mg_smooth<<<pb, MG_THREADS, 0, s>>>(L, nullptr, 0, 0, st, mode);
            launches += 1;
        }
    }
    return launches;
}

// ------------------------------------------------------------ finish
// The finest level's last red half-sweep fused with the outer method's
// preconditioner output: z = x (FP64, z[0] = 0 for the eliminated gauge row),
// r.z and z.q reduced and the flexible-CG decision taken. Without a hierarchy
// (a single level solved densely) z is copied from x.
__global__ void __launch_bounds__(MG_THREADS) k_mg_finish_red(MgLevelDev L, int smooth, SolveState* st,
                                                              double* __restrict__ z, const double* __restrict__ r,
                                                              const double* __restrict__ q, int mode, Partials part,
                                                              rb200_trace* trace) {
    __shared__ BlockReduce<2, 0> red;
    if (!gate(st->flags, mode)) return;
    Neu rz, zq;
    const long pairs = mg_pairs(L);
    for (long t = blockIdx.x * long(blockDim.x) + threadIdx.x; t < pairs; t += long(gridDim.x) * blockDim.x) {
        int i, j, k;
        pair_cell(L, t, 0, i, j, k);
        const int row = L.n[0] * (j + L.n[1] * k);
        const int ib = i ^ 1;
        if (ib < L.n[0]) {  // the black cell of the pair: its value is final
            const int c = ib + row;
            const double zc = c == 0 ? 0.0 : double(L.x[c]);
            z[c] = zc;
            if (c != 0) {
                rz.add(r[c] * zc);
                if (mode == MODE_ITER) zq.add(zc * q[c]);
            }
        }
        if (i < L.n[0]) {
            const int c = i + row;
            float xv = L.x[c];
            if (smooth) {
                xv = gs_value(L, L.b[c], i, j, k, c);
                L.x[c] = xv;
            }
            const double zc = c == 0 ? 0.0 : double(xv);
            z[c] = zc;
            if (c != 0) {
                rz.add(r[c] * zc);
                if (mode == MODE_ITER) zq.add(zc * q[c]);
            }
        }
    }
    dd sums[2] = {rz.as_dd(), zq.as_dd()};
    double none[1];
    block_reduce<2, 0>(red, sums, none);
    if (publish_and_check_last<2, 0>(part, blockIdx.x, gridDim.x, sums, none)) {
        fold_partials<2, 0>(part, gridDim.x, red, sums, none);
        if (threadIdx.x == 0) decide_flexible(st, trace, dd_value(sums[0]), dd_value(sums[1]), mode);
    }
}

int Multigrid::enqueue_finish(void* state, double* z, const double* r, const double* q, int mode, Partials part,
                              rb200_trace* trace, cudaStream_t s) const {
    const MgLevelDev& L = levels_[0];
    int pb = mg_blocks(mg_pairs(L));
    if (pb > 148 * 8) pb = 148 * 8;  // reduction partials capacity
    k_mg_finish_red<<<pb, MG_THREADS, 0, s>>>(L, levels_.size() > 1 ? 1 : 0, static_cast<SolveState*>(state), z, r,
                                              q, mode, part, trace);
    return 1;
}

}  // namespace rb200
