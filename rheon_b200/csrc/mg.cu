// FP32 geometric multigrid V(2,2) with an FP64 coarsest-grid solve; the
// preconditioner of the mixed-precision pressure method (see mg.hpp).
#include <cmath>

#include "mg.hpp"
#include "pcg.hpp"

namespace rb200 {

constexpr int MG_THREADS = 256;

__device__ __forceinline__ bool mg_gate(const SolveState* st, int mode) {
    const int f = st->flags;
    if (mode == 0) return !(f & F_DONE);
    if (mode == 1) return !(f & F_STOP);
    return (f & F_NEED_REPLACE) != 0;
}

__device__ __forceinline__ int mask_of(const int n[3], int i, int j, int k) {
    return int(i > 0) | (int(i + 1 < n[0]) << 1) | (int(j > 0) << 2) | (int(j + 1 < n[1]) << 3) |
           (int(k > 0) << 4) | (int(k + 1 < n[2]) << 5);
}

// Right-hand side of a level: the FP64 PCG residual on the finest level.
template <bool FINE>
__device__ __forceinline__ float rhs_at(const MgLevelDev& L, const double* __restrict__ r0, int c) {
    return FINE ? float(r0[c]) : L.b[c];
}

// Pair mapping of a red-black half-sweep: thread t owns the cells 2m and 2m+1
// of row (j, k); the cell of colour `color` among them is updated.
__device__ __forceinline__ bool pair_cell(const MgLevelDev& L, long t, int color, int& i, int& j, int& k) {
    const int hx = (L.n[0] + 1) >> 1;
    const long rows = long(L.n[1]) * L.n[2];
    if (t >= rows * hx) return false;
    const int m = int(t % hx);
    const long row = t / hx;
    j = int(row % L.n[1]);
    k = int(row / L.n[1]);
    i = 2 * m + ((color + j + k) & 1);
    return true;
}

// Gauss-Seidel update of one cell from its (current) neighbours, FP32:
//   x = (b + sum_nb w x_nb) / D, summed x-, x+, y-, y+, z-, z+.
__device__ __forceinline__ float gs_value(const MgLevelDev& L, const float* __restrict__ x, float b, int i, int j,
                                          int k, int c) {
    const int sy = L.n[0], sz = L.n[0] * L.n[1];
    float s = b;
    if (i > 0) s += L.w[0] * x[c - 1];
    if (i + 1 < L.n[0]) s += L.w[0] * x[c + 1];
    if (j > 0) s += L.w[1] * x[c - sy];
    if (j + 1 < L.n[1]) s += L.w[1] * x[c + sy];
    if (k > 0) s += L.w[2] * x[c - sz];
    if (k + 1 < L.n[2]) s += L.w[2] * x[c + sz];
    return s * L.dinv[mask_of(L.n, i, j, k)];
}

// Red-black half-sweep. With `first` the correction starts from zero: the red
// cells become b/D and the black cells of the pair are cleared.
template <bool FINE>
__global__ void __launch_bounds__(MG_THREADS) k_mg_smooth(MgLevelDev L, const double* __restrict__ r0, int color,
                                                          int first, const SolveState* st, int mode) {
    if (!mg_gate(st, mode)) return;
    const long pairs = long((L.n[0] + 1) >> 1) * L.n[1] * L.n[2];
    for (long t = blockIdx.x * long(blockDim.x) + threadIdx.x; t < pairs; t += long(gridDim.x) * blockDim.x) {
        int i, j, k;
        pair_cell(L, t, color, i, j, k);
        if (first) {
            const int io = i ^ 1;  // the other cell of the pair
            if (io < L.n[0]) L.x[io + L.n[0] * (j + L.n[1] * k)] = 0.0f;
        }
        if (i >= L.n[0]) continue;
        const int c = i + L.n[0] * (j + L.n[1] * k);
        const float b = rhs_at<FINE>(L, r0, c);
        L.x[c] = first ? b * L.dinv[mask_of(L.n, i, j, k)] : gs_value(L, L.x, b, i, j, k, c);
    }
}

// Residual b - K x on the fine cells, summed over each coarse cell's children
// into the coarse right-hand side (restriction = transpose of the
// piecewise-constant prolongation).
template <bool FINE>
__global__ void __launch_bounds__(MG_THREADS) k_mg_restrict(MgLevelDev L, MgLevelDev C, const double* __restrict__ r0,
                                                            const SolveState* st, int mode) {
    if (!mg_gate(st, mode)) return;
    const int sy = L.n[0], sz = L.n[0] * L.n[1];
    for (int cc = blockIdx.x * blockDim.x + threadIdx.x; cc < C.cells; cc += gridDim.x * blockDim.x) {
        const int I = cc % C.n[0], J = (cc / C.n[0]) % C.n[1], K = cc / (C.n[0] * C.n[1]);
        float sum = 0.0f;
        for (int dk = 0; dk < L.cf[2]; ++dk)
            for (int dj = 0; dj < L.cf[1]; ++dj)
                for (int di = 0; di < L.cf[0]; ++di) {
                    const int i = I * L.cf[0] + di, j = J * L.cf[1] + dj, k = K * L.cf[2] + dk;
                    const int c = i + L.n[0] * (j + L.n[1] * k);
                    const float xc = L.x[c];
                    float kx = 0.0f;
                    if (i > 0) kx += L.w[0] * (xc - L.x[c - 1]);
                    if (i + 1 < L.n[0]) kx += L.w[0] * (xc - L.x[c + 1]);
                    if (j > 0) kx += L.w[1] * (xc - L.x[c - sy]);
                    if (j + 1 < L.n[1]) kx += L.w[1] * (xc - L.x[c + sy]);
                    if (k > 0) kx += L.w[2] * (xc - L.x[c - sz]);
                    if (k + 1 < L.n[2]) kx += L.w[2] * (xc - L.x[c + sz]);
                    sum += rhs_at<FINE>(L, r0, c) - kx;
                }
        C.b[cc] = sum;
    }
}

__device__ __forceinline__ float coarse_at(const MgLevelDev& L, const MgLevelDev& C, int i, int j, int k) {
    return C.x[(i / L.cf[0]) + C.n[0] * ((j / L.cf[1]) + C.n[1] * (k / L.cf[2]))];
}

// Prolongation fused with the first post-smoothing half-sweep (black): black
// cells are relaxed against their red neighbours' corrected values x + P xc,
// formed on the fly. The red cells are not written: the red half-sweep that
// follows replaces every red value without reading it, so x + P xc is only
// ever needed here. Nothing this kernel reads is written by it.
template <bool FINE>
__global__ void __launch_bounds__(MG_THREADS) k_mg_prolong_black(MgLevelDev L, MgLevelDev C,
                                                                 const double* __restrict__ r0, const SolveState* st,
                                                                 int mode) {
    if (!mg_gate(st, mode)) return;
    const long pairs = long((L.n[0] + 1) >> 1) * L.n[1] * L.n[2];
    const int sy = L.n[0], sz = L.n[0] * L.n[1];
    for (long t = blockIdx.x * long(blockDim.x) + threadIdx.x; t < pairs; t += long(gridDim.x) * blockDim.x) {
        int i, j, k;
        pair_cell(L, t, 1, i, j, k);  // black cell of the pair
        if (i >= L.n[0]) continue;
        const int c = i + L.n[0] * (j + L.n[1] * k);
        float s = rhs_at<FINE>(L, r0, c);
        if (i > 0) s += L.w[0] * (L.x[c - 1] + coarse_at(L, C, i - 1, j, k));
        if (i + 1 < L.n[0]) s += L.w[0] * (L.x[c + 1] + coarse_at(L, C, i + 1, j, k));
        if (j > 0) s += L.w[1] * (L.x[c - sy] + coarse_at(L, C, i, j - 1, k));
        if (j + 1 < L.n[1]) s += L.w[1] * (L.x[c + sy] + coarse_at(L, C, i, j + 1, k));
        if (k > 0) s += L.w[2] * (L.x[c - sz] + coarse_at(L, C, i, j, k - 1));
        if (k + 1 < L.n[2]) s += L.w[2] * (L.x[c + sz] + coarse_at(L, C, i, j, k + 1));
        L.x[c] = s * L.dinv[mask_of(L.n, i, j, k)];
    }
}

// ------------------------------------------------------------ coarsest level
__device__ __forceinline__ double block_sum(double v, double* red) {
    for (int m = 16; m >= 1; m >>= 1) v += __shfl_xor_sync(0xffffffffu, v, m);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double s = 0.0;
    for (int q = 0; q < nw; ++q) s += red[q];  // same order in every thread
    return s;
}

// FP64 conjugate gradients on the mean-projected singular Neumann system of
// the coarsest level, in one block; deterministic (fixed reduction order).
// r0 (the FP64 PCG residual) is the right-hand side when the whole grid is the
// coarsest level; otherwise C.b.
__global__ void __launch_bounds__(1024) k_mg_coarse_solve(MgLevelDev C, const double* __restrict__ r0,
                                                          const SolveState* st, int mode) {
    if (!mg_gate(st, mode)) return;
    extern __shared__ __align__(16) double cs[];
    __shared__ double red[32];
    const int M = C.cells;
    double* x = cs;
    double* r = cs + M;
    double* p = cs + 2 * M;
    double* q = cs + 3 * M;
    const double w[3] = {double(C.w[0]), double(C.w[1]), double(C.w[2])};
    double part = 0.0;
    for (int c = threadIdx.x; c < M; c += blockDim.x) {
        r[c] = r0 ? r0[c] : double(C.b[c]);
        x[c] = 0.0;
        part += r[c];
    }
    const double mean = block_sum(part, red) / double(M);
    part = 0.0;
    for (int c = threadIdx.x; c < M; c += blockDim.x) {
        r[c] -= mean;
        p[c] = r[c];
        part += r[c] * r[c];
    }
    double rr = block_sum(part, red);
    const double rr0 = rr;
    const int sy = C.n[0], sz = C.n[0] * C.n[1];
    for (int it = 0; it < 400 && rr > 1e-28 * rr0 && rr > 0.0; ++it) {
        __syncthreads();
        part = 0.0;
        for (int c = threadIdx.x; c < M; c += blockDim.x) {
            const int i = c % C.n[0], j = (c / C.n[0]) % C.n[1], k = c / sz;
            const double pc = p[c];
            double kp = 0.0;
            if (i > 0) kp += w[0] * (pc - p[c - 1]);
            if (i + 1 < C.n[0]) kp += w[0] * (pc - p[c + 1]);
            if (j > 0) kp += w[1] * (pc - p[c - sy]);
            if (j + 1 < C.n[1]) kp += w[1] * (pc - p[c + sy]);
            if (k > 0) kp += w[2] * (pc - p[c - sz]);
            if (k + 1 < C.n[2]) kp += w[2] * (pc - p[c + sz]);
            q[c] = kp;
            part += pc * kp;
        }
        const double pq = block_sum(part, red);
        if (!(pq > 0.0)) break;
        const double alpha = rr / pq;
        part = 0.0;
        for (int c = threadIdx.x; c < M; c += blockDim.x) {
            x[c] += alpha * p[c];
            r[c] -= alpha * q[c];
            part += r[c] * r[c];
        }
        const double rr_new = block_sum(part, red);
        const double beta = rr_new / rr;
        rr = rr_new;
        for (int c = threadIdx.x; c < M; c += blockDim.x) p[c] = r[c] + beta * p[c];
    }
    __syncthreads();
    part = 0.0;
    for (int c = threadIdx.x; c < M; c += blockDim.x) part += x[c];
    const double xmean = block_sum(part, red) / double(M);
    for (int c = threadIdx.x; c < M; c += blockDim.x) C.x[c] = float(x[c] - xmean);
}

// ------------------------------------------------------------ host side
Multigrid::~Multigrid() {
    for (auto& L : levels_) {
        cudaFree(L.x);
        cudaFree(L.b);
    }
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

int Multigrid::init(const GridDev& g, cudaStream_t s) {
    (void)s;
    double h[3] = {g.h[0], g.h[1], g.h[2]};
    const double rho = g.area[0] / (g.weight[0] * g.h[0]);  // w = area/(rho h)
    int n[3] = {g.n[0], g.n[1], g.n[2]};
    for (;;) {
        MgLevelDev L{};
        for (int d = 0; d < 3; ++d) L.n[d] = n[d];
        L.cells = n[0] * n[1] * n[2];
        double area[3] = {h[1] * h[2], h[0] * h[2], h[0] * h[1]};
        double w[3];
        for (int d = 0; d < 3; ++d) w[d] = area[d] / (rho * h[d]);
        level_tables(L, w);
        bool coarser = false;
        for (int d = 0; d < 3; ++d) {
            L.cf[d] = (n[d] % 2 == 0 && n[d] > 8) ? 2 : 1;
            coarser = coarser || L.cf[d] == 2;
        }
        if (!coarser) L.cf[0] = L.cf[1] = L.cf[2] = 1;
        if (cudaMalloc(&L.x, size_t(L.cells) * sizeof(float)) != cudaSuccess) return RB200_OUT_OF_MEMORY;
        bytes_ += size_t(L.cells) * sizeof(float);
        if (!levels_.empty()) {
            if (cudaMalloc(&L.b, size_t(L.cells) * sizeof(float)) != cudaSuccess) {
                cudaFree(L.x);
                return RB200_OUT_OF_MEMORY;
            }
            bytes_ += size_t(L.cells) * sizeof(float);
        }
        levels_.push_back(L);
        if (!coarser) break;
        for (int d = 0; d < 3; ++d) {
            h[d] *= L.cf[d];
            n[d] /= L.cf[d];
        }
    }
    if (levels_.back().cells > kMgMaxCoarseCells) {
        set_error("multigrid needs a hierarchy that coarsens to at most 4096 cells");
        return RB200_UNSUPPORTED;
    }
    coarse_smem_ = size_t(levels_.back().cells) * 4 * sizeof(double);
    RB200_CUDA(cudaFuncSetAttribute(k_mg_coarse_solve, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    int(coarse_smem_)));
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
    int launches = 0;
    auto pairs = [](const MgLevelDev& L) { return long((L.n[0] + 1) >> 1) * L.n[1] * L.n[2]; };
    // Pre-smoothing and restriction down to the coarsest level.
    for (int l = 0; l + 1 < nl; ++l) {
        const MgLevelDev& L = levels_[l];
        const int pb = mg_blocks(pairs(L));
        const bool fine = l == 0;
        for (int sweep = 0; sweep < 2; ++sweep) {
            if (fine) {
                k_mg_smooth<true><<<pb, MG_THREADS, 0, s>>>(L, r, 0, sweep == 0, st, mode);
                k_mg_smooth<true><<<pb, MG_THREADS, 0, s>>>(L, r, 1, 0, st, mode);
            } else {
                k_mg_smooth<false><<<pb, MG_THREADS, 0, s>>>(L, r, 0, sweep == 0, st, mode);
                k_mg_smooth<false><<<pb, MG_THREADS, 0, s>>>(L, r, 1, 0, st, mode);
            }
            launches += 2;
        }
        const MgLevelDev& C = levels_[l + 1];
        if (fine)
            k_mg_restrict<true><<<mg_blocks(C.cells), MG_THREADS, 0, s>>>(L, C, r, st, mode);
        else
            k_mg_restrict<false><<<mg_blocks(C.cells), MG_THREADS, 0, s>>>(L, C, r, st, mode);
        launches += 1;
    }
    const MgLevelDev& B = levels_[nl - 1];
    k_mg_coarse_solve<<<1, 1024, coarse_smem_, s>>>(B, nl == 1 ? r : nullptr, st, mode);
    launches += 1;
    // Prolongation and post-smoothing (black then red, twice) back up.
    for (int l = nl - 2; l >= 0; --l) {
        const MgLevelDev& L = levels_[l];
        const MgLevelDev& C = levels_[l + 1];
        const int pb = mg_blocks(pairs(L));
        if (l == 0) {
            k_mg_prolong_black<true><<<pb, MG_THREADS, 0, s>>>(L, C, r, st, mode);
            k_mg_smooth<true><<<pb, MG_THREADS, 0, s>>>(L, r, 0, 0, st, mode);
            k_mg_smooth<true><<<pb, MG_THREADS, 0, s>>>(L, r, 1, 0, st, mode);
            k_mg_smooth<true><<<pb, MG_THREADS, 0, s>>>(L, r, 0, 0, st, mode);
        } else {
            k_mg_prolong_black<false><<<pb, MG_THREADS, 0, s>>>(L, C, r, st, mode);
            k_mg_smooth<false><<<pb, MG_THREADS, 0, s>>>(L, r, 0, 0, st, mode);
            k_mg_smooth<false><<<pb, MG_THREADS, 0, s>>>(L, r, 1, 0, st, mode);
            k_mg_smooth<false><<<pb, MG_THREADS, 0, s>>>(L, r, 0, 0, st, mode);
        }
        launches += 4;
    }
    return launches;
}

}  // namespace rb200
