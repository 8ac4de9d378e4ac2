// FP32 geometric multigrid V(2,2) with an FP64 coarsest-grid solve; the
// preconditioner of the mixed-precision pressure method (see mg.hpp).
#include <algorithm>
#include <cmath>
#include <utility>
#include <vector>

#include "mg.hpp"
#include "pcg.hpp"
#include "slab.cuh"
#include "solve_state.cuh"

namespace rb200 {

constexpr int MG_THREADS = 256;
constexpr int MG_LOWER_THREADS = 1024;

__device__ __forceinline__ bool mg_gate(const SolveState* st, int mode) { return gate(st->flags, mode); }

// Kernels of the V-cycle are launched with programmatic stream serialisation:
// one may start while the kernel before it drains, and waits here, before its
// first memory access, until that kernel has completed and its writes are
// visible (a no-op for a launch without the attribute).
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }

__device__ __forceinline__ int mask_of(const int n[3], int i, int j, int k) {
    return int(i > 0) | (int(i + 1 < n[0]) << 1) | (int(j > 0) << 2) | (int(j + 1 < n[1]) << 3) |
           (int(k > 0) << 4) | (int(k + 1 < n[2]) << 5);
}

__host__ __device__ __forceinline__ long mg_pairs(const MgLevelDev& L) {
    return long((L.n[0] + 1) >> 1) * L.n[1] * L.n[2];
}

// Work mapping of the level loops: the rows (j, k) of a level are dealt to
// warps (row = j + n1*k), and a warp's lanes take the pair index m of the row;
// pair m holds cells 2m and 2m+1, of which the one of colour `color` has
// i = 2m + ((color + j + k) & 1) (i may be n0 for an odd row length).
struct Warps {
    int w0, nw, lane;
};
__device__ __forceinline__ Warps grid_warps() {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    return Warps{t >> 5, int((gridDim.x * blockDim.x) >> 5), int(threadIdx.x & 31)};
}

// Rows with fewer than 32 work items share a warp: the warp splits into
// groups of `lanes` lanes (the largest power of two not above the items per
// row), one row per group.
__host__ __device__ __forceinline__ int lanes_for(int per) {
    int lanes = 32;
    while (lanes > 1 && lanes > per) lanes >>= 1;
    return lanes;
}
struct RowSplit {
    int first, step, lane, lanes;
};
__device__ __forceinline__ RowSplit split_rows(const Warps& W, int per) {
    const int lanes = lanes_for(per), rpw = 32 / lanes;
    return RowSplit{W.w0 * rpw + W.lane / lanes, W.nw * rpw, W.lane % lanes, lanes};
}
// Work items per row of the level loops (quads of 4 cells, or red-black pairs).
__host__ __device__ __forceinline__ int sweep_items(const MgLevelDev& L) {
    return (L.n[0] & 3) == 0 ? (L.n[0] >> 2) : ((L.n[0] + 1) >> 1);
}
__host__ __device__ __forceinline__ int restrict_items(const MgLevelDev& L, const MgLevelDev& C) {
    return ((L.n[0] & 3) == 0 && L.cf[0] == 2) ? (C.n[0] >> 1) : C.n[0];
}

// Loads of level data: through L1 in the grid kernels, from L2 in the cluster
// kernel (its CTAs exchange level data through global memory between
// cluster barriers).
template <bool CG>
__device__ __forceinline__ float ldv(const float* p) {
    if (CG) return __ldcg(p);
    return *p;
}

// Gauss-Seidel value x = (b + sum_nb w x_nb) / D, summed x-, x+, y-, y+, z-, z+.
template <bool CG>
__device__ __forceinline__ float gs_value(const MgLevelDev& L, float b, int i, int j, int k, int c) {
    const int sy = L.n[0], sz = L.n[0] * L.n[1];
    const float* __restrict__ x = L.x;
    float s = b;
    if (i > 0) s += L.w[0] * ldv<CG>(x + c - 1);
    if (i + 1 < L.n[0]) s += L.w[0] * ldv<CG>(x + c + 1);
    if (j > 0) s += L.w[1] * ldv<CG>(x + c - sy);
    if (j + 1 < L.n[1]) s += L.w[1] * ldv<CG>(x + c + sy);
    if (k > 0) s += L.w[2] * ldv<CG>(x + c - sz);
    if (k + 1 < L.n[2]) s += L.w[2] * ldv<CG>(x + c + sz);
    return s * L.dinv[mask_of(L.n, i, j, k)];
}

template <bool CG>
__device__ __forceinline__ float4 ld4(const float* p) {
    if (CG) return __ldcg(reinterpret_cast<const float4*>(p));
    return *reinterpret_cast<const float4*>(p);
}
__device__ __forceinline__ float f4get(const float4& v, int e) {
    return e == 0 ? v.x : (e == 1 ? v.y : (e == 2 ? v.z : v.w));
}
__device__ __forceinline__ void f4put(float4& v, int e, float a) {
    if (e == 0) v.x = a;
    else if (e == 1) v.y = a;
    else if (e == 2) v.z = a;
    else v.w = a;
}

// The half-sweep of smooth_rows for rows whose length is a multiple of 4: a
// lane takes 4 consecutive cells (two of each colour) with 16-byte loads of
// the cell row and of its y and z neighbour rows, updates the two cells of
// colour `color` in the same order of operations as gs_value, and stores the
// 4 cells back (the other colour unchanged: nobody writes it in this sweep).
template <bool CG>
__device__ __forceinline__ void smooth_rows_v4(const MgLevelDev& L, const double* __restrict__ r0, int color,
                                               bool first, const Warps& W) {
    const int n0 = L.n[0], quads = n0 >> 2;
    const int rows = L.n[1] * L.n[2];
    const int sy = n0, sz = n0 * L.n[1];
    const RowSplit S = split_rows(W, quads);
    for (int row = S.first; row < rows; row += S.step) {
        const int j = row % L.n[1], k = row / L.n[1];
        const int base = n0 * row;
        const int par = (color + j + k) & 1;
        const int myz = (int(j > 0) << 2) | (int(j + 1 < L.n[1]) << 3) | (int(k > 0) << 4) |
                        (int(k + 1 < L.n[2]) << 5);
        for (int q = S.lane; q < quads; q += S.lanes) {
            const int i0 = 4 * q;
            const int c0 = base + i0;
            float4 bq;
            if (r0) {
                const double2 lo = *reinterpret_cast<const double2*>(r0 + c0);
                const double2 hi = *reinterpret_cast<const double2*>(r0 + c0 + 2);
                bq = make_float4(float(lo.x), float(lo.y), float(hi.x), float(hi.y));
                *reinterpret_cast<float4*>(L.b + c0) = bq;
            } else {
                bq = ld4<CG>(L.b + c0);
            }
            float4 out;
            if (first) {
                out = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
#pragma unroll
                for (int t = 0; t < 2; ++t) {
                    const int e = par + 2 * t;
                    const int i = i0 + e;
                    const int mask = int(i > 0) | (int(i + 1 < n0) << 1) | myz;
                    f4put(out, e, f4get(bq, e) * L.dinv[mask]);
                }
            } else {
                const float4 xc = ld4<CG>(L.x + c0);
                const float xl = (i0 > 0) ? ldv<CG>(L.x + c0 - 1) : 0.0f;
                const float xr = (i0 + 4 < n0) ? ldv<CG>(L.x + c0 + 4) : 0.0f;
                const float4 z4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                const float4 ym = (myz & 4) ? ld4<CG>(L.x + c0 - sy) : z4;
                const float4 yp = (myz & 8) ? ld4<CG>(L.x + c0 + sy) : z4;
                const float4 zm = (myz & 16) ? ld4<CG>(L.x + c0 - sz) : z4;
                const float4 zp = (myz & 32) ? ld4<CG>(L.x + c0 + sz) : z4;
                out = xc;
#pragma unroll
                for (int t = 0; t < 2; ++t) {
                    const int e = par + 2 * t;
                    const int i = i0 + e;
                    float s = f4get(bq, e);
                    if (i > 0) s += L.w[0] * (e == 0 ? xl : f4get(xc, e - 1));
                    if (i + 1 < n0) s += L.w[0] * (e == 3 ? xr : f4get(xc, e + 1));
                    if (myz & 4) s += L.w[1] * f4get(ym, e);
                    if (myz & 8) s += L.w[1] * f4get(yp, e);
                    if (myz & 16) s += L.w[2] * f4get(zm, e);
                    if (myz & 32) s += L.w[2] * f4get(zp, e);
                    const int mask = int(i > 0) | (int(i + 1 < n0) << 1) | myz;
                    f4put(out, e, s * L.dinv[mask]);
                }
            }
            *reinterpret_cast<float4*>(L.x + c0) = out;
        }
    }
}

// Half-sweep of colour `color` over the level. With `first` the correction
// starts from zero (red = b/D, black cleared); with r0 the FP32 right-hand
// side of the finest level is converted from the FP64 residual on the way
// (both cells of the pair).
template <bool CG>
__device__ __forceinline__ void smooth_rows(const MgLevelDev& L, const double* __restrict__ r0, int color, bool first,
                                            const Warps& W) {
    if ((L.n[0] & 3) == 0) {
        smooth_rows_v4<CG>(L, r0, color, first, W);
        return;
    }
    const int hx = (L.n[0] + 1) >> 1;
    const int rows = L.n[1] * L.n[2];
    const RowSplit S = split_rows(W, hx);
    for (int row = S.first; row < rows; row += S.step) {
        const int j = row % L.n[1], k = row / L.n[1];
        const int base = L.n[0] * row;
        const int par = (color + j + k) & 1;
        for (int m = S.lane; m < hx; m += S.lanes) {
            const int i = 2 * m + par;
            const int io = i ^ 1;
            if (first && io < L.n[0]) {
                if (r0) L.b[io + base] = float(r0[io + base]);
                L.x[io + base] = 0.0f;
            }
            if (i >= L.n[0]) continue;
            const int c = i + base;
            float b;
            if (r0) {
                b = float(r0[c]);
                L.b[c] = b;
            } else {
                b = ldv<CG>(L.b + c);
            }
            L.x[c] = first ? b * L.dinv[mask_of(L.n, i, j, k)] : gs_value<CG>(L, b, i, j, k, c);
        }
    }
}

// restrict_rows for fine rows whose length is a multiple of 4 (halved along
// x): a lane takes two coarse cells, i.e. 4 fine cells of each child row, with
// 16-byte loads; the sums run in the same order as restrict_rows.
template <bool CG>
__device__ __forceinline__ void restrict_rows_v4(const MgLevelDev& L, const MgLevelDev& C, const Warps& W) {
    const int n0 = L.n[0], sy = n0, sz = n0 * L.n[1];
    const int rows = C.n[1] * C.n[2];
    const int cpairs = C.n[0] >> 1;
    const float4 z4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const RowSplit S = split_rows(W, cpairs);
    for (int row = S.first; row < rows; row += S.step) {
        const int J = row % C.n[1], K = row / C.n[1];
        for (int P = S.lane; P < cpairs; P += S.lanes) {
            const int i0 = 4 * P;
            float sum[2] = {0.0f, 0.0f};
            for (int dk = 0; dk < L.cf[2]; ++dk)
                for (int dj = 0; dj < L.cf[1]; ++dj) {
                    const int j = J * L.cf[1] + dj, k = K * L.cf[2] + dk;
                    if (j >= L.n[1] || k >= L.n[2]) continue;
                    const int c0 = i0 + n0 * (j + L.n[1] * k);
                    const float4 xc = ld4<CG>(L.x + c0);
                    const float4 bq = ld4<CG>(L.b + c0);
                    const float xl = i0 > 0 ? ldv<CG>(L.x + c0 - 1) : 0.0f;
                    const float xr = i0 + 4 < n0 ? ldv<CG>(L.x + c0 + 4) : 0.0f;
                    const float4 ym = j > 0 ? ld4<CG>(L.x + c0 - sy) : z4;
                    const float4 yp = j + 1 < L.n[1] ? ld4<CG>(L.x + c0 + sy) : z4;
                    const float4 zm = k > 0 ? ld4<CG>(L.x + c0 - sz) : z4;
                    const float4 zp = k + 1 < L.n[2] ? ld4<CG>(L.x + c0 + sz) : z4;
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        const int i = i0 + e;
                        const float x0 = f4get(xc, e);
                        float kx = 0.0f;
                        if (i > 0) kx += L.w[0] * (x0 - (e == 0 ? xl : f4get(xc, e - 1)));
                        if (i + 1 < n0) kx += L.w[0] * (x0 - (e == 3 ? xr : f4get(xc, e + 1)));
                        if (j > 0) kx += L.w[1] * (x0 - f4get(ym, e));
                        if (j + 1 < L.n[1]) kx += L.w[1] * (x0 - f4get(yp, e));
                        if (k > 0) kx += L.w[2] * (x0 - f4get(zm, e));
                        if (k + 1 < L.n[2]) kx += L.w[2] * (x0 - f4get(zp, e));
                        sum[e >> 1] += f4get(bq, e) - kx;
                    }
                }
            *reinterpret_cast<float2*>(C.b + 2 * P + C.n[0] * row) = make_float2(sum[0], sum[1]);
        }
    }
}

// Residual b - K x on the fine cells summed over each coarse cell's children
// (restriction = transpose of the piecewise-constant prolongation). Warps
// take coarse rows, lanes coarse cells along x.
template <bool CG>
__device__ __forceinline__ void restrict_rows(const MgLevelDev& L, const MgLevelDev& C, const Warps& W) {
    if ((L.n[0] & 3) == 0 && L.cf[0] == 2) {
        restrict_rows_v4<CG>(L, C, W);
        return;
    }
    const int sy = L.n[0], sz = L.n[0] * L.n[1];
    const int rows = C.n[1] * C.n[2];
    const RowSplit S = split_rows(W, C.n[0]);
    for (int row = S.first; row < rows; row += S.step) {
        const int J = row % C.n[1], K = row / C.n[1];
        for (int I = S.lane; I < C.n[0]; I += S.lanes) {
            float sum = 0.0f;
            for (int dk = 0; dk < L.cf[2]; ++dk)
                for (int dj = 0; dj < L.cf[1]; ++dj)
                    for (int di = 0; di < L.cf[0]; ++di) {
                        const int i = I * L.cf[0] + di, j = J * L.cf[1] + dj, k = K * L.cf[2] + dk;
                        if (i >= L.n[0] || j >= L.n[1] || k >= L.n[2]) continue;
                        const int c = i + L.n[0] * (j + L.n[1] * k);
                        const float xc = ldv<CG>(L.x + c);
                        float kx = 0.0f;
                        if (i > 0) kx += L.w[0] * (xc - ldv<CG>(L.x + c - 1));
                        if (i + 1 < L.n[0]) kx += L.w[0] * (xc - ldv<CG>(L.x + c + 1));
                        if (j > 0) kx += L.w[1] * (xc - ldv<CG>(L.x + c - sy));
                        if (j + 1 < L.n[1]) kx += L.w[1] * (xc - ldv<CG>(L.x + c + sy));
                        if (k > 0) kx += L.w[2] * (xc - ldv<CG>(L.x + c - sz));
                        if (k + 1 < L.n[2]) kx += L.w[2] * (xc - ldv<CG>(L.x + c + sz));
                        sum += ldv<CG>(L.b + c) - kx;
                    }
            C.b[I + C.n[0] * row] = sum;
        }
    }
}

template <bool CG>
__device__ __forceinline__ float coarse_at(const MgLevelDev& L, const MgLevelDev& C, int i, int j, int k) {
    return ldv<CG>(C.x + ((i >> (L.cf[0] - 1)) + C.n[0] * ((j >> (L.cf[1] - 1)) + C.n[1] * (k >> (L.cf[2] - 1)))));
}

// Prolongation fused with the first post-smoothing half-sweep (black): black
// cells are relaxed against their red neighbours' corrected values x + P xc,
// formed on the fly. Red cells are not written: the red half-sweep that
// follows replaces every red value without reading it. Nothing this pass reads
// is written by it.
// prolong_black_rows for rows whose length is a multiple of 4, with 16-byte
// loads and stores of the fine rows (the red cells are stored back unchanged:
// the red half-sweep that follows replaces them without reading them).
template <bool CG>
__device__ __forceinline__ void prolong_black_rows_v4(const MgLevelDev& L, const MgLevelDev& C, const Warps& W) {
    const int n0 = L.n[0], quads = n0 >> 2;
    const int rows = L.n[1] * L.n[2];
    const int sy = n0, sz = n0 * L.n[1];
    const float4 z4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const RowSplit S = split_rows(W, quads);
    for (int row = S.first; row < rows; row += S.step) {
        const int j = row % L.n[1], k = row / L.n[1];
        const int base = n0 * row;
        const int par = (1 + j + k) & 1;
        const int myz = (int(j > 0) << 2) | (int(j + 1 < L.n[1]) << 3) | (int(k > 0) << 4) |
                        (int(k + 1 < L.n[2]) << 5);
        for (int q = S.lane; q < quads; q += S.lanes) {
            const int i0 = 4 * q;
            const int c0 = base + i0;
            const float4 bq = ld4<CG>(L.b + c0);
            const float4 xc = ld4<CG>(L.x + c0);
            const float xl = (i0 > 0) ? ldv<CG>(L.x + c0 - 1) : 0.0f;
            const float xr = (i0 + 4 < n0) ? ldv<CG>(L.x + c0 + 4) : 0.0f;
            const float4 ym = (myz & 4) ? ld4<CG>(L.x + c0 - sy) : z4;
            const float4 yp = (myz & 8) ? ld4<CG>(L.x + c0 + sy) : z4;
            const float4 zm = (myz & 16) ? ld4<CG>(L.x + c0 - sz) : z4;
            const float4 zp = (myz & 32) ? ld4<CG>(L.x + c0 + sz) : z4;
            float4 out = xc;
#pragma unroll
            for (int t = 0; t < 2; ++t) {
                const int e = par + 2 * t;
                const int i = i0 + e;
                float s = f4get(bq, e);
                if (i > 0) s += L.w[0] * ((e == 0 ? xl : f4get(xc, e - 1)) + coarse_at<CG>(L, C, i - 1, j, k));
                if (i + 1 < n0) s += L.w[0] * ((e == 3 ? xr : f4get(xc, e + 1)) + coarse_at<CG>(L, C, i + 1, j, k));
                if (myz & 4) s += L.w[1] * (f4get(ym, e) + coarse_at<CG>(L, C, i, j - 1, k));
                if (myz & 8) s += L.w[1] * (f4get(yp, e) + coarse_at<CG>(L, C, i, j + 1, k));
                if (myz & 16) s += L.w[2] * (f4get(zm, e) + coarse_at<CG>(L, C, i, j, k - 1));
                if (myz & 32) s += L.w[2] * (f4get(zp, e) + coarse_at<CG>(L, C, i, j, k + 1));
                const int mask = int(i > 0) | (int(i + 1 < n0) << 1) | myz;
                f4put(out, e, s * L.dinv[mask]);
            }
            *reinterpret_cast<float4*>(L.x + c0) = out;
        }
    }
}

template <bool CG>
__device__ __forceinline__ void prolong_black_rows(const MgLevelDev& L, const MgLevelDev& C, const Warps& W) {
    if ((L.n[0] & 3) == 0) {
        prolong_black_rows_v4<CG>(L, C, W);
        return;
    }
    const int hx = (L.n[0] + 1) >> 1;
    const int rows = L.n[1] * L.n[2];
    const int sy = L.n[0], sz = L.n[0] * L.n[1];
    const RowSplit S = split_rows(W, hx);
    for (int row = S.first; row < rows; row += S.step) {
        const int j = row % L.n[1], k = row / L.n[1];
        const int base = L.n[0] * row;
        const int par = (1 + j + k) & 1;
        for (int m = S.lane; m < hx; m += S.lanes) {
            const int i = 2 * m + par;
            if (i >= L.n[0]) continue;
            const int c = i + base;
            float s = ldv<CG>(L.b + c);
            if (i > 0) s += L.w[0] * (ldv<CG>(L.x + c - 1) + coarse_at<CG>(L, C, i - 1, j, k));
            if (i + 1 < L.n[0]) s += L.w[0] * (ldv<CG>(L.x + c + 1) + coarse_at<CG>(L, C, i + 1, j, k));
            if (j > 0) s += L.w[1] * (ldv<CG>(L.x + c - sy) + coarse_at<CG>(L, C, i, j - 1, k));
            if (j + 1 < L.n[1]) s += L.w[1] * (ldv<CG>(L.x + c + sy) + coarse_at<CG>(L, C, i, j + 1, k));
            if (k > 0) s += L.w[2] * (ldv<CG>(L.x + c - sz) + coarse_at<CG>(L, C, i, j, k - 1));
            if (k + 1 < L.n[2]) s += L.w[2] * (ldv<CG>(L.x + c + sz) + coarse_at<CG>(L, C, i, j, k + 1));
            L.x[c] = s * L.dinv[mask_of(L.n, i, j, k)];
        }
    }
}

// ------------------------------------------------------------ grid kernels (large levels)
__global__ void __launch_bounds__(MG_THREADS) k_mg_smooth(MgLevelDev L, const double* __restrict__ r0, int color,
                                                          int first, const SolveState* st, int mode) {
    pdl_wait();
    if (!mg_gate(st, mode)) return;
    smooth_rows<false>(L, r0, color, first != 0, grid_warps());
}

// Two half-sweeps in one pass (colour c1, then the other colour) over a level
// whose rows are a multiple of 4 long, one tile of PJ x PK rows (j, k) at full
// row length: colour c1 is relaxed on the tile and the rows around it (one
// row of halo in j and k) from the input x into shared memory, exactly as
// smooth_rows_v4 does, then the other colour on the tile from those rows, and
// both colours are stored to x_out. The input x is only read and x_out only
// written, so tiles never see each other's partial results, and the values
// equal two consecutive half-sweeps bit for bit (the same operands in the same
// order). With `first` the correction starts from zero. Every thread of the
// block calls it; srow holds (PJ + 2) (PK + 2) rows.
template <bool CG, int PJ, int PK>
__device__ __forceinline__ void pair_tile(const MgLevelDev& L, float* __restrict__ x_out, int c1, bool first, int j0,
                                          int k0, float4* srow) {
    constexpr int ROWS = (PJ + 2) * (PK + 2);
    const int n0 = L.n[0], quads = n0 >> 2, n1 = L.n[1], n2 = L.n[2];
    const int sy = n0, sz = n0 * n1;
    const float4 z4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const float* __restrict__ x = L.x;
    for (int it = threadIdx.x; it < ROWS * quads; it += blockDim.x) {
        const int q = it % quads, hr = it / quads;
        const int j = j0 - 1 + hr % (PJ + 2), k = k0 - 1 + hr / (PJ + 2);
        if (j < 0 || j >= n1 || k < 0 || k >= n2) continue;
        const int i0 = 4 * q;
        const int c0 = i0 + n0 * (j + n1 * k);
        const int par = (c1 + j + k) & 1;
        const int myz = (int(j > 0) << 2) | (int(j + 1 < n1) << 3) | (int(k > 0) << 4) | (int(k + 1 < n2) << 5);
        const float4 bq = ld4<CG>(L.b + c0);
        float4 out;
        if (first) {
            out = z4;
#pragma unroll
            for (int t = 0; t < 2; ++t) {
                const int e = par + 2 * t;
                const int i = i0 + e;
                f4put(out, e, f4get(bq, e) * L.dinv[int(i > 0) | (int(i + 1 < n0) << 1) | myz]);
            }
        } else {
            const float4 xc = ld4<CG>(x + c0);
            const float xl = i0 > 0 ? ldv<CG>(x + c0 - 1) : 0.0f;
            const float xr = i0 + 4 < n0 ? ldv<CG>(x + c0 + 4) : 0.0f;
            const float4 ym = (myz & 4) ? ld4<CG>(x + c0 - sy) : z4;
            const float4 yp = (myz & 8) ? ld4<CG>(x + c0 + sy) : z4;
            const float4 zm = (myz & 16) ? ld4<CG>(x + c0 - sz) : z4;
            const float4 zp = (myz & 32) ? ld4<CG>(x + c0 + sz) : z4;
            out = xc;
#pragma unroll
            for (int t = 0; t < 2; ++t) {
                const int e = par + 2 * t;
                const int i = i0 + e;
                float sum = f4get(bq, e);
                if (i > 0) sum += L.w[0] * (e == 0 ? xl : f4get(xc, e - 1));
                if (i + 1 < n0) sum += L.w[0] * (e == 3 ? xr : f4get(xc, e + 1));
                if (myz & 4) sum += L.w[1] * f4get(ym, e);
                if (myz & 8) sum += L.w[1] * f4get(yp, e);
                if (myz & 16) sum += L.w[2] * f4get(zm, e);
                if (myz & 32) sum += L.w[2] * f4get(zp, e);
                f4put(out, e, sum * L.dinv[int(i > 0) | (int(i + 1 < n0) << 1) | myz]);
            }
        }
        srow[hr * quads + q] = out;
    }
    __syncthreads();
    const float* __restrict__ sf = reinterpret_cast<const float*>(srow);
    for (int it = threadIdx.x; it < PJ * PK * quads; it += blockDim.x) {
        const int q = it % quads, tr = it / quads;
        const int j = j0 + tr % PJ, k = k0 + tr / PJ;
        if (j >= n1 || k >= n2) continue;
        const int hr = (tr % PJ + 1) + (PJ + 2) * (tr / PJ + 1);
        const int i0 = 4 * q;
        const int c0 = i0 + n0 * (j + n1 * k);
        const int par = (c1 + 1 + j + k) & 1;
        const int myz = (int(j > 0) << 2) | (int(j + 1 < n1) << 3) | (int(k > 0) << 4) | (int(k + 1 < n2) << 5);
        const float4 bq = ld4<CG>(L.b + c0);
        const float4 xc = srow[hr * quads + q];
        const float xl = i0 > 0 ? sf[hr * n0 + i0 - 1] : 0.0f;
        const float xr = i0 + 4 < n0 ? sf[hr * n0 + i0 + 4] : 0.0f;
        const float4 ym = (myz & 4) ? srow[(hr - 1) * quads + q] : z4;
        const float4 yp = (myz & 8) ? srow[(hr + 1) * quads + q] : z4;
        const float4 zm = (myz & 16) ? srow[(hr - (PJ + 2)) * quads + q] : z4;
        const float4 zp = (myz & 32) ? srow[(hr + (PJ + 2)) * quads + q] : z4;
        float4 out = xc;
#pragma unroll
        for (int t = 0; t < 2; ++t) {
            const int e = par + 2 * t;
            const int i = i0 + e;
            float sum = f4get(bq, e);
            if (i > 0) sum += L.w[0] * (e == 0 ? xl : f4get(xc, e - 1));
            if (i + 1 < n0) sum += L.w[0] * (e == 3 ? xr : f4get(xc, e + 1));
            if (myz & 4) sum += L.w[1] * f4get(ym, e);
            if (myz & 8) sum += L.w[1] * f4get(yp, e);
            if (myz & 16) sum += L.w[2] * f4get(zm, e);
            if (myz & 32) sum += L.w[2] * f4get(zp, e);
            f4put(out, e, sum * L.dinv[int(i > 0) | (int(i + 1 < n0) << 1) | myz]);
        }
        *reinterpret_cast<float4*>(x_out + c0) = out;
    }
    __syncthreads();  // srow is free for the block's next tile
}

// Grid kernel of the pairs: one 4 x 4-row tile per block.
constexpr int PJ = 4, PK = 4;
constexpr int PAIR_ROWS = (PJ + 2) * (PK + 2);
constexpr size_t kPairSmemMax = 200 * 1024;

__global__ void __launch_bounds__(MG_THREADS) k_mg_smooth_pair(MgLevelDev L, float* __restrict__ x_out, int c1,
                                                               int first, const SolveState* st, int mode) {
    pdl_wait();
    extern __shared__ float4 srow[];  // PAIR_ROWS rows of n0/4 quads
    if (!mg_gate(st, mode)) return;
    const int tj = (L.n[1] + PJ - 1) / PJ;
    pair_tile<false, PJ, PK>(L, x_out, c1, first != 0, int(blockIdx.x % unsigned(tj)) * PJ,
                             int(blockIdx.x / unsigned(tj)) * PK, srow);
}

// Pairs in the cluster kernel: 8 x 8-row tiles dealt over the cluster's CTAs,
// for levels whose rows are a multiple of 4 and at most LPAIR_N0 long.
constexpr int LPJ = 8, LPK = 8;
constexpr int LPAIR_N0 = 32;

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

// ------------------------------------------------------------ lower levels (one cluster)
__device__ __forceinline__ void cluster_sync_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
    asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}
__device__ __forceinline__ unsigned cluster_rank() {
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;\n" : "=r"(r));
    return r;
}
__device__ __forceinline__ unsigned cluster_size() {
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_nctarank;\n" : "=r"(r));
    return r;
}

// A fused pair on a level of the cluster kernel: the tiles are dealt over the
// cluster's CTAs, which then meet at the cluster barrier.
__device__ __forceinline__ void cluster_pair(const MgLevelDev& L, float* out, int c1, bool first, unsigned rank,
                                             unsigned nct, float4* prow) {
    const int tj = (L.n[1] + LPJ - 1) / LPJ, tiles = tj * ((L.n[2] + LPK - 1) / LPK);
    for (int t = int(rank); t < tiles; t += int(nct))
        pair_tile<true, LPJ, LPK>(L, out, c1, first, (t % tj) * LPJ, (t / tj) * LPK, prow);
    cluster_sync_all();
}

// The whole V-cycle below the grid-kernel levels in one thread-block cluster:
// the CTAs split every half-sweep, restriction and prolongation, and meet at
// hardware cluster barriers (release/acquire) instead of kernel boundaries.
// Level data moves through L2. The coarsest level is solved densely in FP64
// (x = G b, one warp per row). r0 is the FP64 residual when the first level
// here is the finest level; skip_last_red leaves that level's final red
// half-sweep to the finish kernel.
__global__ void __launch_bounds__(MG_LOWER_THREADS, 1) k_mg_lower(MgLower P, const double* __restrict__ r0,
                                                               const double* __restrict__ G,
                                                               const SolveState* st, int mode, int skip_last_red) {
    pdl_wait();
    __shared__ double bs[512];
    __shared__ float4 prow[(LPJ + 2) * (LPK + 2) * LPAIR_N0 / 4];
    if (!mg_gate(st, mode)) return;  // uniform: every CTA reads the same flags
    const unsigned rank = cluster_rank(), nct = cluster_size();
    const Warps W{int((rank * blockDim.x + threadIdx.x) >> 5), int((nct * blockDim.x) >> 5), int(threadIdx.x & 31)};
    const int last = P.count - 1;
    unsigned second = 0;  // bit l: level l's correction is in its second buffer
    for (int l = 0; l < last; ++l) {
        const MgLevelDev& L = P.lv[0][l];
        if (P.paired[l]) {
            const MgLevelDev& La = P.lv[1][l];
            if (l == 0 && r0) {
                // the finest level: red converts the residual, then (black,
                // red) into the second buffer and black there
                smooth_rows<true>(L, r0, 0, true, W);
                cluster_sync_all();
                cluster_pair(L, La.x, 1, false, rank, nct, prow);
                smooth_rows<true>(La, nullptr, 1, false, W);
                cluster_sync_all();
                restrict_rows<true>(La, P.lv[0][l + 1], W);
                second |= 1u << l;
            } else {
                cluster_pair(L, La.x, 0, true, rank, nct, prow);
                cluster_pair(La, L.x, 0, false, rank, nct, prow);
                restrict_rows<true>(L, P.lv[0][l + 1], W);
            }
        } else {
            for (int sweep = 0; sweep < 2; ++sweep) {
                smooth_rows<true>(L, (l == 0 && sweep == 0) ? r0 : nullptr, 0, sweep == 0, W);
                cluster_sync_all();
                smooth_rows<true>(L, nullptr, 1, false, W);
                cluster_sync_all();
            }
            restrict_rows<true>(L, P.lv[0][l + 1], W);
        }
        cluster_sync_all();
    }
    {
        const MgLevelDev& C = P.lv[0][last];
        const int M = C.cells;
        const double* src = last == 0 ? r0 : nullptr;
        for (int c = threadIdx.x; c < M; c += blockDim.x) bs[c] = src ? src[c] : double(__ldcg(C.b + c));
        __syncthreads();
        const int lane = threadIdx.x & 31, warps = blockDim.x >> 5;
        for (int row = int(rank) * warps + (threadIdx.x >> 5); row < M; row += int(nct) * warps) {
            const double* g = G + size_t(row) * M;
            double acc = 0.0;
            for (int c = lane; c < M; c += 32) acc += __ldcg(g + c) * bs[c];
            for (int m = 16; m >= 1; m >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, m);
            if (lane == 0) C.x[row] = float(acc);
        }
        cluster_sync_all();
    }
    for (int l = last - 1; l >= 0; --l) {
        const int in = (second >> l) & 1u;
        const MgLevelDev& L = P.lv[in][l];
        prolong_black_rows<true>(L, P.lv[(second >> (l + 1)) & 1u][l + 1], W);
        cluster_sync_all();
        int now = in;
        if (P.paired[l]) {
            // (red, black) into the other buffer, then red there
            cluster_pair(L, P.lv[in ^ 1][l].x, 0, false, rank, nct, prow);
            second ^= 1u << l;
            now = in ^ 1;
        } else {
            smooth_rows<true>(L, nullptr, 0, false, W);
            cluster_sync_all();
            smooth_rows<true>(L, nullptr, 1, false, W);
            cluster_sync_all();
        }
        if (!(l == 0 && skip_last_red)) {
            smooth_rows<true>(P.lv[now][l], nullptr, 0, false, W);
            cluster_sync_all();
        }
    }
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
        if ((L.n[0] & 3) != 0 || smem > kPairSmemMax) continue;
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

// ------------------------------------------------------------ finish
// The finest level's last red half-sweep fused with the outer method's
// preconditioner output: z = x (FP64, z[0] = 0 for the eliminated gauge row),
// r.z and z.q reduced and the flexible-CG decision taken. Without a hierarchy
// (a single level solved densely) z is copied from x.
__global__ void __launch_bounds__(MG_THREADS) k_mg_finish_red(MgLevelDev L, int smooth, SolveState* st,
                                                              const double* __restrict__ r,
                                                              const double* __restrict__ q, int mode, Partials part,
                                                              rb200_trace* trace) {
    pdl_wait();
    __shared__ BlockReduce<2, 0> red;
    if (!gate(st->flags, mode)) return;
    Neu rz, zq;
    const Warps W = grid_warps();
    const int hx = (L.n[0] + 1) >> 1;
    const int rows = L.n[1] * L.n[2];
    if ((L.n[0] & 3) == 0) {
        // quads of 4 cells with 16-byte loads (the same values as the pairs below)
        const int n0 = L.n[0], quads = n0 >> 2, sy = n0, sz = n0 * L.n[1];
        const float4 z4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        for (int rw = W.w0; rw < rows; rw += W.nw) {
            const int j = rw % L.n[1], k = rw / L.n[1];
            const int par = (j + k) & 1;  // the red cells of the quad: par, par + 2
            const int myz = (int(j > 0) << 2) | (int(j + 1 < L.n[1]) << 3) | (int(k > 0) << 4) |
                            (int(k + 1 < L.n[2]) << 5);
            for (int qd = W.lane; qd < quads; qd += 32) {
                const int i0 = 4 * qd;
                const int c0 = n0 * rw + i0;
                const float4 xc = *reinterpret_cast<const float4*>(L.x + c0);
                float4 out = xc;
                if (smooth) {
                    const float4 bq = *reinterpret_cast<const float4*>(L.b + c0);
                    const float xl = i0 > 0 ? L.x[c0 - 1] : 0.0f;
                    const float xr = i0 + 4 < n0 ? L.x[c0 + 4] : 0.0f;
                    const float4 ym = (myz & 4) ? *reinterpret_cast<const float4*>(L.x + c0 - sy) : z4;
                    const float4 yp = (myz & 8) ? *reinterpret_cast<const float4*>(L.x + c0 + sy) : z4;
                    const float4 zm = (myz & 16) ? *reinterpret_cast<const float4*>(L.x + c0 - sz) : z4;
                    const float4 zp = (myz & 32) ? *reinterpret_cast<const float4*>(L.x + c0 + sz) : z4;
#pragma unroll
                    for (int t = 0; t < 2; ++t) {
                        const int e = par + 2 * t;
                        const int i = i0 + e;
                        float sacc = f4get(bq, e);
                        if (i > 0) sacc += L.w[0] * (e == 0 ? xl : f4get(xc, e - 1));
                        if (i + 1 < n0) sacc += L.w[0] * (e == 3 ? xr : f4get(xc, e + 1));
                        if (myz & 4) sacc += L.w[1] * f4get(ym, e);
                        if (myz & 8) sacc += L.w[1] * f4get(yp, e);
                        if (myz & 16) sacc += L.w[2] * f4get(zm, e);
                        if (myz & 32) sacc += L.w[2] * f4get(zp, e);
                        f4put(out, e, sacc * L.dinv[int(i > 0) | (int(i + 1 < n0) << 1) | myz]);
                    }
                    *reinterpret_cast<float4*>(L.x + c0) = out;
                }
                double zc[4];
#pragma unroll
                for (int e = 0; e < 4; ++e) zc[e] = (c0 + e == 0) ? 0.0 : double(f4get(out, e));
                const double2 r01 = *reinterpret_cast<const double2*>(r + c0);
                const double2 r23 = *reinterpret_cast<const double2*>(r + c0 + 2);
                const double rr[4] = {r01.x, r01.y, r23.x, r23.y};
                double qq[4] = {0.0, 0.0, 0.0, 0.0};
                if (mode == MODE_ITER) {
                    const double2 q01 = *reinterpret_cast<const double2*>(q + c0);
                    const double2 q23 = *reinterpret_cast<const double2*>(q + c0 + 2);
                    qq[0] = q01.x;
                    qq[1] = q01.y;
                    qq[2] = q23.x;
                    qq[3] = q23.y;
                }
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    if (c0 + e == 0) continue;
                    rz.add(rr[e] * zc[e]);
                    if (mode == MODE_ITER) zq.add(zc[e] * qq[e]);
                }
            }
        }
    } else
    for (int rw = W.w0; rw < rows; rw += W.nw) {
        const int j = rw % L.n[1], k = rw / L.n[1];
        const int row = L.n[0] * rw;
        const int par = (j + k) & 1;
        for (int m = W.lane; m < hx; m += 32) {
            const int i = 2 * m + par;  // the red cell of the pair
            const int ib = i ^ 1;
            if (ib < L.n[0]) {  // the black cell of the pair: its value is final
                const int c = ib + row;
                const double zc = c == 0 ? 0.0 : double(L.x[c]);
                if (c != 0) {
                    rz.add(r[c] * zc);
                    if (mode == MODE_ITER) zq.add(zc * q[c]);
                }
            }
            if (i < L.n[0]) {
                const int c = i + row;
                float xv = L.x[c];
                if (smooth) {
                    xv = gs_value<false>(L, L.b[c], i, j, k, c);
                    L.x[c] = xv;
                }
                const double zc = c == 0 ? 0.0 : double(xv);
                if (c != 0) {
                    rz.add(r[c] * zc);
                    if (mode == MODE_ITER) zq.add(zc * q[c]);
                }
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

// The flexible-CG direction pass of the mixed method (src/pressure.rs:657-668,
// :720-731): d = z + beta d (d = z after a restart), q = K d stored, d.q and
// the decision for alpha. z is read straight from the V-cycle's FP32 output x
// of the finest level (z = f64(x), z[0] = 0 for the eliminated gauge row), so
// no FP64 copy of z is stored. One warp per cell row, lanes along x.
__global__ void __launch_bounds__(MG_THREADS) k_mg_pass1(GridDev g, MgLevelDev L, SolveState* st, double* d0,
                                                         double* d1, double* __restrict__ q, Partials part,
                                                         rb200_trace* trace, int kc_len) {
    pdl_wait();
    __shared__ BlockReduce<1, 0> red;
    const int flags = st->flags;
    if (flags & F_STOP) return;
    const bool fresh = (flags & F_REPLACED) != 0;
    const double beta = st->beta;
    const int dsel = st->dsel;
    const double* __restrict__ src = dsel ? d1 : d0;
    double* __restrict__ dst = dsel ? d0 : d1;
    const float* __restrict__ x = L.x;
    auto dn = [&](int c) -> double {
        const double zc = c == 0 ? 0.0 : double(x[c]);
        return fresh ? zc : zc + beta * src[c];
    };
    const int sy = g.n[0], sz = g.n[0] * g.n[1];
    Neu acc;
    const Warps W = grid_warps();
    const int rows = g.n[1] * g.n[2];
    if ((g.n[0] & 3) == 0) {
        // quads of 4 cells: x with 16-byte loads, d with two 16-byte loads
        const int n0 = g.n[0], quads = n0 >> 2;
        auto dn4 = [&](int c0, double (&o)[4]) {
            const float4 xv = *reinterpret_cast<const float4*>(x + c0);
            const double zc[4] = {c0 == 0 ? 0.0 : double(xv.x), double(xv.y), double(xv.z), double(xv.w)};
            if (fresh) {
#pragma unroll
                for (int e = 0; e < 4; ++e) o[e] = zc[e];
            } else {
                const double2 a = *reinterpret_cast<const double2*>(src + c0);
                const double2 b2 = *reinterpret_cast<const double2*>(src + c0 + 2);
                o[0] = zc[0] + beta * a.x;
                o[1] = zc[1] + beta * a.y;
                o[2] = zc[2] + beta * b2.x;
                o[3] = zc[3] + beta * b2.y;
            }
        };
        // A warp takes a line of up to 32 quads of row j and marches along z
        // over kc_len rows, keeping the z-neighbour rows in registers: each
        // row of d and x is loaded once for the line plus once per y
        // neighbour row, instead of once per stencil row that reads it.
        const int qsegs = (quads + 31) >> 5;
        const int kcs = (g.n[2] + kc_len - 1) / kc_len;
        const int lines = qsegs * g.n[1] * kcs;
        for (int line = W.w0; line < lines; line += W.nw) {
            const int qseg = line % qsegs, t = line / qsegs;
            const int j = t % g.n[1], k_begin = (t / g.n[1]) * kc_len;
            const int k_end = min(g.n[2], k_begin + kc_len);
            const int qd = qseg * 32 + W.lane;
            if (qd >= quads) continue;
            const int i0 = 4 * qd;
            double prev[4] = {0, 0, 0, 0}, cur[4], next[4];
            const int base0 = n0 * (j + g.n[1] * k_begin) + i0;
            if (k_begin > 0) dn4(base0 - sz, prev);
            dn4(base0, cur);
            for (int k = k_begin; k < k_end; ++k) {
                const int c0 = base0 + (k - k_begin) * sz;
                double ym[4] = {0, 0, 0, 0}, yp[4] = {0, 0, 0, 0};
#pragma unroll
                for (int e = 0; e < 4; ++e) next[e] = 0.0;
                if (k + 1 < g.n[2]) dn4(c0 + sz, next);
                if (j > 0) dn4(c0 - sy, ym);
                if (j + 1 < g.n[1]) dn4(c0 + sy, yp);
                const double xl = i0 > 0 ? dn(c0 - 1) : 0.0;
                const double xr = i0 + 4 < n0 ? dn(c0 + 4) : 0.0;
                double qq[4];
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    Neigh v;
                    v.c = cur[e];
                    v.xm = e == 0 ? xl : cur[e - 1];
                    v.xp = e == 3 ? xr : cur[e + 1];
                    v.ym = ym[e];
                    v.yp = yp[e];
                    v.zm = prev[e];
                    v.zp = next[e];
                    qq[e] = (c0 + e == 0) ? 0.0 : apply_row(g, i0 + e, j, k, v);
                }
                *reinterpret_cast<double2*>(dst + c0) = make_double2(cur[0], cur[1]);
                *reinterpret_cast<double2*>(dst + c0 + 2) = make_double2(cur[2], cur[3]);
                *reinterpret_cast<double2*>(q + c0) = make_double2(qq[0], qq[1]);
                *reinterpret_cast<double2*>(q + c0 + 2) = make_double2(qq[2], qq[3]);
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    acc.add(cur[e] * qq[e]);
                    prev[e] = cur[e];
                    cur[e] = next[e];
                }
            }
        }
    } else
    for (int rw = W.w0; rw < rows; rw += W.nw) {
        const int j = rw % g.n[1], k = rw / g.n[1];
        const int base = g.n[0] * rw;
        for (int i = W.lane; i < g.n[0]; i += 32) {
            const int c = base + i;
            Neigh v;
            v.c = dn(c);
            v.xm = i > 0 ? dn(c - 1) : 0.0;
            v.xp = i + 1 < g.n[0] ? dn(c + 1) : 0.0;
            v.ym = j > 0 ? dn(c - sy) : 0.0;
            v.yp = j + 1 < g.n[1] ? dn(c + sy) : 0.0;
            v.zm = k > 0 ? dn(c - sz) : 0.0;
            v.zp = k + 1 < g.n[2] ? dn(c + sz) : 0.0;
            const double qv = c == 0 ? 0.0 : apply_row(g, i, j, k, v);
            dst[c] = v.c;
            q[c] = qv;
            acc.add(v.c * qv);
        }
    }
    dd sums[1] = {acc.as_dd()};
    double none[1];
    block_reduce<1, 0>(red, sums, none);
    if (publish_and_check_last<1, 0>(part, blockIdx.x, gridDim.x, sums, none)) {
        fold_partials<1, 0>(part, gridDim.x, red, sums, none);
        if (threadIdx.x == 0) decide_pass1(st, trace, dd_value(sums[0]), flags, dsel);
    }
}

// The flexible-CG update (p += alpha d, r -= alpha q, |r|^2 and the candidate
// test) fused with the V-cycle's first half-sweep on the finest level, which
// needs no neighbour: b = f32(r), red x = b / D, black x = 0. Used when the
// finest level is a grid-kernel level.
__global__ void __launch_bounds__(MG_THREADS) k_mg_update_first(GridDev g, MgLevelDev L, SolveState* st,
                                                                double* __restrict__ p, double* __restrict__ r,
                                                                const double* d0, const double* d1,
                                                                const double* __restrict__ q, Partials part,
                                                                rb200_trace* trace) {
    pdl_wait();
    __shared__ BlockReduce<1, 0> red;
    const int flags = st->flags;
    if (flags & F_STOP) return;
    const double alpha = st->alpha;
    const double* __restrict__ d = st->dsel ? d1 : d0;
    Neu acc;
    const Warps W = grid_warps();
    const int n0 = g.n[0], rows = g.n[1] * g.n[2];
    for (int rw = W.w0; rw < rows; rw += W.nw) {
        const int j = rw % g.n[1], k = rw / g.n[1];
        const int base = n0 * rw;
        const int par = (j + k) & 1;  // the red cells of a quad: par, par + 2
        const int myz = (int(j > 0) << 2) | (int(j + 1 < g.n[1]) << 3) | (int(k > 0) << 4) |
                        (int(k + 1 < g.n[2]) << 5);
        if ((n0 & 3) == 0) {
            for (int qd = W.lane; qd < (n0 >> 2); qd += 32) {
                const int i0 = 4 * qd;
                const int c0 = base + i0;
                double pv[4], rv[4], dv[4], qv[4];
                *reinterpret_cast<double2*>(pv) = *reinterpret_cast<const double2*>(p + c0);
                *reinterpret_cast<double2*>(pv + 2) = *reinterpret_cast<const double2*>(p + c0 + 2);
                *reinterpret_cast<double2*>(rv) = *reinterpret_cast<const double2*>(r + c0);
                *reinterpret_cast<double2*>(rv + 2) = *reinterpret_cast<const double2*>(r + c0 + 2);
                *reinterpret_cast<double2*>(dv) = *reinterpret_cast<const double2*>(d + c0);
                *reinterpret_cast<double2*>(dv + 2) = *reinterpret_cast<const double2*>(d + c0 + 2);
                *reinterpret_cast<double2*>(qv) = *reinterpret_cast<const double2*>(q + c0);
                *reinterpret_cast<double2*>(qv + 2) = *reinterpret_cast<const double2*>(q + c0 + 2);
                float4 bq, xq = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    if (c0 + e != 0) {  // the gauge row keeps p[0] = r[0] = 0
                        pv[e] = pv[e] + alpha * dv[e];
                        rv[e] = rv[e] - alpha * qv[e];
                        acc.add(rv[e] * rv[e]);
                    }
                    f4put(bq, e, float(rv[e]));
                }
#pragma unroll
                for (int t = 0; t < 2; ++t) {
                    const int e = par + 2 * t;
                    const int i = i0 + e;
                    f4put(xq, e, f4get(bq, e) * L.dinv[int(i > 0) | (int(i + 1 < n0) << 1) | myz]);
                }
                *reinterpret_cast<double2*>(p + c0) = *reinterpret_cast<double2*>(pv);
                *reinterpret_cast<double2*>(p + c0 + 2) = *reinterpret_cast<double2*>(pv + 2);
                *reinterpret_cast<double2*>(r + c0) = *reinterpret_cast<double2*>(rv);
                *reinterpret_cast<double2*>(r + c0 + 2) = *reinterpret_cast<double2*>(rv + 2);
                *reinterpret_cast<float4*>(L.b + c0) = bq;
                *reinterpret_cast<float4*>(L.x + c0) = xq;
            }
        } else {
            for (int i = W.lane; i < n0; i += 32) {
                const int c = base + i;
                double rc = r[c];
                if (c != 0) {
                    p[c] = p[c] + alpha * d[c];
                    rc = rc - alpha * q[c];
                    r[c] = rc;
                    acc.add(rc * rc);
                }
                const float b = float(rc);
                L.b[c] = b;
                const bool isred = ((i + j + k) & 1) == 0;
                L.x[c] = isred ? b * L.dinv[int(i > 0) | (int(i + 1 < n0) << 1) | myz] : 0.0f;
            }
        }
    }
    dd sums[1] = {acc.as_dd()};
    double none[1];
    block_reduce<1, 0>(red, sums, none);
    if (publish_and_check_last<1, 0>(part, blockIdx.x, gridDim.x, sums, none)) {
        fold_partials<1, 0>(part, gridDim.x, red, sums, none);
        if (threadIdx.x == 0) {
            if (flags & F_PROFILE) return;
            const int it = st->it + 1;
            st->it = it;
            const double recursive_l2 = sqrt(dd_value(sums[0]));
            st->recursive_l2 = recursive_l2;
            if (trace) trace[it - 1].recursive_l2 = recursive_l2;
            if (recursive_l2 <= st->threshold || it == st->max_it) st->flags = flags | F_CANDIDATE;
        }
    }
}

int Multigrid::enqueue_update_first(const GridDev& g, void* state, double* p, double* r, double* d0, double* d1,
                                    const double* q, Partials part, rb200_trace* trace, cudaStream_t s) const {
    int pb = row_blocks(levels_[0]);
    if (pb > 148 * 8) pb = 148 * 8;  // reduction partials capacity
    pdl_launch(k_mg_update_first, dim3(pb), dim3(MG_THREADS), 0, s, g, levels_[0], static_cast<SolveState*>(state), p,
               r, d0, d1, q, part, trace);
    return 1;
}

int Multigrid::enqueue_pass1(const GridDev& g, void* state, double* d0, double* d1, double* q, Partials part,
                             rb200_trace* trace, cudaStream_t s) const {
    int pb = row_blocks(levels_[0]);
    if (pb > 148 * 8) pb = 148 * 8;  // reduction partials capacity
    // the z-march length of the quad path: long where there are enough lines
    // for every warp of the grid, short otherwise
    const int quads = g.n[0] / 4, qsegs = (quads + 31) / 32;
    const int warps = pb * (MG_THREADS / 32);
    int kc_len = 16;
    while (kc_len > 2 && qsegs * g.n[1] * ((g.n[2] + kc_len - 1) / kc_len) < warps) kc_len /= 2;
    pdl_launch(k_mg_pass1, dim3(pb), dim3(MG_THREADS), 0, s, g, levels_[0], static_cast<SolveState*>(state), d0, d1, q,
               part, trace, kc_len);
    return 1;
}

int Multigrid::enqueue_finish(void* state, const double* r, const double* q, int mode, Partials part,
                              rb200_trace* trace, cudaStream_t s) const {
    const MgLevelDev& L = levels_[0];
    int pb = row_blocks(L);
    if (pb > 148 * 8) pb = 148 * 8;  // reduction partials capacity
    pdl_launch(k_mg_finish_red, dim3(pb), dim3(MG_THREADS), 0, s, L, levels_.size() > 1 ? 1 : 0,
               static_cast<SolveState*>(state), r, q, mode, part, trace);
    return 1;
}

}  // namespace rb200
