// Device bodies of the mixed-precision multigrid method: the V-cycle's level
// loops (red-black half-sweeps, fused pairs, restriction, prolongation) and the
// flexible-CG passes around it. Shared by the single-grid kernels (mg.cu) and
// the packed batch kernels (batch.cu). Each body works on the blocks of one
// grid, given as a Span of the launch: a single-grid launch passes all of its
// blocks, a packed launch the range that belongs to the grid.
#pragma once

#include "mg.hpp"
#include "pcg.hpp"
#include "slab.cuh"
#include "solve_state.cuh"
#include "stencil.cuh"

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
// The warps of the blocks that work on one level (a span of the launch).
__device__ __forceinline__ Warps span_warps(const Span& sp) {
    const int t = sp.block * blockDim.x + threadIdx.x;
    return Warps{t >> 5, int((unsigned(sp.blocks) * blockDim.x) >> 5), int(threadIdx.x & 31)};
}
__device__ __forceinline__ Warps grid_warps() { return span_warps(whole_launch()); }

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

// Pairs in the cluster kernel: 8 x 8-row tiles dealt over the cluster's CTAs,
// for levels whose rows are a multiple of 4 and at most LPAIR_N0 long.
constexpr int LPJ = 8, LPK = 8;
constexpr int LPAIR_N0 = 32;
constexpr int kLowerPairRows = (LPJ + 2) * (LPK + 2) * LPAIR_N0 / 4;

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
// The whole V-cycle below the grid-kernel levels in one thread-block cluster:
// the CTAs split every half-sweep, restriction and prolongation, and meet at
// hardware cluster barriers (release/acquire) instead of kernel boundaries.
// Level data moves through L2. The coarsest level is solved densely in FP64
// (x = G b, one warp per row). r0 is the FP64 residual when the first level
// here is the finest level; skip_last_red leaves that level's final red
// half-sweep to the finish kernel. bs and prow are the block's shared arrays
// (512 doubles, kLowerPairRows quads). Every CTA of the cluster calls it with
// the same arguments.
__device__ __forceinline__ void lower_body(const MgLower& P, const double* __restrict__ r0,
                                           const double* __restrict__ G, int skip_last_red, double* bs,
                                           float4* prow) {
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

// ------------------------------------------------------------ sweep trains
// P consecutive red-black half-sweeps of a level (colours c0, 1 - c0, c0, ...)
// in one pass over global memory. A block owns a strip of SJ rows (j) and a
// chunk of SK planes (k) and marches along k. Phase p of a plane needs phase
// p - 1 of the plane and of its two z neighbours, so phase p trails phase
// p - 1 by one plane; each phase's planes wait in a three-plane ring in shared
// memory for the next phase. A phase is computed on one more row on either
// side (and one more plane at either end of the chunk) than the phase after
// it, the halo the later phase reads; the first phase's input, x, is staged
// with P rows of halo. Phase 0 relaxes against x (TRAIN_OLD) or is the
// prolongation fused with the first post-smoothing half-sweep (TRAIN_PROLONG,
// c0 black: neighbours x + P x_c). The last phase's values of
// the block's own rows and planes go to x_out, another buffer than x (blocks
// read each other's halo rows of x). Every value is formed from the operands,
// and summed in the order, of smooth_rows, prolong_black_rows and pair_tile.
//
// The global reads of a step are asynchronous copies (cp.async) issued one
// step ahead: while the phases of plane s run from shared memory, the copies
// of x's plane s + 1, b's plane s and the coarse rows under plane s + 1 are in
// flight. x waits in a four-plane ring (phase 0 of step s still reads planes
// s - 2 .. s), b in a ring of P + 1 planes (phases of step s read planes
// s - P .. s - 1). A prolongation adds the coarse correction to the staged
// plane once, before its phases: the sum x + P x_c is what every neighbour
// term of the fused half-sweep reads, and the cell's own staged value is
// never read (the half-sweeps that follow replace it).
enum TrainStart : int { TRAIN_OLD = 0, TRAIN_PROLONG = 2 };

// Shared-memory layout of a train (in floats): x (4 planes of SJ + 2P rows),
// the rings of phases 0 .. P - 2 (3 planes of SJ + 2 (P - 1 - p) rows), b
// (P + 1 planes of SJ + 2 (P - 1) rows), the coarse rows of one plane (cn0:
// the coarse row length, 0 unless the train starts with a prolongation; cf1:
// the coarsening factor along j).
__host__ __device__ __forceinline__ int train_coarse_rows(int P, int SJ, int cf1) {
    return cf1 == 2 ? (SJ + 2 * P) / 2 + 2 : SJ + 2 * P;
}
__host__ __device__ __forceinline__ size_t train_smem(int P, int SJ, int n0, int cn0, int cf1) {
    size_t rows = size_t(4) * (SJ + 2 * P);
    for (int m = 1; m < P; ++m) rows += size_t(3) * (SJ + 2 * (P - m));
    rows += size_t(P + 1) * (SJ + 2 * (P - 1));
    return (rows * size_t(n0) + (cn0 ? size_t(train_coarse_rows(P, SJ, cf1)) * size_t(cn0) : 0)) * sizeof(float);
}

// Threads of a train block.
constexpr int kTrainThreads = 256;
// The strip of a level's trains of P phases (cn0: the row length of the
// level below): the fewest rows (2, 4, .., 32) that give the last phase an
// item (a quad) for every thread, within the shared memory that lets two
// blocks share an SM; where that memory holds fewer rows, the most it holds;
// where it holds none, the most within kTrainSmemMax; 0 when none fits. (A
// 384-thread block with one item per thread in every phase took 314 us per
// train of the 64-box batch against 275 us for this choice.)
constexpr size_t kTrainSmemTwoBlocks = 110 * 1024;
constexpr size_t kTrainSmemMax = 200 * 1024;
inline int train_strip(const MgLevelDev& L, int cn0, int P) {
    const int quads = L.n[0] >> 2;
    for (size_t cap : {kTrainSmemTwoBlocks, kTrainSmemMax}) {
        int best = 0;
        for (int sj = 2; sj <= 32; sj *= 2) {
            if (train_smem(P, sj, L.n[0], cn0, L.cf[1]) > cap) break;
            best = sj;
            if (sj * quads >= kTrainThreads) break;
        }
        if (best) return best;
    }
    return 0;
}
// Shared memory of one train launch on level L.
inline size_t train_launch_smem(const MgLevelDev& L, const MgLevelDev& C, int P, int sj, int start) {
    return train_smem(P, sj, L.n[0], start == TRAIN_PROLONG ? C.n[0] : 0, L.cf[1]);
}

__device__ __forceinline__ void cp_async16_cg(void* smem_dst, const void* gmem_src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_u32(smem_dst)), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem_dst, const void* gmem_src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(smem_u32(smem_dst)), "l"(gmem_src) : "memory");
}

// One quad of a train phase whose own-colour cells are PAR and PAR + 2,
// relaxed against the phase's input rows (pk: plane k at the quad's row
// offset; pkm, pkp: the planes either side), with the operands and order of
// smooth_rows_v4.
template <int PAR>
__device__ __forceinline__ float4 train_quad(const float* dinv, float w0, float w1, float w2, const float* pk,
                                             const float* pkm, const float* pkp, float4 bq, int i0, int n0, int myz) {
    const int lo = int(i0 > 0), hi = int(i0 + 4 < n0);
    // dinv index of cells e = PAR and PAR + 2 (the x flags differ only at the row's ends)
    const int m0 = PAR == 0 ? (lo | 2 | myz) : (3 | myz);
    const int m1 = PAR == 0 ? (3 | myz) : (1 | (hi << 1) | myz);
    const float4 z4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const float4 xc = *reinterpret_cast<const float4*>(pk);
    const float4 ym = (myz & 4) ? *reinterpret_cast<const float4*>(pk - n0) : z4;
    const float4 yp = (myz & 8) ? *reinterpret_cast<const float4*>(pk + n0) : z4;
    const float4 zm = (myz & 16) ? *reinterpret_cast<const float4*>(pkm) : z4;
    const float4 zq = (myz & 32) ? *reinterpret_cast<const float4*>(pkp) : z4;
    float4 res = xc;
    if (PAR == 0) {
        const float xl = lo ? pk[-1] : 0.0f;
        float a = bq.x;
        if (lo) a += w0 * xl;
        a += w0 * xc.y;
        if (myz & 4) a += w1 * ym.x;
        if (myz & 8) a += w1 * yp.x;
        if (myz & 16) a += w2 * zm.x;
        if (myz & 32) a += w2 * zq.x;
        res.x = a * dinv[m0];
        float c = bq.z;
        c += w0 * xc.y;
        c += w0 * xc.w;
        if (myz & 4) c += w1 * ym.z;
        if (myz & 8) c += w1 * yp.z;
        if (myz & 16) c += w2 * zm.z;
        if (myz & 32) c += w2 * zq.z;
        res.z = c * dinv[m1];
    } else {
        const float xr = hi ? pk[4] : 0.0f;
        float a = bq.y;
        a += w0 * xc.x;
        a += w0 * xc.z;
        if (myz & 4) a += w1 * ym.y;
        if (myz & 8) a += w1 * yp.y;
        if (myz & 16) a += w2 * zm.y;
        if (myz & 32) a += w2 * zq.y;
        res.y = a * dinv[m0];
        float c = bq.w;
        c += w0 * xc.z;
        if (hi) c += w0 * xr;
        if (myz & 4) c += w1 * ym.w;
        if (myz & 8) c += w1 * yp.w;
        if (myz & 16) c += w2 * zm.w;
        if (myz & 32) c += w2 * zq.w;
        res.w = c * dinv[m1];
    }
    return res;
}

// One block's strip and chunk of a train of P phases on level L (x: the
// input buffer).
template <int P>
__device__ __forceinline__ void train_block(const MgLevelDev& L, const MgLevelDev* C, float* __restrict__ x_out,
                                           int c0, int start, int SJ, int SK, int strip, int chunk, float* smem) {
    const int n0 = L.n[0], n1 = L.n[1], n2 = L.n[2];
    const int j0 = strip * SJ, k0 = chunk * SK;
    const int j1 = min(j0 + SJ, n1), k1 = min(k0 + SK, n2);
    const int plane = n0 * n1;
    const int quads = n0 >> 2;
    const bool prolong = start == TRAIN_PROLONG;
    // the stencil's weights in registers (the shared-memory stores of the
    // phases would otherwise make the compiler reload them)
    const float w0 = L.w[0], w1 = L.w[1], w2 = L.w[2];
    const float* const dinv = L.dinv;
    // x ring: rows j0 - P .. j1 + P - 1 of planes s mod 4
    const int XR = SJ + 2 * P;
    float* const xr = smem;
    // ring m (1 .. P - 1) holds phase m - 1: 3 planes of SJ + 2 (P - m) rows
    // from row j0 - (P - m)
    auto ring_rows = [&](int m) { return SJ + 2 * (P - m); };
    auto ring_base = [&](int m) {
        return xr + 4 * XR * n0 + 3 * n0 * ((m - 1) * (SJ + 2 * P) - (m - 1) * m);
    };
    // b ring: rows j0 - (P - 1) .. of planes k mod (P + 1)
    const int BR = SJ + 2 * (P - 1);
    float* const br = ring_base(P);
    // coarse rows under the staged rows of one plane
    float* const cr = br + (P + 1) * BR * n0;
    const int cs0 = prolong ? L.cf[0] - 1 : 0, cs1 = prolong ? L.cf[1] - 1 : 0, cs2 = prolong ? L.cf[2] - 1 : 0;
    const int cn0 = prolong ? C->n[0] : 0;
    const int xj0 = max(0, j0 - P), xj1 = min(n1, j1 + P);            // staged x rows in the level
    const int bj0 = max(0, j0 - (P - 1)), bj1 = min(n1, j1 + (P - 1));  // staged b rows
    const int cj0 = xj0 >> cs1, cj1 = prolong ? ((xj1 - 1) >> cs1) + 1 : 0;
    const float4 z4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const int tid = threadIdx.x, nth = blockDim.x;
    // (row, quad) of a thread's first item of a phase and the step between its items
    const int r_first = tid / quads, q_first = tid - r_first * quads;
    const int dr = nth / quads, dq = nth - dr * quads;

    // Issues the copies that step s + 1 waits for: x's plane s + 1 (with its
    // coarse rows) and b's plane s.
    auto issue = [&](int s) {
        const int sx = s + 1;
        if (sx >= max(0, k0 - P) && sx < min(n2, k1 + P)) {
            float* dst = xr + (sx & 3) * XR * n0 - (j0 - P) * n0;
            const float* src = L.x + size_t(sx) * plane;
            // rows xj0 .. xj1 - 1 are contiguous in both: 16-byte pieces
            const int off0 = xj0 * n0;
            for (int t = tid; t < (xj1 - xj0) * quads; t += nth) cp_async16_cg(dst + off0 + 4 * t, src + off0 + 4 * t);
            if (prolong) {
                const float* csrc = C->x + size_t(sx >> cs2) * C->n[0] * C->n[1];
                for (int t = tid; t < (cj1 - cj0) * cn0; t += nth) cp_async4(cr + t, csrc + cj0 * cn0 + t);
            }
        }
        const int sb = s;
        if (sb >= max(0, k0 - (P - 1)) && sb < min(n2, k1 + P - 1)) {
            float* dst = br + (sb % (P + 1)) * BR * n0 - (j0 - (P - 1)) * n0;
            const float* src = L.b + size_t(sb) * plane;
            const int off0 = bj0 * n0;
            for (int t = tid; t < (bj1 - bj0) * quads; t += nth) cp_async16_cg(dst + off0 + 4 * t, src + off0 + 4 * t);
        }
        cp_async_commit();
    };

    issue(k0 - P - 1);
    for (int s = k0 - P; s <= k1 + P - 1; ++s) {
        cp_async_wait_all();
        __syncthreads();
        if (prolong && s >= max(0, k0 - P) && s < min(n2, k1 + P)) {
            // x + P x_c on the staged plane, before its phases read it
            float* row = xr + (s & 3) * XR * n0 - (j0 - P) * n0;
            for (int t = tid; t < (xj1 - xj0) * quads; t += nth) {
                const int r = t / quads, q = t - r * quads;
                const int j = xj0 + r, i0 = 4 * q;
                float4 v = *reinterpret_cast<float4*>(row + j * n0 + i0);
                const float* crow = cr + ((j >> cs1) - cj0) * cn0;
                v.x = v.x + crow[(i0 + 0) >> cs0];
                v.y = v.y + crow[(i0 + 1) >> cs0];
                v.z = v.z + crow[(i0 + 2) >> cs0];
                v.w = v.w + crow[(i0 + 3) >> cs0];
                *reinterpret_cast<float4*>(row + j * n0 + i0) = v;
            }
            __syncthreads();
        }
        issue(s);
#pragma unroll
        for (int p = 0; p < P; ++p) {
            const int k = s - 1 - p;
            const int h = P - 1 - p;
            if (k >= max(0, k0 - h) && k < min(n2, k1 + h)) {  // uniform over the block
                const int c = (c0 + p) & 1;
                const int jr0 = max(0, j0 - h), jr1 = min(n1, j1 + h);
                const bool last = p == P - 1;
                float* out = last ? nullptr : ring_base(p + 1) + (k % 3) * ring_rows(p + 1) * n0 - (j0 - h) * n0;
                // the input of phase p at planes k - 1, k, k + 1 (x for p = 0),
                // addressed by level row
                const float* pbase;
                int pstride;
                if (p == 0) {
                    pbase = xr - (j0 - P) * n0;
                    pstride = XR * n0;
                } else {
                    pbase = ring_base(p) - (j0 - (P - p)) * n0;
                    pstride = ring_rows(p) * n0;
                }
                const int nslot = p == 0 ? 4 : 3;
                const float* pk = pbase + (k % nslot) * pstride;
                const float* pkm = k > 0 ? pbase + ((k - 1) % nslot) * pstride : pk;
                const float* pkp = k + 1 < n2 ? pbase + ((k + 1) % nslot) * pstride : pk;
                const float* bk = br + (k % (P + 1)) * BR * n0 - (j0 - (P - 1)) * n0;
                const int kz = (int(k > 0) << 4) | (int(k + 1 < n2) << 5);
                // quads of 4 cells (two of each colour): 16-byte rows from
                // shared memory
                int r = r_first, qd = q_first;
                for (int t = tid; t < (jr1 - jr0) * quads; t += nth, r += dr, qd += dq) {
                    if (qd >= quads) {
                        qd -= quads;
                        ++r;
                    }
                    const int j = jr0 + r;
                    const int i0 = 4 * qd;
                    const int par = (c + j + k) & 1;  // the own-colour cells of the quad: par, par + 2
                    const int myz = (int(j > 0) << 2) | (int(j + 1 < n1) << 3) | kz;
                    const int row = j * n0 + i0;
                    const float4 bq = *reinterpret_cast<const float4*>(bk + row);
                    float4 res;
                    if (par)
                        res = train_quad<1>(dinv, w0, w1, w2, pk + row, pkm + row, pkp + row, bq, i0, n0, myz);
                    else
                        res = train_quad<0>(dinv, w0, w1, w2, pk + row, pkm + row, pkp + row, bq, i0, n0, myz);
                    if (!last)
                        *reinterpret_cast<float4*>(out + row) = res;
                    else if (j >= j0 && j < j1)
                        *reinterpret_cast<float4*>(x_out + k * plane + row) = res;
                }
            }
            __syncthreads();
        }
    }
    cp_async_wait_all();
}

// ------------------------------------------------------------ flexible-CG passes

// The finest level's last red half-sweep fused with the outer method's
// preconditioner output: z = x (FP64, z[0] = 0 for the eliminated gauge row),
// r.z and z.r_old reduced and the flexible-CG decision taken. Without a hierarchy
// (a single level solved densely) z is copied from x.
__device__ __forceinline__ void finish_red_body(const MgLevelDev& L, int smooth, SolveState* st, const double* r0,
                                                const double* r1, int mode, Partials part, rb200_trace* trace,
                                                Span sp) {
    __shared__ BlockReduce<2, 0> red;
    if (!gate(st->flags, mode)) return;
    // r (after this iteration's update) and r_old (before it), for r.z and
    // z.r_old (iterations only)
    const int rsel = st->rsel;
    const double* __restrict__ r = rsel ? r1 : r0;
    const double* __restrict__ r_old = rsel ? r0 : r1;
    Neu rz, zq;
    const Warps W = span_warps(sp);
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
                double ro[4] = {0.0, 0.0, 0.0, 0.0};
                if (mode == MODE_ITER) ld_quad(r_old + c0, ro);
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    if (c0 + e == 0) continue;
                    rz.add(rr[e] * zc[e]);
                    if (mode == MODE_ITER) zq.add(zc[e] * ro[e]);
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
                    if (mode == MODE_ITER) zq.add(zc * r_old[c]);
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
                    if (mode == MODE_ITER) zq.add(zc * r_old[c]);
                }
            }
        }
    }
    dd sums[2] = {rz.as_dd(), zq.as_dd()};
    double none[1];
    block_reduce<2, 0>(red, sums, none);
    if (publish_and_check_last<2, 0>(part, sp.block, sp.blocks, sums, none)) {
        fold_partials<2, 0>(part, sp.blocks, red, sums, none);
        if (threadIdx.x == 0) decide_flexible(st, trace, dd_value(sums[0]), dd_value(sums[1]), mode);
    }
}
// The flexible-CG direction pass of the mixed method (src/pressure.rs:657-668,
// :720-731): d = z + beta d (d = z after a restart), q = K d, d.q and the
// decision for alpha; q is not stored (the later passes recompute it). z is read straight from the V-cycle's FP32 output x
// of the finest level (z = f64(x), z[0] = 0 for the eliminated gauge row), so
// no FP64 copy of z is stored. One warp per cell row, lanes along x.
__device__ __forceinline__ void pass1_body(const GridDev& g, const MgLevelDev& L, SolveState* st, double* d0,
                                           double* d1, Partials part, rb200_trace* trace, int kc_len, Span sp) {
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
    const Warps W = span_warps(sp);
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
            acc.add(v.c * qv);
        }
    }
    dd sums[1] = {acc.as_dd()};
    double none[1];
    block_reduce<1, 0>(red, sums, none);
    if (publish_and_check_last<1, 0>(part, sp.block, sp.blocks, sums, none)) {
        fold_partials<1, 0>(part, sp.blocks, red, sums, none);
        if (threadIdx.x == 0) decide_pass1(st, trace, dd_value(sums[0]), flags, dsel);
    }
}
// The flexible-CG update (p += alpha d, r = r_old - alpha K d into the other
// residual buffer, |r|^2 and the candidate
// test) fused with the V-cycle's first half-sweep on the finest level, which
// needs no neighbour: b = f32(r), red x = b / D, black x = 0. Used when the
// finest level is a grid-kernel level.
__device__ __forceinline__ void update_first_body(const GridDev& g, const MgLevelDev& L, SolveState* st,
                                                  double* __restrict__ p, double* r0, double* r1, const double* d0,
                                                  const double* d1, Partials part, rb200_trace* trace, Span sp) {
    __shared__ BlockReduce<1, 0> red;
    const int flags = st->flags;
    if (flags & F_STOP) return;
    const double alpha = st->alpha;
    const double* __restrict__ d = st->dsel ? d1 : d0;
    // r_old is kept: the new residual goes to the other buffer
    const int rsel = st->rsel;
    const double* __restrict__ r = rsel ? r1 : r0;
    double* __restrict__ r_out = rsel ? r0 : r1;
    Neu acc;
    const Warps W = span_warps(sp);
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
                // q = K d first, so that d's neighbour rows are dead before p and r load
                double pv[4], rv[4], dv[4], qv[4];
                ld_quad(d + c0, dv);
                kd_quad(g, d, c0, i0, j, k, dv, qv);
                ld_quad(p + c0, pv);
                ld_quad(r + c0, rv);
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
                *reinterpret_cast<double2*>(r_out + c0) = *reinterpret_cast<double2*>(rv);
                *reinterpret_cast<double2*>(r_out + c0 + 2) = *reinterpret_cast<double2*>(rv + 2);
                *reinterpret_cast<float4*>(L.b + c0) = bq;
                *reinterpret_cast<float4*>(L.x + c0) = xq;
            }
        } else {
            for (int i = W.lane; i < n0; i += 32) {
                const int c = base + i;
                double rc = r[c];
                if (c != 0) {
                    p[c] = p[c] + alpha * d[c];
                    rc = rc - alpha * kd_at(g, d, i, j, k, c);
                    acc.add(rc * rc);
                }
                r_out[c] = rc;
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
    if (publish_and_check_last<1, 0>(part, sp.block, sp.blocks, sums, none)) {
        fold_partials<1, 0>(part, sp.blocks, red, sums, none);
        if (threadIdx.x == 0) {
            st->rsel = rsel ^ 1;
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
}  // namespace rb200
