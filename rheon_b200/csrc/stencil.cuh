// 2.5-D plane marching for the 7-point sealed-box operator.
//
// A block owns a TX x TY column tile and walks a chunk of z planes. The x/y
// neighbours of the current plane come from a shared-memory tile with a
// one-cell halo; the z neighbours of the block's own column stay in registers.
// Each value is produced once per plane by a caller-supplied `value(c,i,j,k)`
// functor (a load, or a load plus arithmetic such as the fused PCG direction
// update), so every array is streamed from HBM once per sweep.
//
// The operator row follows apply_full's sealed-box path (src/operator.rs:400-416):
//   q = 0; for d in X,Y,Z: if lower exists q += w_d*(x_c - x_lower);
//                          if upper exists q += w_d*(x_c - x_upper)
#pragma once

#include "common.cuh"

namespace rb200 {

constexpr int TX = 32;
constexpr int TY = 8;
constexpr int TILE_THREADS = TX * TY;

struct Neigh {
    double c, xm, xp, ym, yp, zm, zp;
};

// apply_full row (sealed box), same addition order as the reference.
__device__ __forceinline__ double apply_row(const GridDev& g, int i, int j, int k, const Neigh& v) {
    double q = 0.0;
    if (i > 0) q += g.weight[0] * (v.c - v.xm);
    if (i + 1 < g.n[0]) q += g.weight[0] * (v.c - v.xp);
    if (j > 0) q += g.weight[1] * (v.c - v.ym);
    if (j + 1 < g.n[1]) q += g.weight[1] * (v.c - v.yp);
    if (k > 0) q += g.weight[2] * (v.c - v.zm);
    if (k + 1 < g.n[2]) q += g.weight[2] * (v.c - v.zp);
    return q;
}

// q = K d (the sealed-box operator row, apply_row) where the flexible-CG passes
// need it: recomputed from the stored direction instead of stored by the
// direction pass, which saves a write and a read of an FP64 vector per
// iteration. kd_quad takes the four cells c0..c0+3 of row (j, k) of a grid
// whose rows are a multiple of 4 long (dv: d at the quad), with 16-byte loads
// of the y and z neighbour rows; kd_at takes one cell. The gauge row's q is 0.
__device__ __forceinline__ void ld_quad(const double* __restrict__ a, double (&o)[4]) {
    const double2 lo = *reinterpret_cast<const double2*>(a);
    const double2 hi = *reinterpret_cast<const double2*>(a + 2);
    o[0] = lo.x;
    o[1] = lo.y;
    o[2] = hi.x;
    o[3] = hi.y;
}
__device__ __forceinline__ void kd_quad(const GridDev& g, const double* __restrict__ d, int c0, int i0, int j,
                                        int k, const double (&dv)[4], double (&qq)[4]) {
    const int n0 = g.n[0], sy = n0, sz = n0 * g.n[1];
    double ym[4] = {0.0, 0.0, 0.0, 0.0}, yp[4] = {0.0, 0.0, 0.0, 0.0};
    double zm[4] = {0.0, 0.0, 0.0, 0.0}, zp[4] = {0.0, 0.0, 0.0, 0.0};
    if (j > 0) ld_quad(d + c0 - sy, ym);
    if (j + 1 < g.n[1]) ld_quad(d + c0 + sy, yp);
    if (k > 0) ld_quad(d + c0 - sz, zm);
    if (k + 1 < g.n[2]) ld_quad(d + c0 + sz, zp);
    const double xl = i0 > 0 ? d[c0 - 1] : 0.0;
    const double xr = i0 + 4 < n0 ? d[c0 + 4] : 0.0;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        Neigh v;
        v.c = dv[e];
        v.xm = e == 0 ? xl : dv[e - 1];
        v.xp = e == 3 ? xr : dv[e + 1];
        v.ym = ym[e];
        v.yp = yp[e];
        v.zm = zm[e];
        v.zp = zp[e];
        qq[e] = (c0 + e == 0) ? 0.0 : apply_row(g, i0 + e, j, k, v);
    }
}
__device__ __forceinline__ double kd_at(const GridDev& g, const double* __restrict__ d, int i, int j, int k, int c) {
    if (c == 0) return 0.0;
    const int sy = g.n[0], sz = g.n[0] * g.n[1];
    Neigh v;
    v.c = d[c];
    v.xm = i > 0 ? d[c - 1] : 0.0;
    v.xp = i + 1 < g.n[0] ? d[c + 1] : 0.0;
    v.ym = j > 0 ? d[c - sy] : 0.0;
    v.yp = j + 1 < g.n[1] ? d[c + sy] : 0.0;
    v.zm = k > 0 ? d[c - sz] : 0.0;
    v.zp = k + 1 < g.n[2] ? d[c + sz] : 0.0;
    return apply_row(g, i, j, k, v);
}

// Launch geometry of a marching kernel for a z-chunk depth zc.
struct MarchGrid {
    dim3 grid;
    dim3 block;
    int zc;
    int nblocks;
};

inline MarchGrid march_grid(const int n[3], int zc) {
    MarchGrid m;
    m.zc = zc;
    m.block = dim3(TX, TY, 1);
    m.grid = dim3((n[0] + TX - 1) / TX, (n[1] + TY - 1) / TY, (n[2] + zc - 1) / zc);
    m.nblocks = int(m.grid.x * m.grid.y * m.grid.z);
    return m;
}

// Walk the block's z-chunk. `value(c,i,j,k)` yields the marched field at an
// in-domain cell; `body(c,i,j,k,neigh)` consumes the stencil of an in-domain
// cell of the block's own column. Out-of-domain neighbours are never read by
// apply_row (its masks skip them). All threads reach every __syncthreads.
template <class Value, class Body>
__device__ __forceinline__ void march(const GridDev& g, int zc, Value value, Body body) {
    __shared__ double s[TY + 2][TX + 2];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int tid = tx + TX * ty;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const int i = x0 + tx, j = y0 + ty;
    const int k0 = blockIdx.z * zc;
    const int k1 = min(k0 + zc, g.n[2]);
    const bool own = i < g.n[0] && j < g.n[1];
    const int plane = g.n[0] * g.n[1];
    double dm = 0.0, dc = 0.0, dp = 0.0;
    int c = own ? cell_idx(g, i, j, k0) : 0;
    if (own) {
        if (k0 > 0) dm = value(c - plane, i, j, k0 - 1);
        dc = value(c, i, j, k0);
    }
    for (int k = k0; k < k1; ++k) {
        if (own && k + 1 < g.n[2]) dp = value(c + plane, i, j, k + 1);
        s[ty + 1][tx + 1] = dc;
        // Halo of the current plane: TX below, TX above, TY left, TY right.
        for (int h = tid; h < 2 * TX + 2 * TY; h += TILE_THREADS) {
            int hi, hj, si, sj;
            if (h < TX) {
                hi = x0 + h; hj = y0 - 1; si = h + 1; sj = 0;
            } else if (h < 2 * TX) {
                hi = x0 + h - TX; hj = y0 + TY; si = h - TX + 1; sj = TY + 1;
            } else if (h < 2 * TX + TY) {
                hi = x0 - 1; hj = y0 + h - 2 * TX; si = 0; sj = h - 2 * TX + 1;
            } else {
                hi = x0 + TX; hj = y0 + h - 2 * TX - TY; si = TX + 1; sj = h - 2 * TX - TY + 1;
            }
            double hv = 0.0;
            if (hi >= 0 && hi < g.n[0] && hj >= 0 && hj < g.n[1])
                hv = value(cell_idx(g, hi, hj, k), hi, hj, k);
            s[sj][si] = hv;
        }
        __syncthreads();
        if (own) {
            Neigh v;
            v.c = dc;
            v.xm = s[ty + 1][tx];
            v.xp = s[ty + 1][tx + 2];
            v.ym = s[ty][tx + 1];
            v.yp = s[ty + 2][tx + 1];
            v.zm = dm;
            v.zp = dp;
            body(c, i, j, k, v);
        }
        __syncthreads();
        dm = dc;
        dc = dp;
        c += plane;
    }
}

}  // namespace rb200
