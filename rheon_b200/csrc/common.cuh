// Shared device-side definitions for the sm_100a carrier kernels.
//
// Layout in HBM follows Rheon's geometry (src/geometry.rs:250-258): cells are
// x-fastest, index i + nx*(j + ny*k); the faces of axis d have counts[d]+1
// along d and are also x-fastest, each axis in its own array.
//
// The library is compiled with -fmad=false: Rust never contracts a*b+c, so
// every multiply-add below rounds twice, exactly like the reference.
#pragma once

#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

#include "../../include/rheon_b200.h"

namespace rb200 {

// Exact floor(c / d) for 0 <= c < 2^31 by one multiply and shift
// (Granlund and Montgomery, "Division by invariant integers using
// multiplication", 1994, the round-up method): with l = ceil(log2 d) and
// m = floor(2^(31+l) / d) + 1, 2^(31+l) < m d <= 2^(31+l) + 2^l, so
// floor(c m / 2^(31+l)) = floor(c / d); c m < 2^63.
struct FastDiv {
    unsigned long long m;
    int shift;
};

inline FastDiv make_fastdiv(unsigned d) {
    int l = 0;
    while ((1ull << l) < d) ++l;
    return FastDiv{(1ull << (31 + l)) / d + 1, 31 + l};
}

__device__ __forceinline__ int fast_div(int c, const FastDiv& f) {
    return int((unsigned long long)(unsigned)c * f.m >> f.shift);
}

// Geometry and sealed-box operator coefficients, passed by value to kernels.
// PressureOperator::new (src/operator.rs:58-97) fixes area, accel, weight and
// the 64 neighbour-mask diagonals summed lower/upper x X,Y,Z.
struct GridDev {
    int n[3];        // cell counts
    int fc[3][3];    // face counts per axis
    int flen[3];     // face array lengths
    int cells;       // n0*n1*n2
    double h[3];
    double rh[3];    // RN(1/h_d) in double where div_diag may use it, else 0
    float rhf[3];    // RN(1/f32(h_d)) in float where div_f32 may use it, else 0
    int exact_centres;  // nonzero: every cell and face centre scales exactly (make_grid_dev)
    FastDiv frow[3];    // floor(f / fc[a][0]) for a face index f of axis a
    FastDiv fplane[3];  // floor(f / (fc[a][0] fc[a][1]))
    FastDiv crow;       // floor(c / n0) for a cell index c
    FastDiv cplane;     // floor(c / (n0 n1))
    double o[3];
    double up[3];
    double area[3];
    double accel[3];
    double weight[3];
    double volume;
    double diag[64];
    double rdiag[64];  // RN(1/diag) where div_diag may use it, else 0
};

// The blocks of a launch that work on one grid: this block's index among them
// and their number. A launch over one grid gives every block to it; a packed
// launch over a batch of grids gives each grid a contiguous range of blocks.
struct Span {
    int block, blocks;
};
__device__ __forceinline__ Span whole_launch() { return Span{int(blockIdx.x), int(gridDim.x)}; }

__device__ __forceinline__ int cell_idx(const GridDev& g, int i, int j, int k) {
    return i + g.n[0] * (j + g.n[1] * k);
}
// The coordinates of cell c by multiply-shift (cell indices fit 31 bits).
__device__ __forceinline__ void cell_coords(const GridDev& g, int c, int& i, int& j, int& k) {
    k = fast_div(c, g.cplane);
    const int in_plane = c - k * (g.n[0] * g.n[1]);
    j = fast_div(in_plane, g.crow);
    i = in_plane - j * g.n[0];
}

__device__ __forceinline__ int face_idx(const GridDev& g, int a, int i, int j, int k) {
    return i + g.fc[a][0] * (j + g.fc[a][1] * k);
}
// Neighbour mask of a cell: bit 0/1 lower/upper X, 2/3 Y, 4/5 Z.
__device__ __forceinline__ int diag_mask(const GridDev& g, int i, int j, int k) {
    return int(i > 0) | (int(i + 1 < g.n[0]) << 1) | (int(j > 0) << 2) | (int(j + 1 < g.n[1]) << 3) |
           (int(k > 0) << 4) | (int(k + 1 < g.n[2]) << 5);
}
// PressureOperator::diagonal (src/operator.rs:813-822).
__device__ __forceinline__ double diag_at(const GridDev& g, int i, int j, int k) { return g.diag[diag_mask(g, i, j, k)]; }

// r / D rounded to nearest, as IEEE division rounds it, through y = RN(1/D):
// q = RN(r*y) is within one ulp of r/D, the remainder r - q*D is exact by
// FMA, and RN(q + rem*y) is the correctly rounded quotient (Markstein's
// theorem for round-to-nearest: y within half an ulp of 1/D, q within one ulp
// of r/D). Three floating-point operations instead of a division. The
// theorem's conditions (q and the remainder neither overflow nor underflow)
// hold for 2^-450 <= |r| < 2^451 with a table entry y != 0 (set only for
// 2^-500 < D < 2^500): q stays within (2^-950, 2^951) and the remainder above
// 2^-504. r = +-0 gives +0, so the sign is taken from r (r / D has the sign of
// r for D > 0). div_diag_fast_ok tells the cases covered; every other case
// divides.
__device__ __forceinline__ bool div_diag_range_ok(double r) {
    const unsigned ahi = unsigned(__double2hiint(r)) & 0x7fffffffu;
    const unsigned e = ahi >> 20;  // biased exponent; 573..1473: 2^-450 <= |r| < 2^451
    return e - 573u <= 900u || (ahi | unsigned(__double2loint(r))) == 0u;
}
__device__ __forceinline__ bool div_diag_fast_ok(double r, double y) { return y != 0.0 && div_diag_range_ok(r); }
__device__ __forceinline__ double div_diag_fast(double r, double D, double y) {
    const double q = r * y;
    const double rem = fma(-q, D, r);
    return copysign(fma(rem, y, q), r);
}
__device__ __forceinline__ double div_diag(double r, double D, double y) {
    if (div_diag_fast_ok(r, y)) return div_diag_fast(r, D, y);
    return r / D;
}

// The same correctly rounded quotient r / D in binary32 (Markstein's theorem
// holds for any binary precision): y = RN(1/D) in float, set only for
// 2^-60 < D < 2^60; the fast path covers r = +-0 and 2^-60 <= |r| < 2^60, where
// q stays within (2^-120, 2^120) and the remainder above 2^-84, all normal.
__device__ __forceinline__ float div_f32(float r, float D, float y) {
    const unsigned ab = __float_as_uint(r) & 0x7fffffffu;
    const unsigned e = ab >> 23;  // biased exponent; 67..186: 2^-60 <= |r| < 2^60
    if (y != 0.0f && (e - 67u <= 119u || ab == 0u)) {
        const float q = r * y;
        const float rem = fmaf(-q, D, r);
        return copysignf(fmaf(rem, y, q), r);
    }
    return r / D;
}

// ------------------------------------------------------------ double-double
// Error-free two-sum (Knuth). With products rounded exactly as the reference
// rounds them, a double-double accumulation of the rounded products followed
// by one final rounding lands on the same double as Rheon's serial Neumaier
// sum (src/pressure.rs:135-148) except in rare near-tie cases.
struct dd {
    double hi, lo;
};

__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
    s = a + b;
    double bb = s - a;
    e = (a - (s - bb)) + (b - bb);
}

__device__ __forceinline__ dd dd_add(dd a, dd b) {
    double s, e;
    two_sum(a.hi, b.hi, s, e);
    e = e + (a.lo + b.lo);
    dd r;
    two_sum(s, e, r.hi, r.lo);
    return r;
}

__device__ __forceinline__ dd dd_add1(dd a, double b) {
    double s, e;
    two_sum(a.hi, b, s, e);
    e = e + a.lo;
    dd r;
    two_sum(s, e, r.hi, r.lo);
    return r;
}

__device__ __forceinline__ double dd_value(dd a) { return a.hi + a.lo; }

__device__ __forceinline__ dd dd_shfl_xor(dd a, int m) {
    dd r;
    r.hi = __shfl_xor_sync(0xffffffffu, a.hi, m);
    r.lo = __shfl_xor_sync(0xffffffffu, a.lo, m);
    return r;
}

__device__ __forceinline__ dd warp_reduce_dd(dd a) {
#pragma unroll
    for (int m = 16; m >= 1; m >>= 1) a = dd_add(a, dd_shfl_xor(a, m));
    return a;
}

__device__ __forceinline__ double warp_reduce_max(double a) {
#pragma unroll
    for (int m = 16; m >= 1; m >>= 1) a = fmax(a, __shfl_xor_sync(0xffffffffu, a, m));
    return a;
}

// Block reduction of K double-double sums and M maxima. Deterministic: fixed
// lane pattern, fixed warp order. Result valid in thread 0. blockDim.x*y*z
// must be a multiple of 32 and at most 1024.
template <int K, int M>
struct BlockReduce {
    dd s[32][K > 0 ? K : 1];
    double m[32][M > 0 ? M : 1];
};

template <int K, int M>
__device__ __forceinline__ void block_reduce(BlockReduce<K, M>& sm, dd (&sums)[K > 0 ? K : 1],
                                             double (&maxs)[M > 0 ? M : 1]) {
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int nthreads = blockDim.x * blockDim.y * blockDim.z;
    const int lane = tid & 31, warp = tid >> 5, nwarps = (nthreads + 31) >> 5;
#pragma unroll
    for (int q = 0; q < K; ++q) sums[q] = warp_reduce_dd(sums[q]);
#pragma unroll
    for (int q = 0; q < M; ++q) maxs[q] = warp_reduce_max(maxs[q]);
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < K; ++q) sm.s[warp][q] = sums[q];
#pragma unroll
        for (int q = 0; q < M; ++q) sm.m[warp][q] = maxs[q];
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int q = 0; q < K; ++q) sums[q] = lane < nwarps ? sm.s[lane][q] : dd{0.0, 0.0};
#pragma unroll
        for (int q = 0; q < M; ++q) maxs[q] = lane < nwarps ? sm.m[lane][q] : 0.0;
#pragma unroll
        for (int q = 0; q < K; ++q) sums[q] = warp_reduce_dd(sums[q]);
#pragma unroll
        for (int q = 0; q < M; ++q) maxs[q] = warp_reduce_max(maxs[q]);
    }
    __syncthreads();
}

// Partials of one reduction stage: per block K dd sums and M maxima.
// The last block to arrive (atomic ticket, no spinning) folds all partials in
// block order, so the result does not depend on block scheduling.
struct Partials {
    double* data;        // [nblocks][2K + M]
    unsigned* ticket;    // zero between uses
};

template <int K, int M>
__device__ __forceinline__ bool publish_and_check_last(const Partials& P, int block_id, int nblocks,
                                                       const dd (&sums)[K > 0 ? K : 1],
                                                       const double (&maxs)[M > 0 ? M : 1]) {
    __shared__ bool last;
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    if (tid == 0) {
        double* slot = P.data + size_t(block_id) * (2 * K + M);
#pragma unroll
        for (int q = 0; q < K; ++q) {
            slot[2 * q] = sums[q].hi;
            slot[2 * q + 1] = sums[q].lo;
        }
#pragma unroll
        for (int q = 0; q < M; ++q) slot[2 * K + q] = maxs[q];
        __threadfence();
        unsigned t = atomicAdd(P.ticket, 1u);
        last = (t == unsigned(nblocks - 1));
    }
    __syncthreads();
    return last;
}

// Called by all threads of the last block: folds nblocks partials.
template <int K, int M>
__device__ __forceinline__ void fold_partials(const Partials& P, int nblocks, BlockReduce<K, M>& sm,
                                              dd (&sums)[K > 0 ? K : 1],
                                              double (&maxs)[M > 0 ? M : 1]) {
    __threadfence();
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int nthreads = blockDim.x * blockDim.y * blockDim.z;
#pragma unroll
    for (int q = 0; q < K; ++q) sums[q] = dd{0.0, 0.0};
#pragma unroll
    for (int q = 0; q < M; ++q) maxs[q] = 0.0;
    for (int b = tid; b < nblocks; b += nthreads) {
        const double* slot = P.data + size_t(b) * (2 * K + M);
#pragma unroll
        for (int q = 0; q < K; ++q) sums[q] = dd_add(sums[q], dd{__ldcg(slot + 2 * q), __ldcg(slot + 2 * q + 1)});
#pragma unroll
        for (int q = 0; q < M; ++q) maxs[q] = fmax(maxs[q], __ldcg(slot + 2 * K + q));
    }
    block_reduce<K, M>(sm, sums, maxs);
    if (tid == 0) *P.ticket = 0u;
}

// Wall-normal faces of axis a are the ones with coordinate 0 or n_a.
__device__ __forceinline__ bool is_wall_face(const GridDev& g, int a, int i, int j, int k) {
    int c = a == 0 ? i : (a == 1 ? j : k);
    return c == 0 || c == g.n[a];
}

}  // namespace rb200
