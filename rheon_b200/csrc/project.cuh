// Device bodies of the operator steps the resident carrier shares with the
// standalone primitives: build_rhs, the actual divergence, the gradient
// correction and the fused correction/divergence/velocity-rate epilogue.
#pragma once

#include "internal.hpp"

namespace rb200 {

constexpr int EW_THREADS = 256;
constexpr int EW_BLOCKS_CAP = 148 * 8;
constexpr float kF32Max = 3.40282346638528859811704183484516925440e+38f;

// ------------------------------------------------------------ build_rhs
// build_rhs (src/operator.rs:460-509) / build_rhs_f64 (:672-708):
//   flux = 0; flux += area_d * (f64(u_lo) - f64(u_hi)) for d = X,Y,Z; b = flux/dt
// RN(1/x) where div_diag may use it (2^-500 < x < 2^500), else 0.
__device__ __forceinline__ double div_reciprocal(double x) { return (x > 0x1p-500 && x < 0x1p500) ? 1.0 / x : 0.0; }

template <class T>
__device__ __forceinline__ void build_rhs_body(const GridDev& g, const T* __restrict__ u, const T* __restrict__ v,
                                               const T* __restrict__ w, double dt, double* __restrict__ out,
                                               int* flags, Span sp) {
    // flux / dt correctly rounded through RN(1/dt) and one exact remainder
    const double rdt = div_reciprocal(dt);
    for (int c = sp.block * blockDim.x + threadIdx.x; c < g.cells; c += sp.blocks * blockDim.x) {
        int i, j, k;
        cell_coords(g, c, i, j, k);
        double flux = 0.0;
        flux += g.area[0] * (double(u[face_idx(g, 0, i, j, k)]) - double(u[face_idx(g, 0, i + 1, j, k)]));
        flux += g.area[1] * (double(v[face_idx(g, 1, i, j, k)]) - double(v[face_idx(g, 1, i, j + 1, k)]));
        flux += g.area[2] * (double(w[face_idx(g, 2, i, j, k)]) - double(w[face_idx(g, 2, i, j, k + 1)]));
        double value = div_diag(flux, dt, rdt);
        if (!isfinite(value)) atomicOr(flags, VF_ARITH);
        out[c] = value;
    }
}

// ------------------------------------------------------------ divergence
// f32 faces (src/operator.rs:543-567): ((dx/h0 + dy/h1) + dz/h2).
// f64 faces (src/operator.rs:711-742): value = 0; value += diff_d/h_d.
// The quotients are correctly rounded through RN(1/h_d) and one exact
// remainder (div_diag): the bits of the divisions.
template <class T>
__device__ __forceinline__ double cell_divergence(const GridDev& g, double xl, double xh, double yl,
                                                  double yh, double zl, double zh) {
    const double qx = div_diag(xh - xl, g.h[0], g.rh[0]);
    const double qy = div_diag(yh - yl, g.h[1], g.rh[1]);
    const double qz = div_diag(zh - zl, g.h[2], g.rh[2]);
    if (sizeof(T) == 4) {
        return qx + qy + qz;
    } else {
        double value = 0.0;
        value += qx;
        value += qy;
        value += qz;
        return value;
    }
}

// ------------------------------------------------------------ correction
// f32: u <- f32( f64(u) - (dt*accel_d)*(p_c - p_l) )   (src/operator.rs:651-662)
// f64: u <- u - dt*(accel_d*(p_c - p_l))               (src/operator.rs:767-775)
template <class T>
__device__ __forceinline__ T corrected(const GridDev& g, int a, T u, double pc, double pl, double dt,
                                       int& flag) {
    if (sizeof(T) == 4) {
        double value = double(u) - dt * g.accel[a] * (pc - pl);
        if (!isfinite(value) || fabs(value) > double(kF32Max)) flag |= VF_ARITH;
        return T(value);
    } else {
        double gradient = g.accel[a] * (pc - pl);
        double value = double(u) - dt * gradient;
        if (!isfinite(value)) flag |= VF_ARITH;
        return T(value);
    }
}

// ------------------------------------------------------------ fused epilogue
// One thread per cell: corrects the three lower faces the cell owns (writes
// them, wall faces copied through), recomputes its three upper faces to form
// the actual divergence of the stored values (actual_divergence_max,
// src/pressure.rs:330-342), and reduces max|div| and max|u_d| per axis
// (velocity_rate, src/simulation.rs:1415-1429).
template <class T>
__device__ __forceinline__ void correct_divergence_body(const GridDev& g, const double* __restrict__ p, double dt,
                                                        const T* __restrict__ iu, const T* __restrict__ iv,
                                                        const T* __restrict__ iw, T* __restrict__ ou,
                                                        T* __restrict__ ov, T* __restrict__ ow, Partials part,
                                                        double* out_scalars, int* flags, Span sp) {
    __shared__ BlockReduce<0, 4> sm;
    const T* in[3] = {iu, iv, iw};
    T* out[3] = {ou, ov, ow};
    const int s[3] = {1, g.n[0], g.n[0] * g.n[1]};
    double mx[4] = {0.0, 0.0, 0.0, 0.0};
    int local = 0;
    for (int c = sp.block * blockDim.x + threadIdx.x; c < g.cells; c += sp.blocks * blockDim.x) {
        int ijk[3];
        cell_coords(g, c, ijk[0], ijk[1], ijk[2]);
        double lo[3], hi[3];
        const double pc = p[c];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            int flo = face_idx(g, a, ijk[0], ijk[1], ijk[2]);
            int fhi = flo + (a == 0 ? 1 : (a == 1 ? g.fc[1][0] : g.fc[2][0] * g.fc[2][1]));
            T vlo = in[a][flo];
            if (ijk[a] > 0) vlo = corrected<T>(g, a, vlo, pc, p[c - s[a]], dt, local);
            out[a][flo] = vlo;
            T vhi = in[a][fhi];
            if (ijk[a] + 1 < g.n[a]) {
                vhi = corrected<T>(g, a, vhi, p[c + s[a]], pc, dt, local);
            } else {
                out[a][fhi] = vhi;
                mx[1 + a] = fmax(mx[1 + a], fabs(double(vhi)));
            }
            mx[1 + a] = fmax(mx[1 + a], fabs(double(vlo)));
            lo[a] = double(vlo);
            hi[a] = double(vhi);
        }
        double div = cell_divergence<T>(g, lo[0], hi[0], lo[1], hi[1], lo[2], hi[2]);
        if (!isfinite(div)) local |= VF_ARITH;
        mx[0] = fmax(mx[0], fabs(div));
    }
    if (local) atomicOr(flags, local);
    dd none[1];
    block_reduce<0, 4>(sm, none, mx);
    if (publish_and_check_last<0, 4>(part, sp.block, sp.blocks, none, mx)) {
        fold_partials<0, 4>(part, sp.blocks, sm, none, mx);
        if (threadIdx.x == 0)
            for (int q = 0; q < 4; ++q) out_scalars[q] = mx[q];
    }
}

}  // namespace rb200
