// Device bodies of the semi-Lagrangian advection (src/advection.rs,
// src/sampling.rs), shared by the standalone kernels (advection.cu) and the
// resident carrier step (carrier.cu). One thread per face or cell; the
// arithmetic type R is double (the reference's f64 arithmetic, bit for bit on
// f32 or f64 storage) or float (the mixed-precision path).
#pragma once

#include "internal.hpp"

namespace rb200 {

constexpr int ADV_THREADS = 256;


template <class R>
__device__ __forceinline__ R clampd(R x, R lo, R hi) {
    // f64::clamp: if x < min { min } then if x > max { max }.
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}

// (x - o_d) / h_d correctly rounded, through the reciprocal of h_d and one
// exact remainder (common.cuh) instead of a division: the same bits.
template <class R>
__device__ __forceinline__ R div_h(R r, const GridDev& g, int d);
template <>
__device__ __forceinline__ double div_h<double>(double r, const GridDev& g, int d) {
    return div_diag(r, g.h[d], g.rh[d]);
}
template <>
__device__ __forceinline__ float div_h<float>(float r, const GridDev& g, int d) {
    return div_f32(r, float(g.h[d]), g.rhf[d]);
}

// The integer value of an integer-valued fq in [0, 2^31).
__device__ __forceinline__ int cell_of(double fq) { return __double2loint(fq + 0x1p52); }
__device__ __forceinline__ int cell_of(float fq) {
    if (fq < 0x1p22f) return __float_as_int(fq + 0x1p23f) - 0x4B000000;
    return int(fq);
}

// The scaled coordinate (x - o_d) / h_d of a position after the box clamp of
// ScalarSampler::sample (src/sampling.rs:74-122). It depends on the position
// only, so the three components of a velocity sample share it.
template <class R>
__device__ __forceinline__ void scaled_position(const GridDev& g, const R pos[3], R xh[3]) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const R x = clampd<R>(pos[d], R(g.o[d]), R(g.up[d]));
        xh[d] = div_h<R>(x - R(g.o[d]), g, d);
    }
}

// ScalarSampler::sample (src/sampling.rs:74-122) in arithmetic type R from
// the scaled coordinate: q = clamp(xh - offset) per axis, the eight corners
// weighted ((1 * w_x) * w_y) * w_z in the reference's z, y, x order, the sum
// clamped to the corners' range. 1 * w_x is w_x exactly, so the products
// w_x w_y are formed once per (x, y) pair and the corner offsets once per
// axis; the values and every rounding are the reference's. double reproduces
// the reference; float is the mixed-precision path.
template <class T, class R>
__device__ __forceinline__ R sample_at(const T* __restrict__ values, const int dims[3], const R off[3], const R xh[3],
                                       int& flag) {
    int lo[3], hi[3];
    R t[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        R q = clampd<R>(xh[d] - off[d], R(0), R(dims[d] - 1));
        if (!isfinite(q)) {
            flag |= VF_ARITH;
            q = R(0);
        }
        // q >= 0, so floor(q) is its truncation; fq is an integer below 2^31,
        // exactly R(lo), and lo is read from the mantissa of fq + 2^52 (2^23
        // in float, below 2^22) instead of by conversion instructions
        const R fq = trunc(q);
        lo[d] = cell_of(fq);
        hi[d] = min(lo[d] + 1, dims[d] - 1);
        t[d] = q - fq;
    }
    const R wx[2] = {R(1) - t[0], t[0]};
    const R wy[2] = {R(1) - t[1], t[1]};
    const R wz[2] = {R(1) - t[2], t[2]};
    const R wxy[2][2] = {{wx[0] * wy[0], wx[1] * wy[0]}, {wx[0] * wy[1], wx[1] * wy[1]}};
    const int px[2] = {lo[0], hi[0]};
    const int py[2] = {dims[0] * lo[1], dims[0] * hi[1]};
    const int plane = dims[0] * dims[1];
    const int pz[2] = {plane * lo[2], plane * hi[2]};
    R result = R(0);
    R minimum = R(CUDART_INF);
    R maximum = R(-CUDART_INF);
#pragma unroll
    for (int z = 0; z < 2; ++z)
#pragma unroll
        for (int y = 0; y < 2; ++y)
#pragma unroll
            for (int x = 0; x < 2; ++x) {
                const R weight = wxy[y][x] * wz[z];
                const R value = R(__ldg(values + (px[x] + py[y] + pz[z])));
                minimum = fmin(minimum, value);
                maximum = fmax(maximum, value);
                result += weight * value;
            }
    if (!isfinite(result)) flag |= VF_ARITH;
    return clampd<R>(result, minimum, maximum);
}

template <class T, class R>
__device__ __forceinline__ R sample(const GridDev& g, const T* __restrict__ values, const int dims[3], const R off[3],
                                    const R pos[3], int& flag) {
    R xh[3];
    scaled_position<R>(g, pos, xh);
    return sample_at<T, R>(values, dims, off, xh, flag);
}

template <class T>
struct Faces {
    const T* f[3];
};

template <class R>
__device__ __forceinline__ void face_geometry(const GridDev& g, int a, int dims[3], R off[3]) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        dims[d] = g.fc[a][d];
        off[d] = d == a ? R(0) : R(0.5);
    }
}

template <class T, class R>
__device__ __forceinline__ void velocity_sample(const GridDev& g, const Faces<T>& vel, const R pos[3], R out[3],
                                                int& flag) {
    R xh[3];
    scaled_position<R>(g, pos, xh);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        int dims[3];
        R off[3];
        face_geometry<R>(g, a, dims, off);
        out[a] = sample_at<T, R>(vel.f[a], dims, off, xh, flag);
    }
}

// VelocitySampler::departure (src/sampling.rs:160-175).
template <class R>
__device__ __forceinline__ void departure(const GridDev& g, const R pos[3], const R vel[3], R dt, R out[3],
                                          int& flag) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        R value = pos[d] - dt * vel[d];
        if (!isfinite(value)) flag |= VF_ARITH;
        out[d] = clampd<R>(value, R(g.o[d]), R(g.up[d]));
    }
}

// The second half of VelocitySampler::backtrace (src/sampling.rs:151-159),
// midpoint RK2, from the velocity at the start point.
template <class T, class R>
__device__ __forceinline__ void backtrace_from(const GridDev& g, const Faces<T>& vel, const R pos[3],
                                               const R initial[3], R dt, R out[3], int& flag) {
    R mid[3], v1[3];
    departure<R>(g, pos, initial, R(0.5) * dt, mid, flag);
    velocity_sample<T, R>(g, vel, mid, v1, flag);
    departure<R>(g, pos, v1, dt, out, flag);
}

// VelocitySampler::backtrace (src/sampling.rs:151-159): midpoint RK2.
template <class T, class R>
__device__ __forceinline__ void backtrace(const GridDev& g, const Faces<T>& vel, const R pos[3], R dt, R out[3],
                                          int& flag) {
    R initial[3];
    velocity_sample<T, R>(g, vel, pos, initial, flag);
    backtrace_from<T, R>(g, vel, pos, initial, dt, out, flag);
}

// The velocity at the centre of face p of axis a. There the sampler's
// fractions are 0 or 1/2 (exactly so where the grid's centres are exact; the
// FP32 path takes the exact face position in any case), so the face's own
// component is its value and each other component c is the mean of the four
// c-faces around it in the a-c plane: the corners of weight 1/4, summed from 0
// in the sampler's z, y, x order. The corners of weight 0 add only zeros,
// which change no sum that starts from +0, and the mean lies within the
// corners' range, so the result has the bits of the eight-corner sample, with
// four loads per component instead of eight and none for the own one.
template <class T, class R>
__device__ __forceinline__ void face_velocity(const GridDev& g, const Faces<T>& vel, const int p[3], int a, R out[3],
                                              int& flag) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const int s1 = g.fc[c][0], s2 = g.fc[c][0] * g.fc[c][1];
        const int at = p[0] + s1 * p[1] + s2 * p[2];
        const T* f = vel.f[c];
        if (c == a) {
            out[c] = R(0) + R(f[at]);
            if (!isfinite(out[c])) flag |= VF_ARITH;
            continue;
        }
        // c-faces: the corners are p_a - 1 and p_a along a, p_c and p_c + 1
        // along c; the higher of the two axes is the outer one of the sum
        auto stride = [&](int d) { return d == 0 ? 1 : (d == 1 ? s1 : s2); };
        const int su = stride(min(a, c)), sv = stride(max(a, c));
        const int base = at - stride(a);
        const R w = R(0.25);
        R r = R(0);
        r += w * R(f[base]);
        r += w * R(f[base + su]);
        r += w * R(f[base + sv]);
        r += w * R(f[base + su + sv]);
        if (!isfinite(r)) flag |= VF_ARITH;
        out[c] = r;
    }
}

// advect_velocity (src/advection.rs:28-68): wall-normal faces are exactly 0,
// every other face samples its own component at the RK2 departure point.
template <class T, class R>
__device__ __forceinline__ void advect_velocity_body(const GridDev& g, const Faces<T>& vel, double dt, T* ou, T* ov,
                                                     T* ow, const float* __restrict__ tracer, double gb, int* flags,
                                                     Span sp) {
    const long long total = (long long)g.flen[0] + g.flen[1] + g.flen[2];
    int local = 0;
    for (long long t = sp.block * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)sp.blocks * blockDim.x) {
        int a = 0;
        long long f = t;
        if (f >= g.flen[0]) {
            f -= g.flen[0];
            a = 1;
            if (f >= g.flen[1]) {
                f -= g.flen[1];
                a = 2;
            }
        }
        // face coordinates by multiply-shift (face indices of one axis fit 31 bits)
        const int fi = int(f);
        int p[3];
        p[2] = fast_div(fi, g.fplane[a]);
        const int in_plane = fi - p[2] * (g.fc[a][0] * g.fc[a][1]);
        p[1] = fast_div(in_plane, g.frow[a]);
        p[0] = in_plane - p[1] * g.fc[a][0];
        T* dst = a == 0 ? ou : (a == 1 ? ov : ow);
        if (p[a] == 0 || p[a] + 1 == g.fc[a][a]) {
            dst[f] = T(0);
            continue;
        }
        R pos[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) pos[d] = R(g.o[d] + (double(p[d]) + (d == a ? 0.0 : 0.5)) * g.h[d]);
        R dep[3];
        if (std::is_same<R, float>::value || g.exact_centres) {
            R initial[3];
            face_velocity<T, R>(g, vel, p, a, initial, local);
            backtrace_from<T, R>(g, vel, pos, initial, R(dt), dep, local);
        } else {
            backtrace<T, R>(g, vel, pos, R(dt), dep, local);
        }
        int dims[3];
        R off[3];
        face_geometry<R>(g, a, dims, off);
        T value = T(sample<T, R>(g, vel.f[a], dims, off, dep, local));
        if (a == 1 && tracer != nullptr && gb != 0.0) {
            // Buoyancy hook (new): interior Y face, after advection, before pressure.
            int below = cell_idx(g, p[0], p[1] - 1, p[2]);
            int above = cell_idx(g, p[0], p[1], p[2]);
            double c = 0.5 * (double(tracer[below]) + double(tracer[above]));
            double forced = double(value) + dt * (gb * c);
            if (!isfinite(forced)) local |= VF_ARITH;
            value = T(forced);
        }
        dst[f] = value;
    }
    if (local) atomicOr(flags, local);
}

// advect_tracer (src/advection.rs:72-102), evaluated densely; the reference's
// zero-support skip produces the same bits (tests/advection_contract.rs:7-41).
template <class T, class R>
__device__ __forceinline__ void advect_tracer_body(const GridDev& g, const float* __restrict__ old,
                                                   const Faces<T>& vel, double dt, float* __restrict__ out,
                                                   int* flags, Span sp) {
    int local = 0;
    int dims[3] = {g.n[0], g.n[1], g.n[2]};
    R off[3] = {R(0.5), R(0.5), R(0.5)};
    for (int c = sp.block * blockDim.x + threadIdx.x; c < g.cells; c += sp.blocks * blockDim.x) {
        int p[3];
        cell_coords(g, c, p[0], p[1], p[2]);
        R pos[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) pos[d] = R(g.o[d] + (double(p[d]) + 0.5) * g.h[d]);
        R dep[3];
        backtrace<T, R>(g, vel, pos, R(dt), dep, local);
        out[c] = float(sample<float, R>(g, old, dims, off, dep, local));
    }
    if (local) atomicOr(flags, local);
}

}  // namespace rb200
