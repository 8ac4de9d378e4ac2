// Host-side internals shared by the translation units of librheon_b200.
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <string>

#include "../../include/rheon_b200.h"
#include "common.cuh"

namespace rb200 {

// Thread-local message for entry points without a handle.
void set_error(const std::string& msg);
const char* get_error();
// Makes `device` current after checking that it is an sm_100 part.
int select_device(int device);
// A box-flux workspace built for this grid (bit-equal geometry), density
// (bit-equal) and pressure method (box_flux.cu).
bool box_flux_matches(const rb200_box_flux* workspace, const rb200_grid& grid, double density, int method);

#define RB200_CUDA(call)                                                                   \
    do {                                                                                   \
        cudaError_t err__ = (call);                                                        \
        if (err__ != cudaSuccess) {                                                        \
            ::rb200::set_error(std::string(#call) + ": " + cudaGetErrorString(err__));     \
            return RB200_EXECUTION;                                                        \
        }                                                                                  \
    } while (0)

// GridGeometry::new (src/geometry.rs:114-191) plus PressureOperator::new
// (src/operator.rs:58-97). Rejects grids whose cell or face arrays do not fit
// 32-bit indexing (more than 2^31-1 elements), which this library does not use.
inline int make_grid_dev(const rb200_grid* in, double density, GridDev* g) {
    if (!in || !g) return RB200_INVALID_ARGUMENT;
    std::memset(g, 0, sizeof(*g));
    const double eps = std::numeric_limits<double>::epsilon();
    uint64_t n64[3];
    for (int d = 0; d < 3; ++d) {
        if (in->counts[d] == 0) return RB200_INVALID_ARGUMENT;
        if (!std::isfinite(in->spacing[d]) || in->spacing[d] <= 0.0) return RB200_INVALID_ARGUMENT;
        if (!std::isfinite(in->origin[d])) return RB200_INVALID_ARGUMENT;
        n64[d] = in->counts[d];
        if (n64[d] > 2000000000ull) return RB200_UNSUPPORTED;
    }
    const uint64_t lim = 0x7fffffffull;
    uint64_t cells = n64[0] * n64[1];
    if (cells > lim) return RB200_UNSUPPORTED;
    cells *= n64[2];
    if (cells > lim) return RB200_UNSUPPORTED;
    for (int a = 0; a < 3; ++a) {
        uint64_t f = 1;
        for (int d = 0; d < 3; ++d) {
            f *= n64[d] + (a == d ? 1 : 0);
            if (f > lim) return RB200_UNSUPPORTED;
        }
        g->flen[a] = int(f);
        for (int d = 0; d < 3; ++d) g->fc[a][d] = int(n64[d] + (a == d ? 1 : 0));
    }
    for (int d = 0; d < 3; ++d) {
        g->n[d] = int(n64[d]);
        g->h[d] = in->spacing[d];
        g->o[d] = in->origin[d];
    }
    g->cells = int(cells);
    for (int d = 0; d < 3; ++d) {
        const double h = g->h[d];
        g->rh[d] = (h > 0x1p-500 && h < 0x1p500) ? 1.0 / h : 0.0;
        const float hf = float(h);
        g->rhf[d] = (hf > 0x1p-60f && hf < 0x1p60f) ? 1.0f / hf : 0.0f;
        g->frow[d] = make_fastdiv(unsigned(g->fc[d][0]));
        g->fplane[d] = make_fastdiv(unsigned(g->fc[d][0]) * unsigned(g->fc[d][1]));
    }
    g->crow = make_fastdiv(unsigned(g->n[0]));
    g->cplane = make_fastdiv(unsigned(g->n[0]) * unsigned(g->n[1]));
    // Whether every cell and face centre o + (p + s) h (s = 0 or 1/2) and its
    // distance from the origin are exact, so that the sampler's scaled
    // coordinate there is exactly p + s and its fractions exactly 0 or 1/2
    // (with or without a fused multiply-add): the advection then forms the
    // velocity at a face centre from the nonzero corners alone, with the same
    // bits.
    g->exact_centres = 1;
    for (int d = 0; d < 3 && g->exact_centres; ++d) {
        if (n64[d] > (1u << 16)) {
            g->exact_centres = 0;
            break;
        }
        for (uint64_t p = 0; p <= n64[d] && g->exact_centres; ++p)
            for (double s : {0.0, 0.5}) {
                const double q = double(p) + s;
                const double prod = q * g->h[d];
                const double pos = g->o[d] + prod;
                if (std::fma(q, g->h[d], -prod) != 0.0 || pos - g->o[d] != prod || pos - prod != g->o[d] ||
                    prod / g->h[d] != q) {
                    g->exact_centres = 0;
                    break;
                }
            }
    }
    g->volume = g->h[0] * g->h[1] * g->h[2];
    if (!std::isfinite(g->volume) || g->volume <= 0.0) return RB200_INVALID_ARGUMENT;
    for (int d = 0; d < 3; ++d) {
        double n = double(g->n[d]);
        double extent = n * g->h[d];
        g->up[d] = g->o[d] + extent;
        double scale = std::fmax(std::fmax(std::fabs(g->o[d]), std::fabs(g->up[d])), extent);
        if (!std::isfinite(extent) || !std::isfinite(scale) || !std::isnormal(0.5 * g->h[d]) ||
            g->h[d] / scale < 32.0 * eps)
            return RB200_INVALID_ARGUMENT;
        double first = g->o[d] + 0.5 * g->h[d];
        double last = g->o[d] + (n - 0.5) * g->h[d];
        if (!std::isfinite(g->up[d]) || g->up[d] <= g->o[d] || first <= g->o[d] ||
            last >= g->up[d])
            return RB200_INVALID_ARGUMENT;
    }
    if (!std::isfinite(density) || density <= 0.0) return RB200_INVALID_ARGUMENT;
    g->area[0] = g->h[1] * g->h[2];
    g->area[1] = g->h[0] * g->h[2];
    g->area[2] = g->h[0] * g->h[1];
    for (int d = 0; d < 3; ++d) {
        g->accel[d] = 1.0 / (density * g->h[d]);
        g->weight[d] = g->area[d] * g->accel[d];
        if (!std::isfinite(g->area[d]) || g->area[d] <= 0.0 || !std::isfinite(g->accel[d]) ||
            g->accel[d] <= 0.0 || !std::isfinite(g->weight[d]) || g->weight[d] <= 0.0)
            return RB200_INVALID_ARGUMENT;
    }
    for (int mask = 0; mask < 64; ++mask) {
        double v = 0.0;
        for (int side = 0; side < 6; ++side)
            if (mask & (1 << side)) v += g->weight[side / 2];
        g->diag[mask] = v;
        g->rdiag[mask] = (v > 0x1p-500 && v < 0x1p500) ? 1.0 / v : 0.0;
    }
    return RB200_OK;
}

inline bool same_grid(const rb200_grid& a, const rb200_grid& b) {
    for (int d = 0; d < 3; ++d)
        if (a.counts[d] != b.counts[d] || a.spacing[d] != b.spacing[d] || a.origin[d] != b.origin[d])
            return false;
    return true;
}

inline bool settings_valid(const rb200_settings* s) {
    if (!s) return false;
    const double v[3] = {s->relative_residual, s->absolute_residual, s->divergence_limit};
    for (double x : v)
        if (!std::isfinite(x) || x < 0.0) return false;
    return true;
}

// Device-side validation flags written by the operator/advection kernels.
enum : int {
    VF_NONFINITE = 1,
    VF_WALL = 2,
    VF_ARITH = 4,
    VF_F32_RANGE = 8,
};

// ---------------------------------------------------------------- operator.cu
int launch_apply_full(const GridDev& g, const double* p, double* out, int* flags, cudaStream_t s);
// z = r/D (z[0] = 0) and r.z into *rz_out (device), with `part` holding
// precondition_partials_blocks() blocks of partials and a zeroed ticket.
int launch_precondition_jacobi(const GridDev& g, const double* r, double* z, Partials part, double* rz_out,
                               cudaStream_t s);
int precondition_partials_blocks();
// Qualification sums of a candidate pressure into out[5] (device), `part` as
// for launch_precondition_jacobi.
int launch_qualify_pressure(const GridDev& g, const double* b, const double* p, Partials part, double* out,
                            cudaStream_t s);
template <class T>
int launch_projection_witness(const GridDev& g, const double* p, double dt, const T* const in[3],
                              const T* const sup[3], unsigned long long* first, cudaStream_t s);
template <class T>
int launch_validate_faces(const GridDev& g, const T* u, const T* v, const T* w, int* flags,
                          cudaStream_t s);
template <class T>
int launch_build_rhs(const GridDev& g, const T* u, const T* v, const T* w, double dt, double* out,
                     int* flags, cudaStream_t s);
template <class T>
int launch_divergence(const GridDev& g, const T* u, const T* v, const T* w, double* out,
                      int* flags, cudaStream_t s);
template <class T>
int launch_correct(const GridDev& g, const double* p, double dt, T* u, T* v, T* w, int* flags,
                   cudaStream_t s);

// Fused projection epilogue of the resident step: corrected faces are written
// out of place, and the per-cell actual divergence max and per-axis face
// maxima (for velocity_rate) are reduced. Results land in out_scalars[0..3]:
// {divergence_max, max|u|, max|v|, max|w|}.
template <class T>
int launch_correct_divergence(const GridDev& g, const double* p, double dt, const T* const in[3],
                              T* const out[3], Partials part, int nblocks_cap,
                              double* out_scalars, int* flags, cudaStream_t s);
// Per-axis max |u_d| and finiteness of a face state: out_scalars[0..2].
template <class T>
int launch_face_maxima(const GridDev& g, const T* u, const T* v, const T* w, Partials part,
                       int nblocks_cap, double* out_scalars, int* flags, cudaStream_t s);
int partials_blocks_needed(const GridDev& g);

// --------------------------------------------------------------- advection.cu
// buoyancy: if tracer != nullptr and gb != 0, interior Y faces get
// v <- T(f64(v) + dt*(gb*0.5*(c_below + c_above))) after advection.
// fp32_math: sample and backtrace in FP32 arithmetic (mixed-precision path);
// otherwise FP64 arithmetic, as the reference.
template <class T>
int launch_advect_velocity(const GridDev& g, const T* u, const T* v, const T* w, double dt,
                           T* ou, T* ov, T* ow, const float* tracer, double gb, int* flags,
                           cudaStream_t s, bool fp32_math = false);
template <class T>
int launch_advect_tracer(const GridDev& g, const float* old, const T* u, const T* v, const T* w,
                         double dt, float* out, int* flags, cudaStream_t s, bool fp32_math = false);

}  // namespace rb200
