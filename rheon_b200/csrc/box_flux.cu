// Box-flux projection on the device: BoxFluxWorkspace (src/box_flux.rs).
//
// A projection is three device steps on the workspace's stream:
//   k_bf_rhs      one thread per cell: checks every provisional sample, takes
//                 the prescribed side components in place of the outer samples
//                 and writes b = flux/dt straight into the pressure solver's
//                 right-hand side (src/box_flux.rs:263-290);
//   PcgSolver     the workspace's sealed-box pressure solve of that RHS
//                 (:291-296), with every method of the library;
//   k_bf_correct  one thread per cell: corrects the cell's three lower faces
//                 into the output (outer faces take the side components),
//                 recomputes its upper faces to form the stored field's
//                 divergence, and reduces the interior energy terms, the
//                 boundary and residual work and the divergence maximum in the
//                 same pass (:297-362).
// Every per-face and per-cell term is rounded exactly as the reference rounds
// it (the library is built without multiply-add contraction; quotients by the
// spacing and by dt are correctly rounded through div_diag). The reference
// adds the terms serially; the device adds each thread's few terms in double
// and combines the threads' partials in double-double, which is at least as
// accurate as the serial sum.
#include <algorithm>
#include <cmath>
#include <limits>
#include <memory>
#include <new>

#include "internal.hpp"
#include "pcg.hpp"
#include "project.cuh"

namespace rb200 {
namespace {

// Sums of k_bf_correct: kinetic_before, kinetic_after, correction_energy,
// correction_residual_work, boundary_pressure_work, divergence_residual_work.
constexpr int BF_SUMS = 6;
constexpr int BF_SCALARS = BF_SUMS + 1;  // + max |divergence|

struct BfConst {
    float side[3][2];    // PrescribedBoxFlux::component(d, upper) (:36-45)
    double q[3][2];      // area_d * f64(outward) of each side (:342-349)
    double dt;
    double rdt;          // RN(1/dt) for div_diag, or 0 where it may not be used
    double rh[3];        // RN(1/h_d) likewise
    double dt_factor[3]; // dt * (1 / (rho h_d)), the reference's left-to-right product
    double dt_area[3];   // dt * area_d
    double mass;         // rho * cell volume
    double half_mass;    // 0.5 * mass
    FastDiv div_x, div_xy; // cell -> (cell / n0, cell / (n0 n1))
};

__device__ __forceinline__ int face_stride(const GridDev& g, int a) {
    return a == 0 ? 1 : (a == 1 ? g.fc[1][0] : g.fc[2][0] * g.fc[2][1]);
}

// (i, j, k) of a cell without hardware division.
__device__ __forceinline__ void cell_ijk(const GridDev& g, const BfConst& c, int cell, int (&ijk)[3]) {
    const int row = fast_div(cell, c.div_x);
    ijk[2] = fast_div(cell, c.div_xy);
    ijk[0] = cell - row * g.n[0];
    ijk[1] = row - ijk[2] * g.n[1];
}

// validate(old) (:397-404) and the imposed RHS (:263-290). Each face is the
// lower face of one cell or an upper outer face, so every sample is checked once.
__global__ void __launch_bounds__(EW_THREADS) k_bf_rhs(GridDev g, BfConst c, const float* __restrict__ u,
                                                       const float* __restrict__ v, const float* __restrict__ w,
                                                       double* __restrict__ out, int* flags) {
    const float* f3[3] = {u, v, w};
    int local = 0;
    for (int cell = blockIdx.x * blockDim.x + threadIdx.x; cell < g.cells; cell += gridDim.x * blockDim.x) {
        int ijk[3];
        cell_ijk(g, c, cell, ijk);
        double flux = 0.0;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const int flo = face_idx(g, a, ijk[0], ijk[1], ijk[2]);
            const int fhi = flo + face_stride(g, a);
            float lo = f3[a][flo];
            if (!isfinite(lo)) local |= VF_NONFINITE;
            if (ijk[a] == 0) lo = c.side[a][0];
            float hi = f3[a][fhi];
            if (ijk[a] + 1 == g.n[a]) {
                if (!isfinite(hi)) local |= VF_NONFINITE;
                hi = c.side[a][1];
            }
            flux += g.area[a] * (double(lo) - double(hi));
        }
        const double r = div_diag(flux, c.dt, c.rdt);
        if (!isfinite(r)) local |= VF_ARITH;
        out[cell] = r;
    }
    if (local) atomicOr(flags, local);
}

// Correction, stored-field divergence and the work terms (:297-362).
__global__ void __launch_bounds__(EW_THREADS, 4) k_bf_correct(GridDev g, BfConst c, const double* __restrict__ p,
                                                           const float* __restrict__ iu, const float* __restrict__ iv,
                                                           const float* __restrict__ iw, float* __restrict__ ou,
                                                           float* __restrict__ ov, float* __restrict__ ow,
                                                           Partials part, double* out_scalars, int* flags) {
    __shared__ BlockReduce<BF_SUMS, 1> sm;
    const float* in[3] = {iu, iv, iw};
    float* out[3] = {ou, ov, ow};
    const int s[3] = {1, g.n[0], g.n[0] * g.n[1]};
    // Each thread adds its own few terms in plain double (a handful of cells
    // per thread: an error of a few ulps of its partial's magnitude sum);
    // the partials are combined in double-double.
    double acc[BF_SUMS];
#pragma unroll
    for (int q = 0; q < BF_SUMS; ++q) acc[q] = 0.0;
    double mx[1] = {0.0};
    int local = 0;
    for (int cell = blockIdx.x * blockDim.x + threadIdx.x; cell < g.cells; cell += gridDim.x * blockDim.x) {
        int ijk[3];
        cell_ijk(g, c, cell, ijk);
        // gather first (every load unconditional, at an in-range index), so
        // that all of a cell's loads are in flight together
        const double pc = p[cell];
        double pl[3], pu[3];
        float fl[3], fh[3];
        int flo[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            flo[a] = face_idx(g, a, ijk[0], ijk[1], ijk[2]);
            pl[a] = p[ijk[a] > 0 ? cell - s[a] : cell];
            pu[a] = p[ijk[a] + 1 < g.n[a] ? cell + s[a] : cell];
            fl[a] = in[a][flo[a]];
            fh[a] = in[a][flo[a] + face_stride(g, a)];
        }
        double lo[3], hi[3];
        double q = 0.0;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            float vlo;
            if (ijk[a] == 0) {
                vlo = c.side[a][0];
            } else {
                const double difference = pc - pl[a];
                const double uo = double(fl[a]);
                const double value = uo - c.dt_factor[a] * difference;
                if (!isfinite(value) || fabs(value) > double(kF32Max)) local |= VF_ARITH;
                vlo = float(value);
                const double vv = double(vlo);
                const double delta = vv - uo;
                acc[0] += c.half_mass * uo * uo;
                acc[1] += c.half_mass * vv * vv;
                acc[2] += c.half_mass * delta * delta;
                acc[3] += (c.mass * delta + c.dt_area[a] * difference) * vv;
            }
            out[a][flo[a]] = vlo;
            float vhi;
            if (ijk[a] + 1 == g.n[a]) {
                vhi = c.side[a][1];
                out[a][flo[a] + face_stride(g, a)] = vhi;
            } else {
                // the upper neighbour's own corrected value, recomputed
                vhi = float(double(fh[a]) - c.dt_factor[a] * (pu[a] - pc));
            }
            lo[a] = double(vlo);
            hi[a] = double(vhi);
            if (ijk[a] == 0) q += c.q[a][0];
            if (ijk[a] + 1 == g.n[a]) q += c.q[a][1];
        }
        // divergence() (:405-434): value = 0; value += (hi - lo)/h_d
        double value = 0.0;
        value += div_diag(hi[0] - lo[0], g.h[0], c.rh[0]);
        value += div_diag(hi[1] - lo[1], g.h[1], c.rh[1]);
        value += div_diag(hi[2] - lo[2], g.h[2], c.rh[2]);
        if (!isfinite(value)) local |= VF_ARITH;
        mx[0] = fmax(mx[0], fabs(value));
        const double dtp = c.dt * pc;
        acc[4] -= dtp * q;
        acc[5] += dtp * g.volume * value;
    }
    if (local) atomicOr(flags, local);
    dd sums[BF_SUMS];
#pragma unroll
    for (int q = 0; q < BF_SUMS; ++q) sums[q] = dd{acc[q], 0.0};
    block_reduce<BF_SUMS, 1>(sm, sums, mx);
    if (publish_and_check_last<BF_SUMS, 1>(part, blockIdx.x, gridDim.x, sums, mx)) {
        fold_partials<BF_SUMS, 1>(part, gridDim.x, sm, sums, mx);
        if (threadIdx.x == 0) {
#pragma unroll
            for (int q = 0; q < BF_SUMS; ++q) out_scalars[q] = dd_value(sums[q]);
            out_scalars[BF_SUMS] = mx[0];
        }
    }
}

// BoxFluxWorkspace::divergence (:201-206): validate, then divergence().
__global__ void __launch_bounds__(EW_THREADS) k_bf_divergence(GridDev g, BfConst c, const float* __restrict__ u,
                                                              const float* __restrict__ v,
                                                              const float* __restrict__ w, double* __restrict__ out,
                                                              int* flags) {
    const float* f3[3] = {u, v, w};
    int local = 0;
    for (int cell = blockIdx.x * blockDim.x + threadIdx.x; cell < g.cells; cell += gridDim.x * blockDim.x) {
        int ijk[3];
        cell_ijk(g, c, cell, ijk);
        double value = 0.0;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const int flo = face_idx(g, a, ijk[0], ijk[1], ijk[2]);
            const float lo = f3[a][flo], hi = f3[a][flo + face_stride(g, a)];
            if (!isfinite(lo) || (ijk[a] + 1 == g.n[a] && !isfinite(hi))) local |= VF_NONFINITE;
            value += div_diag(double(hi) - double(lo), g.h[a], c.rh[a]);
        }
        if (!isfinite(value)) local |= VF_ARITH;
        out[cell] = value;
    }
    if (local) atomicOr(flags, local);
}

__global__ void __launch_bounds__(EW_THREADS) k_bf_finite(const float* __restrict__ x, int n, int* flags) {
    int local = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (!isfinite(x[i])) local = VF_NONFINITE;
    if (local) atomicOr(flags, local);
}

int bf_blocks(long long n) {
    long long b = (n + EW_THREADS - 1) / EW_THREADS;
    if (b < 1) b = 1;
    return int(b < EW_BLOCKS_CAP ? b : EW_BLOCKS_CAP);
}

// compensated (:444-459): Neumaier summation of the six side terms.
double compensated(const double* v, int n) {
    double sum = 0.0, correction = 0.0;
    for (int i = 0; i < n; ++i) {
        const double next = sum + v[i];
        correction += std::fabs(sum) >= std::fabs(v[i]) ? (sum - next) + v[i] : (v[i] - next) + sum;
        sum = next;
    }
    return sum + correction;
}

float side_component(const float outward[6], int d, bool upper) {
    const float speed = outward[2 * d + (upper ? 1 : 0)];
    if (speed == 0.0f) return 0.0f;
    return upper ? speed : -speed;
}

struct CancelAdapter {
    rb200_box_flux_cancel_fn fn;
    void* ctx;
};

int pressure_cancel(void* a) {
    auto* c = static_cast<CancelAdapter*>(a);
    return c->fn(c->ctx, RB200_BOX_FLUX_PRESSURE_ITERATION);
}

int reject(rb200_box_flux_report* r, int error) {
    r->error = error;
    return RB200_BOX_FLUX_REJECTED;
}

}  // namespace
}  // namespace rb200

using namespace rb200;

struct rb200_box_flux {
    int device = 0;
    cudaStream_t stream = nullptr;
    GridDev g{};
    rb200_grid grid{};
    double density = 0.0;
    int method = 0;
    double mass = 0.0;
    double side_area[3] = {0.0, 0.0, 0.0};
    uint64_t accounted = 0;
    PcgSolver solver;
    int nb = 0;      // blocks of k_bf_correct: one wave of resident blocks at most
    int nb_rhs = 0;  // blocks of k_bf_rhs and k_bf_divergence, likewise
    // device: flags (int), scalars [BF_SCALARS], partials [nb][2*BF_SUMS+1], ticket
    char* d_buf = nullptr;
    int* d_flags = nullptr;
    double* d_scalars = nullptr;
    Partials part{};
    // pinned mirror of flags and scalars
    char* h_buf = nullptr;
    // host-call staging: old u, v, w then output u, v, w
    float* staging = nullptr;
    float* stage[6] = {};
    // the last correction's launch, for rb200_box_flux_profile
    BfConst last{};
    const float* last_in[3] = {};
    float* last_out[3] = {};
    bool has_last = false;
    // events around the RHS pass (0, 1) and the correction pass (2, 3) of the
    // last projection that reached them
    cudaEvent_t ev[4] = {};
    bool timed_rhs = false, timed_correct = false;

    ~rb200_box_flux() {
        if (stream) {
            cudaSetDevice(device);
            cudaStreamSynchronize(stream);
            cudaStreamDestroy(stream);
        }
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
        cudaFree(d_buf);
        cudaFree(staging);
        cudaFreeHost(h_buf);
    }
    int* h_flags() { return reinterpret_cast<int*>(h_buf); }
    double* h_scalars() { return reinterpret_cast<double*>(h_buf + 16); }
};

namespace {

// RN(1/x) where div_diag may use it (2^-500 < x < 2^500), else 0 (divide).
double recip_for_div(double x) { return (x > 0x1p-500 && x < 0x1p500) ? 1.0 / x : 0.0; }

BfConst make_const(const rb200_box_flux* B, const float outward[6], double dt) {
    const GridDev& g = B->g;
    BfConst c;
    for (int d = 0; d < 3; ++d) {
        for (int s = 0; s < 2; ++s) {
            c.side[d][s] = side_component(outward, d, s == 1);
            c.q[d][s] = g.area[d] * double(outward[2 * d + s]);
        }
        c.dt_factor[d] = dt * g.accel[d];
        c.dt_area[d] = dt * g.area[d];
    }
    c.dt = dt;
    c.rdt = recip_for_div(dt);
    for (int d = 0; d < 3; ++d) c.rh[d] = recip_for_div(g.h[d]);
    c.mass = B->mass;
    c.half_mass = 0.5 * B->mass;
    c.div_x = make_fastdiv(unsigned(g.n[0]));
    c.div_xy = make_fastdiv(unsigned(g.n[0]) * unsigned(g.n[1]));
    return c;
}

// Reads the flags word (and, when `scalars`, the correction's scalars) after
// the stream's work so far.
int read_back(rb200_box_flux* B, bool scalars, int* flags) {
    RB200_CUDA(cudaMemcpyAsync(B->h_buf, B->d_buf, scalars ? 16 + BF_SCALARS * sizeof(double) : sizeof(int),
                               cudaMemcpyDeviceToHost, B->stream));
    RB200_CUDA(cudaStreamSynchronize(B->stream));
    *flags = *B->h_flags();
    return RB200_OK;
}

int finite_prefix(rb200_box_flux* B, const float* const old[3], int axes, bool host) {
    for (int a = 0; a < axes; ++a) {
        const int n = B->g.flen[a];
        if (host) {
            for (int i = 0; i < n; ++i)
                if (!std::isfinite(old[a][i])) return RB200_NONFINITE_INPUT;
            continue;
        }
        RB200_CUDA(cudaMemsetAsync(B->d_flags, 0, sizeof(int), B->stream));
        k_bf_finite<<<bf_blocks(n), EW_THREADS, 0, B->stream>>>(old[a], n, B->d_flags);
        RB200_CUDA(cudaGetLastError());
        int f = 0;
        int rc = read_back(B, false, &f);
        if (rc) return rc;
        if (f & VF_NONFINITE) return RB200_NONFINITE_INPUT;
    }
    return RB200_OK;
}

int ensure_staging(rb200_box_flux* B) {
    if (B->staging) return RB200_OK;
    size_t total = 0;
    for (int a = 0; a < 3; ++a) total += 2 * size_t(B->g.flen[a]);
    RB200_CUDA(cudaMalloc(&B->staging, total * sizeof(float)));
    float* at = B->staging;
    for (int k = 0; k < 6; ++k) {
        B->stage[k] = at;
        at += B->g.flen[k % 3];
    }
    return RB200_OK;
}

int project_impl(rb200_box_flux* B, const float* const old[3], const size_t old_len[3], double dt,
                 const rb200_box_flux_boundary* bc, const rb200_settings* settings, double limit,
                 float* const out[3], const size_t out_len[3], rb200_box_flux_report* rep,
                 rb200_box_flux_cancel_fn cancelled, void* ctx, bool host) {
    if (!B || !old || !old_len || !bc || !settings || !out || !out_len || !rep) return RB200_INVALID_ARGUMENT;
    std::memset(rep, 0, sizeof(*rep));
    rep->boundary_id = bc->id;
    rep->boundary_version = bc->version;
    for (int a = 0; a < 3; ++a)
        if (!old[a] || !out[a]) return RB200_INVALID_ARGUMENT;
    // PrescribedBoxFlux::new (:23-28)
    for (int i = 0; i < 6; ++i)
        if (!std::isfinite(bc->outward[i])) return reject(rep, RB200_BOX_FLUX_INVALID_BOUNDARY);
    cudaSetDevice(B->device);
    const GridDev& g = B->g;
    // project (:213-262)
    if (!std::isfinite(dt) || dt <= 0.0) return RB200_INVALID_ARGUMENT;  // OperatorError::InvalidTimeStep
    if (!std::isfinite(limit) || limit < 0.0) return reject(rep, RB200_BOX_FLUX_INVALID_SETTINGS);
    for (int a = 0; a < 3; ++a)
        if (old_len[a] != size_t(g.flen[a])) {
            // validate() checks each axis' values before the next axis' length
            int rc = finite_prefix(B, old, a, host);
            return rc ? rc : RB200_LENGTH_MISMATCH;
        }
    const float* src[3] = {old[0], old[1], old[2]};
    float* dst[3] = {out[0], out[1], out[2]};
    if (host) {
        int rc = ensure_staging(B);
        if (rc) return rc;
        for (int a = 0; a < 3; ++a) {
            RB200_CUDA(cudaMemcpyAsync(B->stage[a], old[a], old_len[a] * sizeof(float), cudaMemcpyHostToDevice,
                                       B->stream));
            src[a] = B->stage[a];
            dst[a] = B->stage[3 + a];
        }
    }
    const BfConst c = make_const(B, bc->outward, dt);
    RB200_CUDA(cudaMemsetAsync(B->d_flags, 0, sizeof(int), B->stream));
    RB200_CUDA(cudaEventRecord(B->ev[0], B->stream));
    k_bf_rhs<<<B->nb_rhs, EW_THREADS, 0, B->stream>>>(g, c, src[0], src[1], src[2], B->solver.b(), B->d_flags);
    RB200_CUDA(cudaGetLastError());
    RB200_CUDA(cudaEventRecord(B->ev[1], B->stream));
    B->timed_rhs = true;
    B->timed_correct = false;
    int flags = 0;
    int rc = read_back(B, false, &flags);
    if (rc) return rc;
    if (flags & VF_NONFINITE) return RB200_NONFINITE_INPUT;
    for (int a = 0; a < 3; ++a)
        if (out_len[a] != size_t(g.flen[a])) return RB200_LENGTH_MISMATCH;
    // the compatibility gate (:238-262)
    double terms[6], absolute_terms[6];
    for (int i = 0; i < 6; ++i) {
        terms[i] = B->side_area[i / 2] * double(bc->outward[i]);
        if (terms[i] == 0.0 && bc->outward[i] != 0.0f) return reject(rep, RB200_BOX_FLUX_ARITHMETIC_FAILURE);
        absolute_terms[i] = std::fabs(terms[i]);
    }
    const double net = compensated(terms, 6), absolute = compensated(absolute_terms, 6);
    const double budget = 64.0 * std::numeric_limits<double>::epsilon() * absolute;
    rep->net_outward_flux = net;
    rep->flux_rounding_budget = budget;
    if (!std::isfinite(net) || !std::isfinite(absolute)) return reject(rep, RB200_BOX_FLUX_ARITHMETIC_FAILURE);
    if (std::fabs(net) > budget) {
        rep->error_actual = net;
        rep->error_limit = budget;
        return reject(rep, RB200_BOX_FLUX_INCOMPATIBLE_FLUX);
    }
    if (cancelled && cancelled(ctx, RB200_BOX_FLUX_BEFORE_SOLVE)) {
        rep->stage = RB200_BOX_FLUX_BEFORE_SOLVE;
        return reject(rep, RB200_BOX_FLUX_CANCELLED);
    }
    if (flags & VF_ARITH) return reject(rep, RB200_BOX_FLUX_ARITHMETIC_FAILURE);
    // the pressure solve (:291-296)
    if (!settings_valid(settings)) return RB200_INVALID_ARGUMENT;  // PressureError::InvalidSettings
    CancelAdapter adapter{cancelled, ctx};
    rc = B->solver.solve(dt, *settings, &rep->pressure, cancelled ? pressure_cancel : nullptr, &adapter);
    if (rc) return rc;
    // correction, divergence and work (:297-362)
    if (cancelled && cancelled(ctx, RB200_BOX_FLUX_CORRECTION_SLICE)) {
        rep->stage = RB200_BOX_FLUX_CORRECTION_SLICE;
        return reject(rep, RB200_BOX_FLUX_CANCELLED);
    }
    RB200_CUDA(cudaMemsetAsync(B->d_flags, 0, sizeof(int), B->stream));
    RB200_CUDA(cudaEventRecord(B->ev[2], B->stream));
    k_bf_correct<<<B->nb, EW_THREADS, 0, B->stream>>>(g, c, B->solver.p(), src[0], src[1], src[2], dst[0], dst[1],
                                                      dst[2], B->part, B->d_scalars, B->d_flags);
    RB200_CUDA(cudaGetLastError());
    RB200_CUDA(cudaEventRecord(B->ev[3], B->stream));
    B->timed_correct = true;
    B->last = c;
    for (int a = 0; a < 3; ++a) {
        B->last_in[a] = src[a];
        B->last_out[a] = dst[a];
    }
    B->has_last = true;
    bool cancel_late = false;
    const long long slices = 3ll * g.n[2] + 1;
    for (long long t = 1; t < slices && cancelled && !cancel_late; ++t)
        cancel_late = cancelled(ctx, RB200_BOX_FLUX_CORRECTION_SLICE) != 0;
    if (host)
        for (int a = 0; a < 3; ++a)
            RB200_CUDA(cudaMemcpyAsync(out[a], dst[a], out_len[a] * sizeof(float), cudaMemcpyDeviceToHost,
                                       B->stream));
    if ((rc = read_back(B, true, &flags))) return rc;
    if (cancel_late) {
        rep->stage = RB200_BOX_FLUX_CORRECTION_SLICE;
        return reject(rep, RB200_BOX_FLUX_CANCELLED);
    }
    if (flags & VF_ARITH) return reject(rep, RB200_BOX_FLUX_ARITHMETIC_FAILURE);
    const double* sc = B->h_scalars();
    const double actual = sc[BF_SUMS];
    rep->actual_divergence_max = actual;
    if (actual > limit) {
        rep->error_actual = actual;
        rep->error_limit = limit;
        return reject(rep, RB200_BOX_FLUX_DIVERGENCE_LIMIT);
    }
    rep->kinetic_before = sc[0];
    rep->kinetic_after = sc[1];
    rep->correction_energy = sc[2];
    rep->correction_residual_work = sc[3];
    rep->boundary_pressure_work = sc[4];
    rep->divergence_residual_work = sc[5];
    rep->budget_error = rep->kinetic_after - rep->kinetic_before + rep->correction_energy -
                        (rep->boundary_pressure_work + rep->divergence_residual_work + rep->correction_residual_work);
    const double work[7] = {rep->kinetic_before,           rep->kinetic_after,
                            rep->correction_energy,        rep->boundary_pressure_work,
                            rep->divergence_residual_work, rep->correction_residual_work,
                            rep->budget_error};
    for (double x : work)
        if (!std::isfinite(x)) return reject(rep, RB200_BOX_FLUX_ARITHMETIC_FAILURE);
    if (cancelled && cancelled(ctx, RB200_BOX_FLUX_BEFORE_ACCEPTANCE)) {
        rep->stage = RB200_BOX_FLUX_BEFORE_ACCEPTANCE;
        return reject(rep, RB200_BOX_FLUX_CANCELLED);
    }
    return RB200_OK;
}

}  // namespace

namespace rb200 {
bool box_flux_matches(const rb200_box_flux* B, const rb200_grid& grid, double density, int method) {
    if (!B || B->method != method) return false;
    uint64_t a, b;
    std::memcpy(&a, &B->density, 8);
    std::memcpy(&b, &density, 8);
    return a == b && same_grid(B->grid, grid);
}
}  // namespace rb200

extern "C" {

int rb200_box_flux_create(const rb200_grid* grid, double density, uint64_t limit, int method, int device,
                          rb200_box_flux** out, rb200_box_flux_report* error) {
    if (!grid || !out) return RB200_INVALID_ARGUMENT;
    *out = nullptr;
    rb200_box_flux_report scratch;
    rb200_box_flux_report* rep = error ? error : &scratch;
    std::memset(rep, 0, sizeof(*rep));
    GridDev g;
    int rc = make_grid_dev(grid, density, &g);  // PressureOperator::new
    if (rc) return rc;
    if (method < RB200_JACOBI_PCG_V1 || method > RB200_MG_MIXED) return RB200_UNSUPPORTED;
    // BoxFluxWorkspace::new (:132-186)
    double side_area[3];
    for (int d = 0; d < 3; ++d)
        side_area[d] = g.area[d] * double(g.n[(d + 1) % 3]) * double(g.n[(d + 2) % 3]);
    const double mass = density * g.volume;
    if (!std::isfinite(mass) || mass <= 0.0) return reject(rep, RB200_BOX_FLUX_INVALID_MASS);
    for (double a : side_area)
        if (!std::isfinite(a) || a <= 0.0) return reject(rep, RB200_BOX_FLUX_ARITHMETIC_FAILURE);
    const uint64_t cells = uint64_t(g.cells);
    const uint64_t required = cells * 56;
    if (required > limit) {
        rep->required = required;
        rep->limit = limit;
        return reject(rep, RB200_BOX_FLUX_BUFFER_LIMIT);
    }
    // the pressure workspace gets what the f64 cell array leaves
    // (PressureWorkspace::with_implementation): 48 bytes per cell, 62 for multigrid
    const uint64_t remaining = limit - cells * 8;
    if (cells * (method == RB200_MG_MIXED ? 62 : 48) > remaining) return RB200_OUT_OF_MEMORY;
    if ((rc = select_device(device))) return rc;
    std::unique_ptr<rb200_box_flux> B(new (std::nothrow) rb200_box_flux());
    if (!B) return RB200_OUT_OF_MEMORY;
    B->device = device;
    B->g = g;
    B->grid = *grid;
    B->density = density;
    B->method = method;
    B->mass = mass;
    for (int d = 0; d < 3; ++d) B->side_area[d] = side_area[d];
    B->accounted = required;
    RB200_CUDA(cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking));
    if ((rc = B->solver.init(g, method, B->stream))) return rc;
    int sms = 0, occ_correct = 0, occ_rhs = 0;
    RB200_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    RB200_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_correct, k_bf_correct, EW_THREADS, 0));
    RB200_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_rhs, k_bf_rhs, EW_THREADS, 0));
    B->nb = std::min(bf_blocks(g.cells), std::max(1, sms * occ_correct));
    B->nb_rhs = std::min(bf_blocks(g.cells), std::max(1, sms * occ_rhs));
    const size_t part_doubles = size_t(B->nb) * (2 * BF_SUMS + 1);
    const size_t bytes = 16 + BF_SCALARS * sizeof(double) + part_doubles * sizeof(double) + 16;
    RB200_CUDA(cudaMalloc(&B->d_buf, bytes));
    RB200_CUDA(cudaMemset(B->d_buf, 0, bytes));
    RB200_CUDA(cudaMallocHost(&B->h_buf, 16 + BF_SCALARS * sizeof(double)));
    for (auto& e : B->ev) RB200_CUDA(cudaEventCreate(&e));
    B->d_flags = reinterpret_cast<int*>(B->d_buf);
    B->d_scalars = reinterpret_cast<double*>(B->d_buf + 16);
    B->part.data = B->d_scalars + BF_SCALARS;
    B->part.ticket = reinterpret_cast<unsigned*>(B->part.data + part_doubles);
    *out = B.release();
    return RB200_OK;
}

void rb200_box_flux_destroy(rb200_box_flux* B) { delete B; }

// BoxFluxWorkspace::allocated_bytes: the reference's accounting (56 bytes per
// cell); the device holds the pressure solver's arrays (its RHS array doubles
// as the f64 cell array), the reduction partials and, after a host call, the
// staging faces.
uint64_t rb200_box_flux_allocated_bytes(const rb200_box_flux* B) { return B ? B->accounted : 0; }

void* rb200_box_flux_stream(rb200_box_flux* B) { return B ? (void*)B->stream : nullptr; }

int rb200_box_flux_project_device(rb200_box_flux* B, const float* const old[3], const size_t old_len[3], double dt,
                                  const rb200_box_flux_boundary* boundary, const rb200_settings* pressure_settings,
                                  double actual_divergence_limit, float* const out[3], const size_t out_len[3],
                                  rb200_box_flux_report* report, rb200_box_flux_cancel_fn cancelled, void* ctx) {
    return project_impl(B, old, old_len, dt, boundary, pressure_settings, actual_divergence_limit, out, out_len,
                        report, cancelled, ctx, false);
}

int rb200_box_flux_project(rb200_box_flux* B, const float* const old[3], const size_t old_len[3], double dt,
                           const rb200_box_flux_boundary* boundary, const rb200_settings* pressure_settings,
                           double actual_divergence_limit, float* const out[3], const size_t out_len[3],
                           rb200_box_flux_report* report, rb200_box_flux_cancel_fn cancelled, void* ctx) {
    return project_impl(B, old, old_len, dt, boundary, pressure_settings, actual_divergence_limit, out, out_len,
                        report, cancelled, ctx, true);
}

int rb200_box_flux_divergence_device(rb200_box_flux* B, const float* const faces[3], const size_t len[3],
                                     double* out, size_t out_len) {
    if (!B || !faces || !len || !out) return RB200_INVALID_ARGUMENT;
    for (int a = 0; a < 3; ++a)
        if (!faces[a]) return RB200_INVALID_ARGUMENT;
    cudaSetDevice(B->device);
    for (int a = 0; a < 3; ++a)
        if (len[a] != size_t(B->g.flen[a])) {
            int rc = finite_prefix(B, faces, a, false);
            return rc ? rc : RB200_LENGTH_MISMATCH;
        }
    if (out_len != size_t(B->g.cells)) {
        int rc = finite_prefix(B, faces, 3, false);
        return rc ? rc : RB200_LENGTH_MISMATCH;
    }
    RB200_CUDA(cudaMemsetAsync(B->d_flags, 0, sizeof(int), B->stream));
    const float zero[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    const BfConst c = make_const(B, zero, 1.0);
    k_bf_divergence<<<B->nb_rhs, EW_THREADS, 0, B->stream>>>(B->g, c, faces[0], faces[1], faces[2], out,
                                                            B->d_flags);
    RB200_CUDA(cudaGetLastError());
    int flags = 0;
    int rc = read_back(B, false, &flags);
    if (rc) return rc;
    if (flags & VF_NONFINITE) return RB200_NONFINITE_INPUT;
    if (flags & VF_ARITH) return RB200_BOX_FLUX_REJECTED;  // BoxFluxError::ArithmeticFailure
    return RB200_OK;
}

int rb200_box_flux_pressure(rb200_box_flux* B, double* out, size_t len) {
    if (!B || !out) return RB200_INVALID_ARGUMENT;
    if (len != size_t(B->g.cells)) return RB200_LENGTH_MISMATCH;
    cudaSetDevice(B->device);
    RB200_CUDA(cudaMemcpyAsync(out, B->solver.p(), len * sizeof(double), cudaMemcpyDefault, B->stream));
    RB200_CUDA(cudaStreamSynchronize(B->stream));
    return RB200_OK;
}

const double* rb200_box_flux_pressure_device(rb200_box_flux* B) { return B ? B->solver.p() : nullptr; }

// Device times (CUDA events on the workspace's stream) of the RHS pass and
// the correction pass inside the last projection that reached them; a pass
// that did not run reports -1.
int rb200_box_flux_last_pass_ms(rb200_box_flux* B, double* rhs_ms, double* correct_ms) {
    if (!B || !rhs_ms || !correct_ms) return RB200_INVALID_ARGUMENT;
    cudaSetDevice(B->device);
    *rhs_ms = *correct_ms = -1.0;
    float ms = 0.0f;
    if (B->timed_rhs) {
        RB200_CUDA(cudaEventSynchronize(B->ev[1]));
        RB200_CUDA(cudaEventElapsedTime(&ms, B->ev[0], B->ev[1]));
        *rhs_ms = ms;
    }
    if (B->timed_correct) {
        RB200_CUDA(cudaEventSynchronize(B->ev[3]));
        RB200_CUDA(cudaEventElapsedTime(&ms, B->ev[2], B->ev[3]));
        *correct_ms = ms;
    }
    return RB200_OK;
}

// Average device time of `launches` back-to-back launches of the last
// projection's RHS pass (which = 0) or correction pass (which = 1), CUDA
// events on the workspace's stream. Both passes are idempotent.
int rb200_box_flux_profile(rb200_box_flux* B, int which, int launches, double* avg_ms) {
    if (!B || !avg_ms || launches < 1 || (which != 0 && which != 1)) return RB200_INVALID_ARGUMENT;
    if (!B->has_last) return RB200_INVALID_ARGUMENT;
    cudaSetDevice(B->device);
    cudaEvent_t e0, e1;
    RB200_CUDA(cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return RB200_EXECUTION;
    }
    const BfConst& c = B->last;
    int rc = RB200_OK;
    cudaEventRecord(e0, B->stream);
    for (int i = 0; i < launches; ++i) {
        if (which == 0)
            k_bf_rhs<<<B->nb_rhs, EW_THREADS, 0, B->stream>>>(B->g, c, B->last_in[0], B->last_in[1], B->last_in[2],
                                                          B->solver.scratch(), B->d_flags);
        else
            k_bf_correct<<<B->nb, EW_THREADS, 0, B->stream>>>(B->g, c, B->solver.p(), B->last_in[0], B->last_in[1],
                                                              B->last_in[2], B->last_out[0], B->last_out[1],
                                                              B->last_out[2], B->part, B->d_scalars, B->d_flags);
    }
    cudaEventRecord(e1, B->stream);
    float ms = 0.0f;
    if (cudaGetLastError() != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
        cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess)
        rc = RB200_EXECUTION;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *avg_ms = double(ms) / launches;
    return rc;
}

}  // extern "C"
