// The step owner with its forcing and boundary domains on the resident
// carrier: Simulation::step / step_with_forces / step_with_box_flux
// (src/simulation.rs:393-581, prepare_impl :812-1403).
//
// Host-driven, on the carrier's stream, in the reference's stage order:
//   accepted-state statistics (velocity rate; interior energy and tracer
//   integral for the box-flux ledger) -> dt policy with the smoke and
//   body-force accelerations -> advection into the provisional buffer ->
//   smoke source's Y-face force (apply_force :1449-1472) -> body forces
//   (src/forces.rs:144-212, k_fs_forces: update, energies and work in one
//   pass) -> the sealed projection (validate + build_rhs, the carrier's
//   pressure solve, fused correction/divergence) or the box-flux projection
//   (rb200_box_flux_project_device) into the candidate buffer -> Courant gate
//   -> tracer advection -> smoke source's tracer (apply_source :1473-1496) ->
//   tracer range check -> [with an attached liquid state: the liquid-volume
//   transport through the candidate faces] -> commit (index rotation on the
//   device; the liquid state commits with the carrier).
// Cancellation is asked at the reference's stages; a slice stage is asked
// as often as the reference asks it (its first time before the device pass,
// the others while the pass runs). Nothing is published before the commit,
// so every error and cancellation leaves the accepted state untouched.
// Per-face and per-cell arithmetic is the reference's, rounding for
// rounding; its serial sums (energies, work, tracer integral) are summed per
// thread in double and combined in double-double.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <new>

#include "carrier.hpp"
#include "internal.hpp"
#include "project.cuh"

namespace rb200 {

struct ForcedScratch {
    int nb = 0;
    char* d_buf = nullptr;  // flags (16 B), scalars [FS_SCALARS], partials [nb][9], ticket
    int* d_flags = nullptr;
    double* d_scalars = nullptr;
    Partials part{};
    char* h_buf = nullptr;  // pinned mirror of flags and scalars
    rb200_body_force* d_forces = nullptr;
    size_t force_cap = 0;
};

void forced_scratch_free(ForcedScratch* s) {
    if (!s) return;
    cudaFree(s->d_buf);
    cudaFree(s->d_forces);
    if (s->h_buf) cudaFreeHost(s->h_buf);
    delete s;
}

namespace {

constexpr int FS_SCALARS = 8;
constexpr int FS_SLOT = 9;  // doubles per block: up to 3 double-double sums and 3 maxima

__device__ __forceinline__ void face_coords(const GridDev& g, int a, int f, int (&c)[3]) {
    const int row = f / g.fc[a][0];
    c[0] = f - row * g.fc[a][0];
    c[2] = row / g.fc[a][1];
    c[1] = row - c[2] * g.fc[a][1];
}

// face_position (src/geometry.rs:242-248): origin + (p + offset) * h, offset 0 on the face's own axis
__device__ __forceinline__ double face_pos(const GridDev& g, int a, const int (&c)[3], int d) {
    return g.o[d] + (double(c[d]) + (d == a ? 0.0 : 0.5)) * g.h[d];
}

__device__ __forceinline__ bool in_box(double x, double y, double z, const double* lower, const double* upper) {
    return x >= lower[0] && x < upper[0] && y >= lower[1] && y < upper[1] && z >= lower[2] && z < upper[2];
}

// All-face and interior-face sums of squares (forces.rs:153-161,
// box_flux_step.rs:118-149), per-axis max |u_d| (velocity_rate,
// simulation.rs:1415-1429) and finiteness of a face state. One grid-stride
// sweep per axis (the axis is a compile-time constant in each).
// out: {all, interior, max x, max y, max z}
__global__ void __launch_bounds__(EW_THREADS) k_fs_face_stats(GridDev g, const float* __restrict__ u,
                                                              const float* __restrict__ v,
                                                              const float* __restrict__ w, Partials part,
                                                              double* out, int* flags) {
    __shared__ BlockReduce<2, 3> sm;
    double all = 0.0, interior = 0.0;
    double mx[3] = {0.0, 0.0, 0.0};
    int local = 0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float* __restrict__ x3 = a == 0 ? u : (a == 1 ? v : w);
        const int n0 = g.fc[a][0], n1 = g.fc[a][1], na = g.n[a];
        for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < g.flen[a]; f += gridDim.x * blockDim.x) {
            const int row = f / n0;
            const int ca = a == 0 ? f - row * n0 : (a == 1 ? row % n1 : row / n1);
            const double x = double(x3[f]);
            if (!isfinite(x)) local |= VF_NONFINITE;
            const double sq = x * x;
            all += sq;
            if (ca > 0 && ca < na) interior += sq;
            mx[a] = fmax(mx[a], fabs(x));
        }
    }
    if (local) atomicOr(flags, local);
    dd sums[2] = {dd{all, 0.0}, dd{interior, 0.0}};
    block_reduce<2, 3>(sm, sums, mx);
    if (publish_and_check_last<2, 3>(part, blockIdx.x, gridDim.x, sums, mx)) {
        fold_partials<2, 3>(part, gridDim.x, sm, sums, mx);
        if (threadIdx.x == 0) {
            out[0] = dd_value(sums[0]);
            out[1] = dd_value(sums[1]);
            for (int q = 0; q < 3; ++q) out[2 + q] = mx[q];
        }
    }
}

// apply_force (src/simulation.rs:1449-1472): interior Y faces whose position
// lies in the source box get f32(f64(v) + dt * vertical_acceleration).
__global__ void __launch_bounds__(EW_THREADS) k_fs_smoke_force(GridDev g, float* __restrict__ y,
                                                               rb200_smoke_source s, double dt, int* flags) {
    int local = 0;
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < g.flen[1]; f += gridDim.x * blockDim.x) {
        int c[3];
        face_coords(g, 1, f, c);
        if (c[1] < 1 || c[1] >= g.n[1]) continue;
        if (!in_box(face_pos(g, 1, c, 0), face_pos(g, 1, c, 1), face_pos(g, 1, c, 2), s.lower, s.upper)) continue;
        const double value = double(y[f]) + dt * s.vertical_acceleration;
        if (!isfinite(value) || fabs(value) > double(kF32Max)) {
            local |= VF_ARITH;
            continue;
        }
        y[f] = float(value);
    }
    if (local) atomicOr(flags, local);
}

// forces::apply_evaluated (src/forces.rs:144-212) for constant vectors: each
// interior face adds dt times the sum of the accelerations of the forces
// whose support holds its position (in the caller's order); out: {sum of
// squares before, sum of squares after, work}. One grid-stride sweep per
// axis (the axis is a compile-time constant in each).
__global__ void __launch_bounds__(EW_THREADS) k_fs_forces(GridDev g, float* __restrict__ u, float* __restrict__ v,
                                                          float* __restrict__ w,
                                                          const rb200_body_force* __restrict__ forces, int nforces,
                                                          double density, double dt, double mass, Partials part,
                                                          double* out, int* flags) {
    __shared__ BlockReduce<3, 0> sm;
    double before = 0.0, after = 0.0, work = 0.0;
    int local = 0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float* __restrict__ x3 = a == 0 ? u : (a == 1 ? v : w);
        const int n0 = g.fc[a][0], n1 = g.fc[a][1], na = g.n[a];
        for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < g.flen[a]; f += gridDim.x * blockDim.x) {
            const int row = f / n0;
            const int i = f - row * n0, k = row / n1, j = row - k * n1;
            const int ca = a == 0 ? i : (a == 1 ? j : k);
            const double old = double(x3[f]);
            const double old_sq = old * old;
            before += old_sq;
            double new_sq = old_sq;
            if (ca > 0 && ca < na) {
                // face_position (src/geometry.rs:242-248)
                const double px = g.o[0] + (double(i) + (a == 0 ? 0.0 : 0.5)) * g.h[0];
                const double py = g.o[1] + (double(j) + (a == 1 ? 0.0 : 0.5)) * g.h[1];
                const double pz = g.o[2] + (double(k) + (a == 2 ? 0.0 : 0.5)) * g.h[2];
                double sum = 0.0;
                for (int q = 0; q < nforces; ++q) {
                    const rb200_body_force& F = forces[q];
                    if (F.has_region && !in_box(px, py, pz, F.lower, F.upper)) continue;
                    sum += F.units == RB200_FORCE_DENSITY ? F.value[a] / density : F.value[a];
                }
                const double updated = old + dt * sum;
                if (!isfinite(updated) || fabs(updated) > double(kF32Max)) {
                    local |= VF_ARITH;
                } else {
                    const float stored = float(updated);
                    const double nv = double(stored);
                    const double delta = nv - old;
                    work += mass * delta * (old + 0.5 * delta);
                    x3[f] = stored;
                    new_sq = nv * nv;
                }
            }
            after += new_sq;
        }
    }
    if (local) atomicOr(flags, local);
    dd sums[3] = {dd{before, 0.0}, dd{after, 0.0}, dd{work, 0.0}};
    double none[1];
    block_reduce<3, 0>(sm, sums, none);
    if (publish_and_check_last<3, 0>(part, blockIdx.x, gridDim.x, sums, none)) {
        fold_partials<3, 0>(part, gridDim.x, sm, sums, none);
        if (threadIdx.x == 0)
            for (int q = 0; q < 3; ++q) out[q] = dd_value(sums[q]);
    }
}

// apply_source (src/simulation.rs:1473-1496): cells whose centre lies in the
// source box get f32(min(f64(t) + dt * tracer_rate, 1)).
__global__ void __launch_bounds__(EW_THREADS) k_fs_smoke_source(GridDev g, float* __restrict__ tracer,
                                                                rb200_smoke_source s, double amount) {
    for (int cell = blockIdx.x * blockDim.x + threadIdx.x; cell < g.cells; cell += gridDim.x * blockDim.x) {
        const int row = cell / g.n[0];
        const int c[3] = {cell - row * g.n[0], row % g.n[1], row / g.n[1]};
        if (!in_box(g.o[0] + (double(c[0]) + 0.5) * g.h[0], g.o[1] + (double(c[1]) + 0.5) * g.h[1],
                    g.o[2] + (double(c[2]) + 0.5) * g.h[2], s.lower, s.upper))
            continue;
        tracer[cell] = float(fmin(double(tracer[cell]) + amount, 1.0));
    }
}

// Tracer sum (and, when `check`, the range check of prepare_impl :1337-1346):
// out: {sum}
__global__ void __launch_bounds__(EW_THREADS) k_fs_tracer_sum(GridDev g, const float* __restrict__ tracer, int check,
                                                              Partials part, double* out, int* flags) {
    __shared__ BlockReduce<1, 0> sm;
    double sum = 0.0;
    int local = 0;
    for (int cell = blockIdx.x * blockDim.x + threadIdx.x; cell < g.cells; cell += gridDim.x * blockDim.x) {
        const float t = tracer[cell];
        if (check && (!isfinite(t) || !(t >= 0.0f && t <= 1.0f))) local |= VF_ARITH;
        sum += double(t);
    }
    if (local) atomicOr(flags, local);
    dd sums[1] = {dd{sum, 0.0}};
    double none[1];
    block_reduce<1, 0>(sm, sums, none);
    if (publish_and_check_last<1, 0>(part, blockIdx.x, gridDim.x, sums, none)) {
        fold_partials<1, 0>(part, gridDim.x, sm, sums, none);
        if (threadIdx.x == 0) out[0] = dd_value(sums[0]);
    }
}

// commit_prepared (src/simulation.rs:805-811): publication by index rotation.
// The warm-start history restarts: the next seeded graph step starts cold.
__global__ void k_fs_commit(CarrierDev* cd, int acc, int tacc, double time, unsigned long long generation,
                            double rate) {
    cd->acc = acc;
    cd->tacc = tacc;
    cd->time = time;
    cd->generation = generation;
    cd->rate = rate;
    cd->history = 0;
    cd->flags = 0;
    cd->status = RB200_OK;
    cd->step_status = RB200_OK;
}

struct Cancel {
    rb200_step_cancel_fn fn;
    void* ctx;
    bool ask(int stage) const { return fn && fn(ctx, stage) != 0; }
};

int pressure_poll(void* c) { return static_cast<Cancel*>(c)->ask(RB200_STAGE_PRESSURE_ITERATION) ? 1 : 0; }

// The box-flux projection's stages as the step's (prepare_impl :1151-1160):
// BeforeSolve was the step's own BeforePressure already.
int projection_poll(void* c, int stage) {
    const Cancel* k = static_cast<Cancel*>(c);
    switch (stage) {
        case RB200_BOX_FLUX_PRESSURE_ITERATION: return k->ask(RB200_STAGE_PRESSURE_ITERATION) ? 1 : 0;
        case RB200_BOX_FLUX_CORRECTION_SLICE: return k->ask(RB200_STAGE_PROJECTION_SLICE) ? 1 : 0;
        case RB200_BOX_FLUX_BEFORE_ACCEPTANCE: return k->ask(RB200_STAGE_BEFORE_PROJECTION_ACCEPTANCE) ? 1 : 0;
        default: return 0;
    }
}

int rejected(rb200_forced_step_report* r, int error) {
    r->error = error;
    return RB200_SIMULATION_REJECTED;
}

int cancelled_at(rb200_forced_step_report* r, int stage) {
    r->stage = stage;
    return rejected(r, RB200_SIMULATION_CANCELLED);
}

bool finite_in_box(const double* lower, const double* upper, const GridDev& g) {
    for (int d = 0; d < 3; ++d)
        if (!std::isfinite(lower[d]) || !std::isfinite(upper[d]) || lower[d] >= upper[d] || lower[d] < g.o[d] ||
            upper[d] > g.up[d])
            return false;
    return true;
}

int ensure_scratch(rb200_carrier* c, size_t nforces) {
    if (!c->forced) {
        auto* s = new (std::nothrow) ForcedScratch();
        if (!s) return RB200_OUT_OF_MEMORY;
        long long b = (std::max<long long>(c->g.cells, (long long)c->g.flen[0] + c->g.flen[1] + c->g.flen[2]) +
                       EW_THREADS - 1) /
                      EW_THREADS;
        s->nb = int(std::min<long long>(std::max<long long>(b, 1), EW_BLOCKS_CAP));
        const size_t bytes = 16 + FS_SCALARS * sizeof(double) + size_t(s->nb) * FS_SLOT * sizeof(double) + 16;
        // attached only when complete: a failed allocation leaves no half-made scratch behind
        if (cudaMalloc(&s->d_buf, bytes) != cudaSuccess || cudaMemset(s->d_buf, 0, bytes) != cudaSuccess ||
            cudaMallocHost(&s->h_buf, 16 + FS_SCALARS * sizeof(double)) != cudaSuccess) {
            cudaGetLastError();
            forced_scratch_free(s);
            set_error("forced step scratch allocation failed");
            return RB200_OUT_OF_MEMORY;
        }
        s->d_flags = reinterpret_cast<int*>(s->d_buf);
        s->d_scalars = reinterpret_cast<double*>(s->d_buf + 16);
        s->part.data = s->d_scalars + FS_SCALARS;
        s->part.ticket = reinterpret_cast<unsigned*>(s->part.data + size_t(s->nb) * FS_SLOT);
        c->forced = s;
    }
    ForcedScratch* s = c->forced;
    if (nforces > s->force_cap) {
        cudaFree(s->d_forces);
        s->d_forces = nullptr;
        s->force_cap = 0;
        RB200_CUDA(cudaMalloc(&s->d_forces, nforces * sizeof(rb200_body_force)));
        s->force_cap = nforces;
    }
    return RB200_OK;
}

// Reads the flags and `n` scalars after the stream's work so far.
int read_back(rb200_carrier* c, int n, int* flags, double* scalars) {
    ForcedScratch* s = c->forced;
    RB200_CUDA(cudaMemcpyAsync(s->h_buf, s->d_buf, 16 + n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    RB200_CUDA(cudaStreamSynchronize(c->stream));
    *flags = *reinterpret_cast<int*>(s->h_buf);
    std::memcpy(scalars, s->h_buf + 16, n * sizeof(double));
    return RB200_OK;
}

int clear_flags(rb200_carrier* c) {
    RB200_CUDA(cudaMemsetAsync(c->forced->d_flags, 0, sizeof(int), c->stream));
    return RB200_OK;
}

struct FaceStats {
    double all, interior, mx[3];
};

int face_stats(rb200_carrier* c, int buf, FaceStats* st, int* flags) {
    ForcedScratch* s = c->forced;
    int rc = clear_flags(c);
    if (rc) return rc;
    k_fs_face_stats<<<s->nb, EW_THREADS, 0, c->stream>>>(c->g, (const float*)c->faces[buf][0],
                                                         (const float*)c->faces[buf][1],
                                                         (const float*)c->faces[buf][2], s->part, s->d_scalars,
                                                         s->d_flags);
    RB200_CUDA(cudaGetLastError());
    double sc[5];
    if ((rc = read_back(c, 5, flags, sc))) return rc;
    *st = FaceStats{sc[0], sc[1], {sc[2], sc[3], sc[4]}};
    return RB200_OK;
}

int tracer_sum(rb200_carrier* c, const float* tracer, bool check, double* sum, int* flags) {
    ForcedScratch* s = c->forced;
    int rc = clear_flags(c);
    if (rc) return rc;
    k_fs_tracer_sum<<<s->nb, EW_THREADS, 0, c->stream>>>(c->g, tracer, check ? 1 : 0, s->part, s->d_scalars,
                                                         s->d_flags);
    RB200_CUDA(cudaGetLastError());
    return read_back(c, 1, flags, sum);
}

// interior_energy (src/box_flux_step.rs:118-149) from an interior sum of squares
int interior_energy(double density, const GridDev& g, double sum, double* out) {
    const double e = 0.5 * density * g.volume * sum;
    if (!std::isfinite(e)) return RB200_ARITHMETIC_FAILURE;
    *out = e;
    return RB200_OK;
}

}  // namespace
}  // namespace rb200

using namespace rb200;

extern "C" int rb200_carrier_step_forced(rb200_carrier* c, const rb200_forced_step_params* prm,
                                         rb200_forced_step_report* rep, rb200_step_cancel_fn cancel_fn,
                                         void* ctx) {
    if (!c || !prm || !rep) return RB200_INVALID_ARGUMENT;
    std::memset(rep, 0, sizeof(*rep));
    if (c->in_flight) return RB200_INVALID_ARGUMENT;
    if (c->elem != 4 || !c->tracer[0]) return RB200_UNSUPPORTED;
    if (c->lq_d && !c->lq_inputs) return RB200_INVALID_ARGUMENT;  // the liquid step's inputs are not set
    const bool boundary = prm->box_flux != nullptr;
    if ((boundary && !prm->boundary) || (prm->force_count && !prm->forces)) return RB200_INVALID_ARGUMENT;
    if (boundary)
        for (float x : prm->boundary->outward)
            if (!std::isfinite(x)) {  // PrescribedBoxFlux::new (src/box_flux.rs:23-28)
                rep->projection.error = RB200_BOX_FLUX_INVALID_BOUNDARY;
                return RB200_BOX_FLUX_REJECTED;
            }
    cudaSetDevice(c->device);
    const GridDev& g = c->g;
    const double density = c->cfg.density;
    const Cancel cancel{cancel_fn, ctx};
    rep->has_boundary = boundary ? 1 : 0;
    rep->tracer_policy = prm->tracer_policy;
    // prepare_impl (src/simulation.rs:812-880)
    const double requested_dt = prm->requested_dt;
    if (!std::isfinite(requested_dt) || requested_dt <= 0.0) return RB200_INVALID_ARGUMENT;  // InvalidTimeStep
    const rb200_smoke_source* src = prm->source;
    if (src) {
        if (!std::isfinite(src->tracer_rate) || src->tracer_rate < 0.0 || !std::isfinite(src->vertical_acceleration) ||
            !finite_in_box(src->lower, src->upper, g))
            return rejected(rep, RB200_SIMULATION_INVALID_SOURCE);
    }
    double external_rate = 0.0;  // forces::validate (src/forces.rs:63-94)
    for (size_t i = 0; i < prm->force_count; ++i) {
        const rb200_body_force& f = prm->forces[i];
        for (double x : f.value)
            if (!std::isfinite(x)) return rejected(rep, RB200_SIMULATION_INVALID_FORCE);
        if (f.has_region && !finite_in_box(f.lower, f.upper, g)) return rejected(rep, RB200_SIMULATION_INVALID_FORCE);
        for (int d = 0; d < 3; ++d) {
            const double a = f.units == RB200_FORCE_DENSITY ? f.value[d] / density : f.value[d];
            external_rate += std::fabs(a) / g.h[d];
        }
    }
    if (!std::isfinite(external_rate)) return RB200_ARITHMETIC_FAILURE;
    if (boundary && !box_flux_matches(prm->box_flux, c->cfg.grid, density, c->cfg.method))
        return rejected(rep, RB200_SIMULATION_BOUNDARY_WORKSPACE_MISMATCH);
    int rc = ensure_scratch(c, prm->force_count);
    if (rc) return rc;
    ForcedScratch* S = c->forced;
    if (prm->force_count)
        RB200_CUDA(cudaMemcpyAsync(S->d_forces, prm->forces, prm->force_count * sizeof(rb200_body_force),
                                   cudaMemcpyHostToDevice, c->stream));
    RB200_CUDA(cudaMemcpyAsync(c->h_cd, c->cd, sizeof(CarrierDev), cudaMemcpyDeviceToHost, c->stream));
    RB200_CUDA(cudaStreamSynchronize(c->stream));
    const int A = c->h_cd->acc, B = (A + 1) % 3, Cb = (A + 2) % 3;
    const int tacc = c->h_cd->tacc;
    const double time = c->h_cd->time;
    const unsigned long long generation = c->h_cd->generation;
    float* tracer_old = c->tracer[tacc];
    float* tracer_new = c->tracer[tacc ^ 1];
    float* prov[3] = {(float*)c->faces[B][0], (float*)c->faces[B][1], (float*)c->faces[B][2]};
    float* cand[3] = {(float*)c->faces[Cb][0], (float*)c->faces[Cb][1], (float*)c->faces[Cb][2]};
    const float* acc[3] = {(const float*)c->faces[A][0], (const float*)c->faces[A][1], (const float*)c->faces[A][2]};
    int flags = 0;
    FaceStats old{};
    if ((rc = face_stats(c, A, &old, &flags))) return rc;
    if (boundary) {
        if ((rc = interior_energy(density, g, old.interior, &rep->kinetic_old))) return rc;
        double ts = 0.0;
        if ((rc = tracer_sum(c, tracer_old, false, &ts, &flags))) return rc;
        rep->tracer_old_integral = ts * g.volume;
    }
    // dt policy (:927-979)
    double rate = 0.0;
    if (boundary) {
        const float* o = prm->boundary->outward;
        for (int d = 0; d < 3; ++d)
            rate += std::fmax(std::fmax(old.mx[d], std::fabs(double(o[2 * d]))), std::fabs(double(o[2 * d + 1]))) /
                    g.h[d];
    } else {
        for (int d = 0; d < 3; ++d) rate += old.mx[d] / g.h[d];
    }
    if (!std::isfinite(rate)) return RB200_ARITHMETIC_FAILURE;
    const double acceleration = (src ? std::fabs(src->vertical_acceleration) / g.h[1] : 0.0) + external_rate;
    if (!std::isfinite(acceleration)) return RB200_ARITHMETIC_FAILURE;
    const double max_courant = c->cfg.max_courant;
    double dt = requested_dt;
    if (rate > 0.0) dt = std::fmin(dt, 0.5 * max_courant / rate);
    if (acceleration > 0.0) dt = std::fmin(dt, std::sqrt(0.5 * max_courant / acceleration));
    const double next_time = time + dt;
    if (dt <= 0.0 || !std::isfinite(next_time) || next_time <= time)
        return rejected(rep, RB200_SIMULATION_TIME_RESOLUTION);
    rep->dt = dt;
    const long long nz = g.n[2];
    const long long face_slices = 3 * nz + 1;
    // advection (:992-1003): VelocitySlice once per face plane of each axis
    if (cancel.ask(RB200_STAGE_BEFORE_ADVECTION)) return cancelled_at(rep, RB200_STAGE_BEFORE_ADVECTION);
    if (cancel.ask(RB200_STAGE_VELOCITY_SLICE)) return cancelled_at(rep, RB200_STAGE_VELOCITY_SLICE);
    if ((rc = clear_flags(c))) return rc;
    const bool fp32 = c->cfg.fp32_advection != 0;
    if ((rc = launch_advect_velocity<float>(g, acc[0], acc[1], acc[2], dt, prov[0], prov[1], prov[2], nullptr, 0.0,
                                            S->d_flags, c->stream, fp32)))
        return rc;
    for (long long t = 1; t < face_slices; ++t)
        if (cancel.ask(RB200_STAGE_VELOCITY_SLICE)) {
            cudaStreamSynchronize(c->stream);
            return cancelled_at(rep, RB200_STAGE_VELOCITY_SLICE);
        }
    FaceStats st{};
    if (boundary) {
        if ((rc = face_stats(c, B, &st, &flags))) return rc;
        if ((rc = interior_energy(density, g, st.interior, &rep->kinetic_after_advection))) return rc;
        rep->advection_change = rep->kinetic_after_advection - rep->kinetic_old;
    }
    // the smoke source's force (:1018-1020)
    if (src) {
        if ((rc = clear_flags(c))) return rc;
        k_fs_smoke_force<<<S->nb, EW_THREADS, 0, c->stream>>>(g, prov[1], *src, dt, S->d_flags);
        RB200_CUDA(cudaGetLastError());
        double none[1];
        if ((rc = read_back(c, 0, &flags, none))) return rc;
        if (flags & VF_ARITH) return RB200_ARITHMETIC_FAILURE;
    }
    if (boundary) {
        if ((rc = face_stats(c, B, &st, &flags))) return rc;
        if ((rc = interior_energy(density, g, st.interior, &rep->kinetic_after_smoke_force))) return rc;
        rep->smoke_force_work = rep->kinetic_after_smoke_force - rep->kinetic_after_advection;
    }
    // body forces (:1043-1082): ForceSlice once per face plane of each axis
    if (prm->force_count) {
        if (cancel.ask(RB200_STAGE_BEFORE_FORCES)) return cancelled_at(rep, RB200_STAGE_BEFORE_FORCES);
        if (cancel.ask(RB200_STAGE_FORCE_SLICE)) return cancelled_at(rep, RB200_STAGE_FORCE_SLICE);
        if ((rc = clear_flags(c))) return rc;
        const double mass = density * g.volume;
        k_fs_forces<<<S->nb, EW_THREADS, 0, c->stream>>>(g, prov[0], prov[1], prov[2], S->d_forces,
                                                         int(prm->force_count), density, dt, mass, S->part,
                                                         S->d_scalars, S->d_flags);
        RB200_CUDA(cudaGetLastError());
        bool late = false;
        for (long long t = 1; t < face_slices && !late; ++t) late = cancel.ask(RB200_STAGE_FORCE_SLICE);
        double sc[3];
        if ((rc = read_back(c, 3, &flags, sc))) return rc;
        if (late) return cancelled_at(rep, RB200_STAGE_FORCE_SLICE);
        if (flags & VF_ARITH) return RB200_ARITHMETIC_FAILURE;
        const double before = 0.5 * mass * sc[0], after = 0.5 * mass * sc[1];
        if (!std::isfinite(before) || !std::isfinite(after) || !std::isfinite(sc[2])) return RB200_ARITHMETIC_FAILURE;
        rep->has_forces = 1;
        rep->force_kinetic_before = before;
        rep->force_kinetic_after = after;
        rep->force_applied_work = sc[2];
    }
    if (cancel.ask(RB200_STAGE_BEFORE_PRESSURE)) return cancelled_at(rep, RB200_STAGE_BEFORE_PRESSURE);
    // projection (:1104-1262)
    if (boundary) {
        RB200_CUDA(cudaStreamSynchronize(c->stream));
        const float* in[3] = {prov[0], prov[1], prov[2]};
        const size_t lens[3] = {size_t(g.flen[0]), size_t(g.flen[1]), size_t(g.flen[2])};
        rc = rb200_box_flux_project_device(prm->box_flux, in, lens, dt, prm->boundary, &c->cfg.settings,
                                           c->cfg.actual_divergence_limit, cand, lens, &rep->projection,
                                           cancel_fn ? projection_poll : nullptr, const_cast<Cancel*>(&cancel));
        rep->pressure = rep->projection.pressure;
        if (rc == RB200_BOX_FLUX_REJECTED && rep->projection.error == RB200_BOX_FLUX_CANCELLED) {
            const int s = rep->projection.stage;
            return cancelled_at(rep, s == RB200_BOX_FLUX_CORRECTION_SLICE     ? RB200_STAGE_PROJECTION_SLICE
                                     : s == RB200_BOX_FLUX_BEFORE_ACCEPTANCE ? RB200_STAGE_BEFORE_PROJECTION_ACCEPTANCE
                                                                             : RB200_STAGE_BEFORE_PRESSURE);
        }
        if (rc == RB200_BOX_FLUX_REJECTED && rep->projection.error == RB200_BOX_FLUX_DIVERGENCE_LIMIT) {
            rep->error_actual = rep->projection.error_actual;
            rep->error_limit = rep->projection.error_limit;
            rep->actual_divergence_max = rep->projection.actual_divergence_max;
            return RB200_DIVERGENCE_LIMIT;  // SimulationError::DivergenceLimit (:125-128)
        }
        if (rc) return rc;
        rep->actual_divergence_max = rep->projection.actual_divergence_max;
        const rb200_box_flux_report& p = rep->projection;
        rep->kinetic_before_projection = p.kinetic_before;
        rep->kinetic_accepted = p.kinetic_after;
        rep->external_force_work = rep->has_forces ? rep->force_applied_work : 0.0;
        rep->boundary_volume_imbalance = dt * p.net_outward_flux;
        rep->budget_error = rep->kinetic_accepted - rep->kinetic_old + p.correction_energy -
                            (rep->advection_change + rep->smoke_force_work + rep->external_force_work +
                             p.boundary_pressure_work + p.divergence_residual_work + p.correction_residual_work);
    } else {
        if ((rc = clear_flags(c))) return rc;
        if ((rc = launch_validate_faces<float>(g, prov[0], prov[1], prov[2], S->d_flags, c->stream))) return rc;
        if ((rc = launch_build_rhs<float>(g, prov[0], prov[1], prov[2], dt, c->solver.b(), S->d_flags, c->stream)))
            return rc;
        double none[1];
        if ((rc = read_back(c, 0, &flags, none))) return rc;
        if (flags & VF_NONFINITE) return RB200_NONFINITE_INPUT;
        if (flags & VF_WALL) return RB200_NONZERO_WALL_VELOCITY;
        if (flags & VF_ARITH) return RB200_ARITHMETIC_FAILURE;
        if (!settings_valid(&c->cfg.settings)) return RB200_INVALID_ARGUMENT;
        c->last_rejected = true;  // the solver's pressure is no longer the accepted one
        rc = c->solver.solve(dt, c->cfg.settings, &rep->pressure, cancel_fn ? pressure_poll : nullptr,
                             const_cast<Cancel*>(&cancel));
        if (rc) return rc;
        if ((rc = clear_flags(c))) return rc;
        const float* const in3[3] = {prov[0], prov[1], prov[2]};
        float* const out3[3] = {cand[0], cand[1], cand[2]};
        if ((rc = launch_correct_divergence<float>(g, c->solver.p(), dt, in3, out3, c->solver.partials(),
                                                   c->solver.partial_blocks(), S->d_scalars, S->d_flags, c->stream)))
            return rc;
        double sc[4];
        if ((rc = read_back(c, 4, &flags, sc))) return rc;
        if (flags & (VF_ARITH | VF_F32_RANGE)) return RB200_ARITHMETIC_FAILURE;
        rep->actual_divergence_max = sc[0];
        if (sc[0] > c->cfg.actual_divergence_limit) {
            rep->error_actual = sc[0];
            rep->error_limit = c->cfg.actual_divergence_limit;
            return RB200_DIVERGENCE_LIMIT;
        }
    }
    // Courant gate (:1268-1277)
    FaceStats fin{};
    if ((rc = face_stats(c, Cb, &fin, &flags))) return rc;
    double crate = 0.0;
    for (int d = 0; d < 3; ++d) crate += fin.mx[d] / g.h[d];
    if (!std::isfinite(crate)) return RB200_ARITHMETIC_FAILURE;
    const double courant = dt * crate;
    rep->courant = courant;
    if (!std::isfinite(courant)) return RB200_ARITHMETIC_FAILURE;
    if (courant > max_courant) {
        rep->error_actual = courant;
        rep->error_limit = max_courant;
        return RB200_COURANT_LIMIT;
    }
    // tracer (:1278-1346): TracerSlice once per cell plane
    if (cancel.ask(RB200_STAGE_BEFORE_TRACER)) return cancelled_at(rep, RB200_STAGE_BEFORE_TRACER);
    if (cancel.ask(RB200_STAGE_TRACER_SLICE)) return cancelled_at(rep, RB200_STAGE_TRACER_SLICE);
    if ((rc = clear_flags(c))) return rc;
    if ((rc = launch_advect_tracer<float>(g, tracer_old, cand[0], cand[1], cand[2], dt, tracer_new, S->d_flags,
                                          c->stream, fp32)))
        return rc;
    for (long long t = 1; t < nz; ++t)
        if (cancel.ask(RB200_STAGE_TRACER_SLICE)) {
            cudaStreamSynchronize(c->stream);
            return cancelled_at(rep, RB200_STAGE_TRACER_SLICE);
        }
    double transported = 0.0;
    if (boundary) {
        double ts = 0.0;
        if ((rc = tracer_sum(c, tracer_new, false, &ts, &flags))) return rc;
        transported = ts * g.volume;
    }
    if (src) {
        const double amount = dt * src->tracer_rate;
        if (!std::isfinite(amount)) return RB200_ARITHMETIC_FAILURE;
        k_fs_smoke_source<<<S->nb, EW_THREADS, 0, c->stream>>>(g, tracer_new, *src, amount);
        RB200_CUDA(cudaGetLastError());
    }
    double tsum = 0.0;
    if ((rc = tracer_sum(c, tracer_new, true, &tsum, &flags))) return rc;
    if (flags & VF_ARITH) return RB200_ARITHMETIC_FAILURE;
    const double tracer_integral = tsum * g.volume;
    const double kinetic = boundary ? rep->kinetic_accepted : 0.5 * density * g.volume * fin.all;
    if (boundary) {
        rep->tracer_transport_change = transported - rep->tracer_old_integral;
        rep->tracer_source_change = tracer_integral - transported;
        const double check[5] = {rep->budget_error, rep->boundary_volume_imbalance, rep->tracer_old_integral,
                                 rep->tracer_transport_change, rep->tracer_source_change};
        for (double x : check)
            if (!std::isfinite(x)) return RB200_ARITHMETIC_FAILURE;
    }
    if (!std::isfinite(tracer_integral) || !std::isfinite(kinetic)) return RB200_ARITHMETIC_FAILURE;
    if (cancel.ask(RB200_STAGE_BEFORE_COMMIT)) return cancelled_at(rep, RB200_STAGE_BEFORE_COMMIT);
    // the liquid step (LiquidTransportSimulation::step_impl, src/liquid_step.rs:867-917):
    // the transport through the candidate faces over [time, time + dt], stamped
    // {flow_id, candidate generation}; a rejection rejects the step
    if (c->lq_d) {
        LiquidFlowDev& lf = *c->lflow_h;
        for (int d = 0; d < 3; ++d) lf.vel[d] = cand[d];
        lf.start = time;
        lf.dt = dt;
        lf.flow = rb200_liquid_stamp{c->h_cd->flow_id, generation + 1};
        lf.active = 1;
        lf.periodic = 0;
        RB200_CUDA(cudaMemcpyAsync(c->lflow_d, c->lflow_h, sizeof(LiquidFlowDev), cudaMemcpyHostToDevice, c->stream));
        RB200_CUDA(launch_liquid_advance(g, c->lq_d, c->lflow_d, c->lq_sc, c->lq_blocks, c->lrep_d, c->stream));
        RB200_CUDA(cudaMemcpyAsync(c->lrep_h, c->lrep_d, sizeof(rb200_liquid_report), cudaMemcpyDeviceToHost,
                                   c->stream));
        RB200_CUDA(cudaStreamSynchronize(c->stream));
        if (c->lrep_h->error) return RB200_LIQUID_REJECTED;
        if (cancel.ask(RB200_STAGE_LIQUID_BEFORE_COMMIT))
            return cancelled_at(rep, RB200_STAGE_LIQUID_BEFORE_COMMIT);
    }
    // commit: the step's pressure becomes the accepted one (the dense3D
    // frame's pressure field)
    const size_t pbytes = size_t(g.cells) * sizeof(double);
    if (boundary)
        RB200_CUDA(cudaMemcpyAsync(c->solver.p(), rb200_box_flux_pressure_device(prm->box_flux), pbytes,
                                   cudaMemcpyDeviceToDevice, c->stream));
    if (c->accepted_p)
        RB200_CUDA(cudaMemcpyAsync(c->accepted_p, c->solver.p(), pbytes, cudaMemcpyDeviceToDevice, c->stream));
    k_fs_commit<<<1, 1, 0, c->stream>>>(c->cd, Cb, tacc ^ 1, next_time, generation + 1, crate);
    RB200_CUDA(cudaGetLastError());
    if (c->lq_d) {
        RB200_CUDA(launch_liquid_commit(c->lq_d, c->lrep_d, c->stream));
        RB200_CUDA(cudaMemcpyAsync(c->lq_h, c->lq_d, sizeof(LiquidDev), cudaMemcpyDeviceToHost, c->stream));
    }
    RB200_CUDA(cudaMemcpyAsync(c->h_cd, c->cd, sizeof(CarrierDev), cudaMemcpyDeviceToHost, c->stream));
    RB200_CUDA(cudaStreamSynchronize(c->stream));
    c->accepted_steps += 1;
    c->last_rejected = false;
    rep->time = next_time;
    rep->generation = generation + 1;
    rep->tracer_integral = tracer_integral;
    rep->kinetic_energy = kinetic;
    rep->simulation_array_bytes = c->bytes;
    if (boundary)
        rep->boundary_workspace_array_bytes =
            rb200_box_flux_allocated_bytes(prm->box_flux) + 4ull * uint64_t(g.flen[0] + g.flen[1] + g.flen[2]);
    return RB200_OK;
}
