// Resident fixed-box carrier step: the state stays in HBM and one step is
// one CUDA graph, composed as Rheon's step owner orders it
// (Simulation::prepare_impl, src/simulation.rs:812-1403):
//   dt policy -> advect_velocity (+ buoyancy hook) -> build_rhs -> pressure
//   solve (WHILE node over iteration chunks) -> correct_candidate + actual
//   divergence + velocity rate -> gates -> advect_tracer -> commit.
// Every decision (dt, solve control, gates, commit) is taken on the device;
// the host launches the graph and reads one small report afterwards. The
// accepted state is never written by a rejected step (transactional, as
// commit_prepared, src/simulation.rs:805-811): the step writes candidate and
// corrected buffers and publishes by rotating buffer indices on the device.
#include <cmath>
#include <memory>
#include <mutex>
#include <new>
#include <string>

#include "advect.cuh"
#include "internal.hpp"
#include "carrier.hpp"
#include "project.cuh"

namespace rb200 {

__device__ __forceinline__ bool step_running(const CarrierDev* cd) { return cd->status == STEP_RUNNING; }

// Proceed to the correction: the solve converged, or an exact-iteration-count
// solve reached its limit.
__device__ __forceinline__ bool solve_usable(const CarrierDev* cd, const SolveState* st) {
    return step_running(cd) &&
           (st->status == RB200_OK || (st->status == RB200_ITERATION_LIMIT && cd->iteration_limit_ok));
}

// dt policy (src/simulation.rs:952-979): dt = min(requested, cfl/rate).
__global__ void k_step_begin(CarrierDev* cd) {
    double dt = cd->requested_dt;
    if (cd->cfl > 0.0 && cd->rate > 0.0) dt = fmin(dt, cd->cfl / cd->rate);
    cd->dt = dt;
    cd->flags = 0;
    cd->skip = 0;
    cd->status = STEP_RUNNING;
    const double next = cd->time + dt;
    if (!isfinite(dt) || dt <= 0.0 || !isfinite(next) || next <= cd->time) {
        cd->status = RB200_INVALID_ARGUMENT;
        cd->skip = 1;
    }
    cd->warm = (cd->warm_policy && cd->history) ? 1 : 0;
}

template <class T, class R>
__global__ void __launch_bounds__(ADV_THREADS) k_carrier_advect(GridDev g, CarrierDev* cd) {
    if (!step_running(cd)) return;
    const int a = cd->acc, b = (a + 1) % 3;
    if (cd->project_only) {
        // a projection takes the accepted faces as the provisional velocity
        for (int d = 0; d < 3; ++d) {
            const T* __restrict__ src = (const T*)cd->faces[a][d];
            T* __restrict__ dst = (T*)cd->faces[b][d];
            for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < g.flen[d]; f += gridDim.x * blockDim.x)
                dst[f] = src[f];
        }
        return;
    }
    Faces<T> vel{{(const T*)cd->faces[a][0], (const T*)cd->faces[a][1], (const T*)cd->faces[a][2]}};
    const float* tr = cd->tracer[0] ? cd->tracer[cd->tacc] : nullptr;
    advect_velocity_body<T, R>(g, vel, cd->dt, (T*)cd->faces[b][0], (T*)cd->faces[b][1], (T*)cd->faces[b][2], tr,
                               cd->buoyancy, &cd->flags, whole_launch());
}

template <class T>
__global__ void k_carrier_rhs(GridDev g, CarrierDev* cd, double* __restrict__ rhs) {
    if (!step_running(cd)) return;
    const int b = (cd->acc + 1) % 3;
    build_rhs_body<T>(g, (const T*)cd->faces[b][0], (const T*)cd->faces[b][1], (const T*)cd->faces[b][2], cd->dt,
                      rhs, &cd->flags, whole_launch());
}

template <class T>
__global__ void __launch_bounds__(EW_THREADS) k_carrier_correct(GridDev g, CarrierDev* cd, const SolveState* st,
                                                                const double* __restrict__ p, Partials part) {
    if (!solve_usable(cd, st)) return;
    const int b = (cd->acc + 1) % 3, c = (cd->acc + 2) % 3;
    correct_divergence_body<T>(g, p, cd->dt, (const T*)cd->faces[b][0], (const T*)cd->faces[b][1],
                               (const T*)cd->faces[b][2], (T*)cd->faces[c][0], (T*)cd->faces[c][1],
                               (T*)cd->faces[c][2], part, cd->scalars, &cd->flags, whole_launch());
}

template <class T, class R>
__global__ void __launch_bounds__(ADV_THREADS) k_carrier_tracer(GridDev g, CarrierDev* cd, const SolveState* st) {
    if (!cd->tracer[0] || !solve_usable(cd, st)) return;
    const int c = (cd->acc + 2) % 3;
    Faces<T> vel{{(const T*)cd->faces[c][0], (const T*)cd->faces[c][1], (const T*)cd->faces[c][2]}};
    advect_tracer_body<T, R>(g, cd->tracer[cd->tacc], vel, cd->dt, cd->tracer[cd->tacc ^ 1], &cd->flags,
                            whole_launch());
}

// The liquid interval of the step (src/liquid_step.rs:869-887): the
// corrected candidate faces over [time, time + dt], stamped with the
// candidate generation. Inactive when the carrier part already failed.
__global__ void k_carrier_liquid_flow(CarrierDev* cd, const SolveState* st) {
    LiquidFlowDev* f = cd->lflow;
    const bool run = solve_usable(cd, st) && !(cd->flags & (VF_NONFINITE | VF_ARITH | VF_F32_RANGE));
    f->active = run ? 1 : 0;
    if (!run) return;
    const int c = (cd->acc + 2) % 3;
    for (int d = 0; d < 3; ++d) f->vel[d] = static_cast<const float*>(cd->faces[c][d]);
    f->start = cd->time;
    f->dt = cd->dt;
    f->flow = rb200_liquid_stamp{cd->flow_id, cd->generation + 1};
}

// Gates and commit: actual divergence (simulation.rs:1235-1243), Courant
// (simulation.rs:1268-1277), then publication by index rotation.
__global__ void k_step_end(GridDev g, CarrierDev* cd, const SolveState* st) {
    rb200_step_report& rep = cd->report;
    rep.dt = cd->dt;
    rep.pressure.iterations = uint64_t(st->it);
    rep.pressure.true_residual_l2 = st->true_l2;
    rep.pressure.true_residual_max = st->true_max;
    rep.pressure.predicted_divergence_max = st->true_div;
    rep.pressure.incompatible_sum = st->incompatible_sum;
    rep.pressure.incompatible_budget = st->incompatible_budget;
    rep.pressure.breakdown_iteration = uint64_t(st->breakdown_it);
    rep.pressure_status = st->status;
    cd->trips = st->trips;
    int status = cd->status;
    if (status == STEP_RUNNING) {
        if (!solve_usable(cd, st)) {
            status = st->status;
        } else if (cd->flags & VF_NONFINITE) {
            status = RB200_NONFINITE_INPUT;
        } else if (cd->flags & (VF_ARITH | VF_F32_RANGE)) {
            status = RB200_ARITHMETIC_FAILURE;
        } else {
            // velocity_rate (src/simulation.rs:1415-1429): sum_d max|u_d| / h_d
            double rate = 0.0;
            for (int d = 0; d < 3; ++d) rate += cd->scalars[1 + d] / g.h[d];
            rep.actual_divergence_max = cd->scalars[0];
            rep.velocity_rate = rate;
            rep.courant = cd->dt * rate;
            status = RB200_OK;
            if (!cd->skip_gates) {
                if (rep.actual_divergence_max > cd->divergence_limit)
                    status = RB200_DIVERGENCE_LIMIT;
                else if (!isfinite(rep.courant))
                    status = RB200_ARITHMETIC_FAILURE;
                else if (rep.courant > cd->max_courant && !cd->project_only)
                    status = RB200_COURANT_LIMIT;
            }
            // the liquid interval is part of the transaction: a rejected
            // transport rejects the step (src/liquid_step.rs:881-900)
            if (status == RB200_OK && cd->liquid && cd->lrep->error) status = RB200_LIQUID_REJECTED;
            if (status == RB200_OK) {
                cd->acc = (cd->acc + 2) % 3;
                if (cd->tracer[0]) cd->tacc ^= 1;
                cd->time += cd->dt;
                cd->generation += 1;
                cd->rate = rate;
                if (cd->liquid) liquid_commit(cd->liquid, *cd->lrep);
            }
        }
    }
    rep.time = cd->time;
    rep.generation = cd->generation;
    rep.pressure_initialization = cd->warm;
    cd->step_status = status;
    cd->status = status;
}

// Keeps the pressure of an accepted step as the next step's seed; a rejected
// step leaves the previous one in place.
__global__ void __launch_bounds__(EW_THREADS) k_keep_pressure(GridDev g, CarrierDev* cd, const double* __restrict__ p) {
    if (cd->step_status != RB200_OK) return;
    double* dst = cd->accepted_p;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < g.cells; c += gridDim.x * blockDim.x) dst[c] = p[c];
    if (blockIdx.x == 0 && threadIdx.x == 0) cd->history = 1;
}

// Random-Fourier initial state on the device: u_d(x) = sum_m a_{m,d}
// sin(2 pi k_m.x/L + phi_m) + noise * U(-1,1) at the face centres, wall-normal
// faces 0. The noise is the counter-based SplitMix64 stream 16+d of the host
// generator (rheon_b200/workloads.py), so it matches the host bit for bit;
// sin is the device's double-precision sine.
struct FourierModes {
    double k[8][3];
    double phase[8];
    double amp[8][3];
    int modes;
    double amplitude, noise;
    unsigned long long seed;
};

__device__ __forceinline__ unsigned long long splitmix64(unsigned long long x) {
    unsigned long long z = x + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

template <class T>
__global__ void k_fourier_init(GridDev g, CarrierDev* cd, FourierModes fm) {
    const long long total = (long long)g.flen[0] + g.flen[1] + g.flen[2];
    const double two_pi = 6.283185307179586;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
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
        const int p[3] = {int(f % g.fc[a][0]), int((f / g.fc[a][0]) % g.fc[a][1]),
                          int(f / ((long long)g.fc[a][0] * g.fc[a][1]))};
        T* dst = (T*)cd->faces[cd->acc][a];
        if (p[a] == 0 || p[a] == g.n[a]) {
            dst[f] = T(0);
            continue;
        }
        double x[3];
        for (int d = 0; d < 3; ++d) x[d] = double(p[d]) + (d == a ? 0.0 : 0.5);
        double val = 0.0;
        for (int m = 0; m < fm.modes; ++m) {
            double arg = two_pi * (fm.k[m][0] * x[0] / g.n[0] + fm.k[m][1] * x[1] / g.n[1] +
                                   fm.k[m][2] * x[2] / g.n[2]) + fm.phase[m];
            val += fm.amplitude * fm.amp[m][a] * sin(arg);
        }
        const unsigned long long key = fm.seed ^ ((unsigned long long)(16 + a) << 48);
        const unsigned long long u = splitmix64((unsigned long long)f ^ key);
        const double r = 2.0 * double(u >> 11) * 1.1102230246251565e-16 - 1.0;
        dst[f] = T(val + fm.noise * r);
    }
}

// Per-axis face maxima and validation of an uploaded state.
template <class T>
int launch_validate_faces(const GridDev& g, const T* u, const T* v, const T* w, int* flags, cudaStream_t s);

}  // namespace rb200

using namespace rb200;

namespace {

int select_carrier_device(int device) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        set_error("no CUDA device");
        return RB200_NO_DEVICE;
    }
    if (device < 0 || device >= count) return RB200_INVALID_ARGUMENT;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major != 10) {
        set_error("librheon_b200 is built for sm_100a (B200) only");
        return RB200_NO_DEVICE;
    }
    return cudaSetDevice(device) == cudaSuccess ? RB200_OK : RB200_NO_DEVICE;
}

int blocks_for(long long n, int threads, int cap) {
    long long b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    return int(b < cap ? b : cap);
}

template <class T>
int capture_step(rb200_carrier* c) {
    const GridDev& g = c->g;
    cudaStream_t s = c->stream;
    const long long faces = (long long)g.flen[0] + g.flen[1] + g.flen[2];
    const int fb = blocks_for(faces, ADV_THREADS, 148 * 64);
    const int cb = blocks_for(g.cells, ADV_THREADS, 148 * 64);
    const int eb = blocks_for(g.cells, EW_THREADS, std::min(EW_BLOCKS_CAP, c->solver.partial_blocks()));
    const bool fp32 = c->cfg.fp32_advection != 0;
    cudaGraph_t graph = nullptr;
    RB200_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
    k_step_begin<<<1, 1, 0, s>>>(c->cd);
    if (fp32)
        k_carrier_advect<T, float><<<fb, ADV_THREADS, 0, s>>>(g, c->cd);
    else
        k_carrier_advect<T, double><<<fb, ADV_THREADS, 0, s>>>(g, c->cd);
    k_carrier_rhs<T><<<cb, ADV_THREADS, 0, s>>>(g, c->cd, c->solver.b());
    RB200_CUDA(cudaEventRecordWithFlags(c->ev[0], s, cudaEventRecordExternal));
    int rc = c->accepted_p
                 ? c->solver.enqueue_reset(&c->cd->dt, &c->cd->skip, c->cfg.settings, s, &c->cd->warm, c->accepted_p)
                 : c->solver.enqueue_reset(&c->cd->dt, &c->cd->skip, c->cfg.settings, s);
    if (!rc) rc = c->solver.enqueue_loop(s, c->body_stream, c->cfg.settings);
    if (rc) {
        cudaGraph_t dummy = nullptr;
        cudaStreamEndCapture(s, &dummy);
        if (dummy) cudaGraphDestroy(dummy);
        return rc;
    }
    RB200_CUDA(cudaEventRecordWithFlags(c->ev[1], s, cudaEventRecordExternal));
    k_carrier_correct<T><<<eb, EW_THREADS, 0, s>>>(g, c->cd, c->solver.state(), c->solver.p(), c->solver.partials());
    if (c->tracer[0]) {
        if (fp32)
            k_carrier_tracer<T, float><<<cb, ADV_THREADS, 0, s>>>(g, c->cd, c->solver.state());
        else
            k_carrier_tracer<T, double><<<cb, ADV_THREADS, 0, s>>>(g, c->cd, c->solver.state());
    }
    if (c->lq_d) {
        k_carrier_liquid_flow<<<1, 1, 0, s>>>(c->cd, c->solver.state());
        RB200_CUDA(launch_liquid_advance(g, c->lq_d, c->lflow_d, c->lq_sc, c->lq_blocks, c->lrep_d, s));
    }
    k_step_end<<<1, 1, 0, s>>>(g, c->cd, c->solver.state());
    if (c->accepted_p) k_keep_pressure<<<eb, EW_THREADS, 0, s>>>(g, c->cd, c->solver.p());
    RB200_CUDA(cudaMemcpyAsync(c->h_cd, c->cd, sizeof(CarrierDev), cudaMemcpyDeviceToHost, s));
    if (c->lq_d) {
        RB200_CUDA(cudaMemcpyAsync(c->lq_h, c->lq_d, sizeof(LiquidDev), cudaMemcpyDeviceToHost, s));
        RB200_CUDA(cudaMemcpyAsync(c->lrep_h, c->lrep_d, sizeof(rb200_liquid_report), cudaMemcpyDeviceToHost, s));
    }
    cudaError_t le = cudaGetLastError();
    cudaError_t ee = cudaStreamEndCapture(s, &graph);
    if (le != cudaSuccess || ee != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        set_error(std::string("step capture: ") + cudaGetErrorString(le != cudaSuccess ? le : ee));
        return RB200_EXECUTION;
    }
    cudaError_t ie = cudaGraphInstantiate(&c->step_exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ie != cudaSuccess) {
        set_error(std::string("step graph instantiate: ") + cudaGetErrorString(ie));
        return RB200_EXECUTION;
    }
    // begin, advect, rhs, reset (+start kernels counted by the solver), correct, tracer, end
    // (+ seed and keep kernels with the warm-start policy)
    c->fixed_nodes = 5 + (c->tracer[0] ? 1 : 0) + (c->accepted_p ? 2 : 0) + (c->lq_d ? 2 : 0);
    return RB200_OK;
}

int upload_rate(rb200_carrier* c) {
    // velocity rate and validation of the accepted state (after an upload)
    c->accepted_steps = 0;
    c->last_rejected = false;
    const GridDev& g = c->g;
    int* d_flags = &c->cd->flags;
    double* sc = c->cd->scalars;
    RB200_CUDA(cudaMemsetAsync(d_flags, 0, sizeof(int), c->stream));
    const int a = c->h_cd->acc;
    int rc;
    if (c->elem == 4) {
        rc = launch_face_maxima<float>(g, (const float*)c->faces[a][0], (const float*)c->faces[a][1],
                                       (const float*)c->faces[a][2], c->solver.partials(), c->solver.partial_blocks(),
                                       sc, d_flags, c->stream);
        if (!rc)
            rc = launch_validate_faces<float>(g, (const float*)c->faces[a][0], (const float*)c->faces[a][1],
                                              (const float*)c->faces[a][2], d_flags, c->stream);
    } else {
        rc = launch_face_maxima<double>(g, (const double*)c->faces[a][0], (const double*)c->faces[a][1],
                                        (const double*)c->faces[a][2], c->solver.partials(),
                                        c->solver.partial_blocks(), sc, d_flags, c->stream);
        if (!rc)
            rc = launch_validate_faces<double>(g, (const double*)c->faces[a][0], (const double*)c->faces[a][1],
                                               (const double*)c->faces[a][2], d_flags, c->stream);
    }
    if (rc) return rc;
    RB200_CUDA(cudaMemcpyAsync(c->h_cd, c->cd, sizeof(CarrierDev), cudaMemcpyDeviceToHost, c->stream));
    RB200_CUDA(cudaStreamSynchronize(c->stream));
    if (c->h_cd->flags & VF_NONFINITE) return RB200_NONFINITE_INPUT;
    if (c->h_cd->flags & VF_WALL) return RB200_NONZERO_WALL_VELOCITY;
    double r = 0.0;
    for (int d = 0; d < 3; ++d) r += c->h_cd->scalars[d] / g.h[d];
    c->h_cd->rate = r;
    c->h_cd->time = 0.0;
    c->h_cd->generation = 0;
    c->h_cd->status = RB200_OK;
    c->h_cd->flags = 0;
    // a new accepted state has no accepted pressure: the next seeded step
    // starts cold (PressureColdReason::Invalidated, src/pressure_initialization.rs:31-36)
    c->h_cd->history = 0;
    RB200_CUDA(cudaMemcpyAsync(c->cd, c->h_cd, sizeof(CarrierDev), cudaMemcpyHostToDevice, c->stream));
    if (c->lq_h) {
        // the liquid state keeps its fraction and stamp; its clock follows the
        // carrier's, which a new accepted state restarts at zero
        c->lq_h->time = 0.0;
        RB200_CUDA(cudaMemcpyAsync(c->lq_d, c->lq_h, sizeof(LiquidDev), cudaMemcpyHostToDevice, c->stream));
    }
    RB200_CUDA(cudaStreamSynchronize(c->stream));
    return RB200_OK;
}

}  // namespace

extern "C" {

int rb200_carrier_create(const rb200_carrier_config* config, rb200_carrier** out) {
    if (!config || !out) return RB200_INVALID_ARGUMENT;
    *out = nullptr;
    GridDev g;
    int rc = make_grid_dev(&config->grid, config->density, &g);
    if (rc) return rc;
    if (config->storage != RB200_FACES_F32 && config->storage != RB200_FACES_F64) return RB200_INVALID_ARGUMENT;
    if (!settings_valid(&config->settings)) return RB200_INVALID_ARGUMENT;
    if (!(config->max_courant > 0.0) || !std::isfinite(config->actual_divergence_limit)) return RB200_INVALID_ARGUMENT;
    if ((rc = select_carrier_device(config->device))) return rc;
    std::unique_ptr<rb200_carrier> c(new (std::nothrow) rb200_carrier());
    if (!c) return RB200_OUT_OF_MEMORY;
    c->cfg = *config;
    c->g = g;
    c->device = config->device;
    c->elem = config->storage == RB200_FACES_F32 ? 4 : 8;
    RB200_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    RB200_CUDA(cudaStreamCreateWithFlags(&c->body_stream, cudaStreamNonBlocking));
    for (int b = 0; b < 3; ++b)
        for (int a = 0; a < 3; ++a) {
            if (cudaMalloc(&c->faces[b][a], size_t(g.flen[a]) * c->elem) != cudaSuccess) return RB200_OUT_OF_MEMORY;
            c->bytes += size_t(g.flen[a]) * c->elem;
            RB200_CUDA(cudaMemsetAsync(c->faces[b][a], 0, size_t(g.flen[a]) * c->elem, c->stream));
        }
    if (config->with_tracer)
        for (int t = 0; t < 2; ++t) {
            if (cudaMalloc(&c->tracer[t], size_t(g.cells) * 4) != cudaSuccess) return RB200_OUT_OF_MEMORY;
            c->bytes += size_t(g.cells) * 4;
            RB200_CUDA(cudaMemsetAsync(c->tracer[t], 0, size_t(g.cells) * 4, c->stream));
        }
    if (config->warm_start != 0 && config->warm_start != 1) return RB200_INVALID_ARGUMENT;
    if (config->warm_start) {
        if (cudaMalloc(&c->accepted_p, size_t(g.cells) * sizeof(double)) != cudaSuccess) return RB200_OUT_OF_MEMORY;
        c->bytes += size_t(g.cells) * sizeof(double);
    }
    RB200_CUDA(cudaMalloc(&c->cd, sizeof(CarrierDev)));
    RB200_CUDA(cudaMallocHost(&c->h_cd, sizeof(CarrierDev)));
    std::memset(c->h_cd, 0, sizeof(CarrierDev));
    c->h_cd->warm_policy = config->warm_start;
    c->h_cd->accepted_p = c->accepted_p;
    for (int b = 0; b < 3; ++b)
        for (int a = 0; a < 3; ++a) c->h_cd->faces[b][a] = c->faces[b][a];
    c->h_cd->tracer[0] = c->tracer[0];
    c->h_cd->tracer[1] = c->tracer[1];
    c->h_cd->max_courant = config->max_courant;
    c->h_cd->divergence_limit = config->actual_divergence_limit;
    c->h_cd->status = RB200_OK;
    RB200_CUDA(cudaMemcpyAsync(c->cd, c->h_cd, sizeof(CarrierDev), cudaMemcpyHostToDevice, c->stream));
    for (auto& e : c->ev) RB200_CUDA(cudaEventCreate(&e));
    if ((rc = c->solver.init(g, config->method, c->stream))) return rc;
    c->bytes += c->solver.bytes();
    RB200_CUDA(cudaStreamSynchronize(c->stream));
    rc = c->elem == 4 ? capture_step<float>(c.get()) : capture_step<double>(c.get());
    if (rc) return rc;
    *out = c.release();
    return RB200_OK;
}

void rb200_carrier_destroy(rb200_carrier* carrier) { delete carrier; }
uint64_t rb200_carrier_allocated_bytes(const rb200_carrier* carrier) { return carrier ? carrier->bytes : 0; }
void* rb200_carrier_stream(rb200_carrier* carrier) { return carrier ? (void*)carrier->stream : nullptr; }

int rb200_carrier_upload(rb200_carrier* carrier, const void* u, const void* v, const void* w, const float* tracer) {
    if (!carrier || !u || !v || !w) return RB200_INVALID_ARGUMENT;
    rb200_carrier* c = carrier;
    if (c->in_flight) return RB200_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    const int a = c->h_cd->acc;
    const void* src[3] = {u, v, w};
    for (int d = 0; d < 3; ++d)
        RB200_CUDA(cudaMemcpyAsync(c->faces[a][d], src[d], size_t(c->g.flen[d]) * c->elem, cudaMemcpyDefault,
                                   c->stream));
    if (tracer) {
        if (!c->tracer[0]) return RB200_INVALID_ARGUMENT;
        RB200_CUDA(cudaMemcpyAsync(c->tracer[c->h_cd->tacc], tracer, size_t(c->g.cells) * 4, cudaMemcpyDefault,
                                   c->stream));
    }
    return upload_rate(c);
}

int rb200_carrier_init_fourier(rb200_carrier* carrier, uint64_t seed, int modes, const double* k, const double* phase,
                               const double* amp, double amplitude, double noise) {
    if (!carrier || modes < 0 || modes > 8 || (modes > 0 && (!k || !phase || !amp))) return RB200_INVALID_ARGUMENT;
    rb200_carrier* c = carrier;
    if (c->in_flight) return RB200_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    FourierModes fm{};
    fm.modes = modes;
    for (int m = 0; m < modes; ++m) {
        for (int d = 0; d < 3; ++d) {
            fm.k[m][d] = k[3 * m + d];
            fm.amp[m][d] = amp[3 * m + d];
        }
        fm.phase[m] = phase[m];
    }
    fm.amplitude = amplitude;
    fm.noise = noise;
    fm.seed = seed;
    const GridDev& g = c->g;
    const long long faces = (long long)g.flen[0] + g.flen[1] + g.flen[2];
    const int fb = blocks_for(faces, 256, 148 * 64);
    if (c->elem == 4)
        k_fourier_init<float><<<fb, 256, 0, c->stream>>>(g, c->cd, fm);
    else
        k_fourier_init<double><<<fb, 256, 0, c->stream>>>(g, c->cd, fm);
    RB200_CUDA(cudaGetLastError());
    if (c->tracer[0]) RB200_CUDA(cudaMemsetAsync(c->tracer[c->h_cd->tacc], 0, size_t(g.cells) * 4, c->stream));
    return upload_rate(c);
}

int rb200_carrier_download(rb200_carrier* carrier, void* u, void* v, void* w, float* tracer) {
    if (!carrier) return RB200_INVALID_ARGUMENT;
    rb200_carrier* c = carrier;
    if (c->in_flight) return RB200_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    const int a = c->h_cd->acc;
    void* dst[3] = {u, v, w};
    for (int d = 0; d < 3; ++d)
        if (dst[d])
            RB200_CUDA(cudaMemcpyAsync(dst[d], c->faces[a][d], size_t(c->g.flen[d]) * c->elem, cudaMemcpyDefault,
                                       c->stream));
    if (tracer && c->tracer[0])
        RB200_CUDA(cudaMemcpyAsync(tracer, c->tracer[c->h_cd->tacc], size_t(c->g.cells) * 4, cudaMemcpyDefault,
                                   c->stream));
    RB200_CUDA(cudaStreamSynchronize(c->stream));
    return RB200_OK;
}

int rb200_carrier_state_device(rb200_carrier* carrier, void** u, void** v, void** w, float** tracer) {
    if (!carrier) return RB200_INVALID_ARGUMENT;
    const int a = carrier->h_cd->acc;
    if (u) *u = carrier->faces[a][0];
    if (v) *v = carrier->faces[a][1];
    if (w) *w = carrier->faces[a][2];
    if (tracer) *tracer = carrier->tracer[0] ? carrier->tracer[carrier->h_cd->tacc] : nullptr;
    return RB200_OK;
}

int rb200_carrier_pressure(rb200_carrier* carrier, double* out, size_t len) {
    if (!carrier || !out) return RB200_INVALID_ARGUMENT;
    if (len != size_t(carrier->g.cells)) return RB200_LENGTH_MISMATCH;
    cudaSetDevice(carrier->device);
    RB200_CUDA(cudaMemcpyAsync(out, carrier->solver.p(), len * sizeof(double), cudaMemcpyDeviceToHost,
                               carrier->stream));
    RB200_CUDA(cudaStreamSynchronize(carrier->stream));
    return RB200_OK;
}

int rb200_carrier_profile(rb200_carrier* carrier, int which, int launches, double* avg_ms) {
    if (!carrier || !avg_ms) return RB200_INVALID_ARGUMENT;
    if (carrier->in_flight) return RB200_INVALID_ARGUMENT;
    cudaSetDevice(carrier->device);
    return carrier->solver.profile(which, launches, avg_ms);
}

// Steps whose solve is the persistent (cooperative, grid-barrier) kernel are
// ordered one after another on each device: two such kernels never compete
// for co-residency. Other carriers' steps overlap freely.
static cudaEvent_t cooperative_lane(int device) {
    static std::mutex mu;
    static cudaEvent_t lanes[64] = {};
    if (device < 0 || device >= 64) return nullptr;
    std::lock_guard<std::mutex> lock(mu);
    if (!lanes[device] && cudaEventCreateWithFlags(&lanes[device], cudaEventDisableTiming) != cudaSuccess)
        lanes[device] = nullptr;
    return lanes[device];
}

static int launch_step(rb200_carrier* carrier, const rb200_step_params* params, int project_only);

int rb200_carrier_step_async(rb200_carrier* carrier, const rb200_step_params* params) {
    return launch_step(carrier, params, 0);
}

// ProjectionStepWorkspace::project (src/projection_step.rs:863-1033) on the
// resident state: the accepted faces are the provisional velocity, projected
// with the requested dt (build_rhs, the pressure solve, correction and the
// actual divergence gate) and committed as the new accepted state.
int rb200_carrier_project_async(rb200_carrier* carrier, const rb200_step_params* params) {
    if (!carrier || !params) return RB200_INVALID_ARGUMENT;
    if (params->cfl != 0.0 || params->buoyancy != 0.0 || carrier->tracer[0] || carrier->lq_d) {
        carrier->err = "a projection takes its dt as requested and carries no tracer or liquid state";
        return RB200_INVALID_ARGUMENT;
    }
    return launch_step(carrier, params, 1);
}

int rb200_carrier_project(rb200_carrier* carrier, const rb200_step_params* params, rb200_step_report* report) {
    if (!carrier || !params || !report) return RB200_INVALID_ARGUMENT;
    std::memset(report, 0, sizeof(*report));
    int rc = rb200_carrier_project_async(carrier, params);
    if (rc) return rc;
    return rb200_carrier_step_wait(carrier, report);
}

static int launch_step(rb200_carrier* carrier, const rb200_step_params* params, int project_only) {
    if (!carrier || !params) return RB200_INVALID_ARGUMENT;
    rb200_carrier* c = carrier;
    if (c->in_flight) return RB200_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    c->h_cd->project_only = project_only;
    // Step parameters into the device descriptor, then the step graph; both
    // ordered on the carrier's stream.
    c->h_cd->requested_dt = params->requested_dt;
    c->h_cd->cfl = params->cfl;
    c->h_cd->buoyancy = params->buoyancy;
    c->h_cd->iteration_limit_ok = params->iteration_limit_ok;
    c->h_cd->skip_gates = params->skip_gates;
    if (c->lq_d && !c->lq_inputs) {
        c->err = "liquid step: rb200_carrier_liquid_inputs has not been called";
        return RB200_INVALID_ARGUMENT;
    }
    RB200_CUDA(cudaMemcpyAsync(&c->cd->requested_dt, &c->h_cd->requested_dt,
                               offsetof(CarrierDev, max_courant) - offsetof(CarrierDev, requested_dt),
                               cudaMemcpyHostToDevice, c->stream));
    if (c->lq_d)
        RB200_CUDA(cudaMemcpyAsync(c->lflow_d, c->lflow_h, sizeof(LiquidFlowDev), cudaMemcpyHostToDevice, c->stream));
    cudaEvent_t lane = c->solver.persistent_blocks() ? cooperative_lane(c->device) : nullptr;
    if (c->solver.persistent_blocks() && !lane) return RB200_EXECUTION;
    if (lane) RB200_CUDA(cudaStreamWaitEvent(c->stream, lane, 0));
    RB200_CUDA(cudaEventRecord(c->ev[2], c->stream));
    RB200_CUDA(cudaGraphLaunch(c->step_exec, c->stream));
    RB200_CUDA(cudaEventRecord(c->ev[3], c->stream));
    if (lane) RB200_CUDA(cudaEventRecord(lane, c->stream));
    c->in_flight = true;
    return RB200_OK;
}

int rb200_carrier_step_poll(const rb200_carrier* carrier) {
    if (!carrier || !carrier->in_flight) return 0;
    cudaSetDevice(carrier->device);
    return cudaEventQuery(carrier->ev[3]) == cudaSuccess ? 1 : 0;
}

int rb200_carrier_step_wait(rb200_carrier* carrier, rb200_step_report* report) {
    if (!carrier || !report) return RB200_INVALID_ARGUMENT;
    rb200_carrier* c = carrier;
    if (!c->in_flight) return RB200_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    c->in_flight = false;
    RB200_CUDA(cudaStreamSynchronize(c->stream));
    const CarrierDev& h = *c->h_cd;
    *report = h.report;
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]) == cudaSuccess) report->pressure_ms = double(ms);
    report->kernel_launches = uint64_t(c->fixed_nodes) + uint64_t(h.trips) * uint64_t(c->solver.nodes_per_chunk());
    c->last_rejected = h.step_status != RB200_OK;
    if (!c->last_rejected) c->accepted_steps += 1;
    return h.step_status;
}

// LiquidTransportSimulation (src/liquid_step.rs:828-900) on the resident
// carrier: a liquid-volume state owned by the carrier, advanced in every step
// through the step's corrected faces and committed with it.
int rb200_carrier_attach_liquid(rb200_carrier* carrier, double density, rb200_liquid_stamp stamp,
                                uint64_t flow_id, const double* fraction, uint64_t limit,
                                rb200_liquid_report* error) {
    if (!carrier || !fraction) return RB200_INVALID_ARGUMENT;
    rb200_carrier* c = carrier;
    if (c->in_flight || c->lq_d) return RB200_INVALID_ARGUMENT;
    if (c->cfg.storage != RB200_FACES_F32) {
        c->err = "liquid step: needs f32 face storage (LiquidFlowInterval carries f32 velocities)";
        return RB200_UNSUPPORTED;
    }
    cudaSetDevice(c->device);
    if (cudaMallocHost(&c->lq_h, sizeof(LiquidDev)) != cudaSuccess ||
        cudaMallocHost(&c->lflow_h, sizeof(LiquidFlowDev)) != cudaSuccess ||
        cudaMallocHost(&c->lrep_h, sizeof(rb200_liquid_report)) != cudaSuccess ||
        cudaMalloc(&c->lflow_d, sizeof(LiquidFlowDev)) != cudaSuccess ||
        cudaMalloc(&c->lrep_d, sizeof(rb200_liquid_report)) != cudaSuccess) {
        cudaGetLastError();
        return RB200_OUT_OF_MEMORY;
    }
    std::memset(c->lflow_h, 0, sizeof(LiquidFlowDev));
    std::memset(c->lrep_h, 0, sizeof(rb200_liquid_report));
    LiquidDev* d = nullptr;
    int rc = liquid_state_create(c->g, density, stamp, c->h_cd->time, fraction, limit, c->lq_h, &d, &c->lq_sc,
                                 &c->lq_blocks, error, c->stream);
    if (rc) {
        liquid_state_free(c->lq_h, d, &c->lq_sc);
        cudaFreeHost(c->lq_h);
        c->lq_h = nullptr;
        return rc;
    }
    c->lq_d = d;
    RB200_CUDA(cudaMemsetAsync(c->lrep_d, 0, sizeof(rb200_liquid_report), c->stream));
    c->h_cd->liquid = c->lq_d;
    c->h_cd->lflow = c->lflow_d;
    c->h_cd->lrep = c->lrep_d;
    c->h_cd->flow_id = flow_id;
    RB200_CUDA(cudaMemcpyAsync(&c->cd->liquid, &c->h_cd->liquid,
                               offsetof(CarrierDev, flow_id) + sizeof(unsigned long long) - offsetof(CarrierDev, liquid),
                               cudaMemcpyHostToDevice, c->stream));
    c->bytes += 2ull * uint64_t(c->g.cells) * 8;
    RB200_CUDA(cudaStreamSynchronize(c->stream));
    // the step graph now holds the liquid interval
    if (c->step_exec) cudaGraphExecDestroy(c->step_exec);
    c->step_exec = nullptr;
    return capture_step<float>(c);
}

// LiquidStepInputs' inlet, source and volume settings (src/liquid_step.rs)
// for the following steps. source may be NULL; its rate is device memory that
// must stay valid while steps run.
int rb200_carrier_liquid_inputs(rb200_carrier* carrier, const rb200_liquid_inlet* inlet,
                                const rb200_liquid_source* source, const rb200_liquid_settings* settings) {
    if (!carrier || !inlet || !settings) return RB200_INVALID_ARGUMENT;
    rb200_carrier* c = carrier;
    if (!c->lq_d || c->in_flight) return RB200_INVALID_ARGUMENT;
    LiquidFlowDev& f = *c->lflow_h;
    f.inlet = inlet->stamp;
    for (int q = 0; q < 6; ++q) f.inlet_fraction[q] = inlet->fraction[q];
    f.src = source ? source->rate : nullptr;
    f.source = source ? source->stamp : rb200_liquid_stamp{0, 0};
    f.max_courant = settings->max_outward_courant;
    f.divergence_limit = settings->actual_divergence_limit;
    c->lq_inputs = true;
    return RB200_OK;
}

int rb200_carrier_liquid_report(const rb200_carrier* carrier, rb200_liquid_report* report) {
    if (!carrier || !report || !carrier->lq_d) return RB200_INVALID_ARGUMENT;
    if (carrier->in_flight) return RB200_INVALID_ARGUMENT;
    *report = *carrier->lrep_h;
    return RB200_OK;
}

int rb200_carrier_liquid_state(const rb200_carrier* carrier, const double** fraction, rb200_liquid_stamp* stamp,
                               double* time) {
    if (!carrier || !carrier->lq_d || carrier->in_flight) return RB200_INVALID_ARGUMENT;
    const LiquidDev& L = *carrier->lq_h;
    if (fraction) *fraction = L.frac[L.acc];
    if (stamp) *stamp = rb200_liquid_stamp{L.id, L.version};
    if (time) *time = L.time;
    return RB200_OK;
}

int rb200_carrier_liquid_download(rb200_carrier* carrier, double* out, size_t len) {
    if (!carrier || !out || !carrier->lq_d || carrier->in_flight) return RB200_INVALID_ARGUMENT;
    rb200_carrier* c = carrier;
    if (len != size_t(c->g.cells)) return RB200_LENGTH_MISMATCH;
    cudaSetDevice(c->device);
    RB200_CUDA(cudaMemcpyAsync(out, c->lq_h->frac[c->lq_h->acc], len * 8, cudaMemcpyDefault, c->stream));
    RB200_CUDA(cudaStreamSynchronize(c->stream));
    return RB200_OK;
}

int rb200_carrier_dense3d_fields(rb200_carrier* carrier, rb200_dense3d_fields* f) {
    if (!carrier || !f) return RB200_INVALID_ARGUMENT;
    rb200_carrier* c = carrier;
    if (c->in_flight) return RB200_INVALID_ARGUMENT;
    const int a = c->h_cd->acc;
    f->velocity_storage = c->cfg.storage;
    f->u = c->faces[a][0];
    f->v = c->faces[a][1];
    f->w = c->faces[a][2];
    f->tracer = c->tracer[0] ? c->tracer[c->h_cd->tacc] : nullptr;
    f->fraction = c->lq_h ? c->lq_h->frac[c->lq_h->acc] : nullptr;
    if (c->accepted_steps == 0) {
        f->pressure = nullptr;
    } else if (c->accepted_p) {
        f->pressure = c->accepted_p;
    } else if (!c->last_rejected) {
        f->pressure = c->solver.p();
    } else {
        c->err = "dense3D export: InvalidState(\"no accepted pressure after a rejected step\")";
        return RB200_DENSE3D_INVALID_STATE;
    }
    return RB200_OK;
}

int rb200_carrier_step(rb200_carrier* carrier, const rb200_step_params* params, rb200_step_report* report,
                       rb200_cancel_fn cancelled, void* ctx) {
    if (!carrier || !params || !report) return RB200_INVALID_ARGUMENT;
    std::memset(report, 0, sizeof(*report));
    if (cancelled && cancelled(ctx)) return RB200_CANCELLED;
    int rc = rb200_carrier_step_async(carrier, params);
    if (rc) return rc;
    return rb200_carrier_step_wait(carrier, report);
}

int rb200_carriers_step(rb200_carrier* const* carriers, size_t count, const rb200_step_params* params,
                        rb200_step_report* reports, int* statuses) {
    if (!carriers || !params || !reports || !statuses) return RB200_INVALID_ARGUMENT;
    int first_error = RB200_OK;
    for (size_t i = 0; i < count; ++i) {
        statuses[i] = rb200_carrier_step_async(carriers[i], &params[i]);
        if (statuses[i] && !first_error) first_error = statuses[i];
    }
    for (size_t i = 0; i < count; ++i) {
        if (statuses[i]) continue;
        statuses[i] = rb200_carrier_step_wait(carriers[i], &reports[i]);
    }
    return first_error;
}

}  // extern "C"
