// extern "C" entry points of librheon_b200 (declared in include/rheon_b200.h).
#include <algorithm>
#include <cmath>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "internal.hpp"
#include "pcg.hpp"

namespace rb200 {

static thread_local std::string g_error;
void set_error(const std::string& msg) { g_error = msg; }
const char* get_error() { return g_error.c_str(); }

int launch_check_finite(const double* x, int n, int* flags, cudaStream_t s);

int select_device(int device) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        set_error("no CUDA device");
        return RB200_NO_DEVICE;
    }
    if (device < 0 || device >= count) {
        set_error("device ordinal out of range");
        return RB200_INVALID_ARGUMENT;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return RB200_NO_DEVICE;
    if (prop.major != 10) {
        set_error("librheon_b200 is built for sm_100a (B200) only");
        return RB200_NO_DEVICE;
    }
    if (cudaSetDevice(device) != cudaSuccess) return RB200_NO_DEVICE;
    return RB200_OK;
}

}  // namespace rb200

using namespace rb200;

namespace {

// Flags word for the stream-ordered primitive entry points.
struct FlagsScope {
    int* d = nullptr;
    cudaStream_t s;
    explicit FlagsScope(cudaStream_t stream) : s(stream) {}
    int open() {
        RB200_CUDA(cudaMallocAsync(&d, sizeof(int), s));
        RB200_CUDA(cudaMemsetAsync(d, 0, sizeof(int), s));
        return RB200_OK;
    }
    int close(int* out) {
        int h = 0;
        RB200_CUDA(cudaMemcpyAsync(&h, d, sizeof(int), cudaMemcpyDeviceToHost, s));
        RB200_CUDA(cudaFreeAsync(d, s));
        d = nullptr;
        RB200_CUDA(cudaStreamSynchronize(s));
        *out = h;
        return RB200_OK;
    }
    ~FlagsScope() {
        if (d) cudaFreeAsync(d, s);
    }
};

}  // namespace

// ---------------------------------------------------------------- handles
struct rb200_workspace {
    int device = 0;
    cudaStream_t stream = nullptr;
    GridDev g{};
    rb200_grid grid{};
    int method = 0;
    uint64_t limit = 0;
    PcgSolver solver;
    std::string err;
    ~rb200_workspace() {
        if (stream) {
            cudaSetDevice(device);
            cudaStreamSynchronize(stream);
            cudaStreamDestroy(stream);
        }
    }
};

struct rb200_provider {
    rb200_provider_config cfg{};
    rb200_workspace* ws = nullptr;
    std::string err;
    rb200_report last{};
    int last_status = RB200_OK;
    ~rb200_provider() { delete ws; }
};

#define RB200_PRIM_BEGIN(grid, density)                 \
    GridDev g;                                          \
    int rc = make_grid_dev(grid, density, &g);          \
    if (rc) return rc;                                  \
    cudaStream_t s = (cudaStream_t)stream;              \
    FlagsScope fl(s);                                   \
    if ((rc = fl.open())) return rc;

static int flags_status(int flags, bool walls_matter) {
    if (flags & VF_NONFINITE) return RB200_NONFINITE_INPUT;
    if (walls_matter && (flags & VF_WALL)) return RB200_NONZERO_WALL_VELOCITY;
    if (flags & (VF_ARITH | VF_F32_RANGE)) return RB200_ARITHMETIC_FAILURE;
    return RB200_OK;
}

template <class T>
static int build_rhs_prim(const rb200_grid* grid, double density, const T* u, const T* v, const T* w, double dt,
                          double* rhs, void* stream) {
    if (!std::isfinite(dt) || dt <= 0.0) return RB200_INVALID_ARGUMENT;
    RB200_PRIM_BEGIN(grid, density)
    if ((rc = launch_validate_faces<T>(g, u, v, w, fl.d, s))) return rc;
    if ((rc = launch_build_rhs<T>(g, u, v, w, dt, rhs, fl.d, s))) return rc;
    int f = 0;
    if ((rc = fl.close(&f))) return rc;
    return flags_status(f, true);
}

template <class T>
static int divergence_prim(const rb200_grid* grid, const T* u, const T* v, const T* w, double* out, void* stream) {
    RB200_PRIM_BEGIN(grid, 1.0)
    if ((rc = launch_validate_faces<T>(g, u, v, w, fl.d, s))) return rc;
    if ((rc = launch_divergence<T>(g, u, v, w, out, fl.d, s))) return rc;
    int f = 0;
    if ((rc = fl.close(&f))) return rc;
    return flags_status(f, true);
}

template <class T>
static int correct_prim(const rb200_grid* grid, double density, const double* p, double dt, T* u, T* v, T* w,
                        void* stream) {
    if (!std::isfinite(dt) || dt <= 0.0) return RB200_INVALID_ARGUMENT;
    RB200_PRIM_BEGIN(grid, density)
    if ((rc = launch_validate_faces<T>(g, u, v, w, fl.d, s))) return rc;
    if ((rc = launch_check_finite(p, g.cells, fl.d, s))) return rc;
    int f = 0;
    if ((rc = fl.close(&f))) return rc;
    if ((rc = flags_status(f, true))) return rc;
    FlagsScope fl2(s);
    if ((rc = fl2.open())) return rc;
    if ((rc = launch_correct<T>(g, p, dt, u, v, w, fl2.d, s))) return rc;
    if ((rc = fl2.close(&f))) return rc;
    return flags_status(f, true);
}

template <class T>
static int advect_prim(const rb200_grid* grid, const T* u, const T* v, const T* w, double dt, T* ou, T* ov, T* ow,
                       void* stream) {
    if (!std::isfinite(dt) || dt <= 0.0) return RB200_INVALID_ARGUMENT;
    RB200_PRIM_BEGIN(grid, 1.0)
    if ((rc = launch_validate_faces<T>(g, u, v, w, fl.d, s))) return rc;
    int f = 0;
    if ((rc = fl.close(&f))) return rc;
    if (f & VF_NONFINITE) return RB200_NONFINITE_INPUT;
    FlagsScope fl2(s);
    if ((rc = fl2.open())) return rc;
    if ((rc = launch_advect_velocity<T>(g, u, v, w, dt, ou, ov, ow, nullptr, 0.0, fl2.d, s))) return rc;
    if ((rc = fl2.close(&f))) return rc;
    return flags_status(f, false);
}


template <class T>
static int witness_prim(const rb200_grid* grid, double density, const double* pressure, double dt, const T* iu,
                        const T* iv, const T* iw, const T* su, const T* sv, const T* sw, int* axis, uint64_t* index,
                        void* stream) {
    if (!pressure || !iu || !iv || !iw || !su || !sv || !sw) return RB200_INVALID_ARGUMENT;
    if (axis) *axis = -1;
    if (index) *index = 0;
    if (!std::isfinite(dt) || dt <= 0.0) return RB200_INVALID_ARGUMENT;
    RB200_PRIM_BEGIN(grid, density)
    // validate_cells(pressure), validate_velocity(supplied) (projection.rs:521-526)
    if ((rc = launch_check_finite(pressure, g.cells, fl.d, s))) return rc;
    if ((rc = launch_validate_faces<T>(g, su, sv, sw, fl.d, s))) return rc;
    if ((rc = launch_validate_faces<T>(g, iu, iv, iw, fl.d, s))) return rc;
    unsigned long long* first = nullptr;
    RB200_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&first), 3 * sizeof(unsigned long long), s));
    cudaMemsetAsync(first, 0xff, 3 * sizeof(unsigned long long), s);
    const T* in[3] = {iu, iv, iw};
    const T* sup[3] = {su, sv, sw};
    rc = launch_projection_witness<T>(g, pressure, dt, in, sup, first, s);
    unsigned long long h[3] = {0, 0, 0};
    if (!rc && cudaMemcpyAsync(h, first, sizeof(h), cudaMemcpyDeviceToHost, s) != cudaSuccess) rc = RB200_EXECUTION;
    cudaFreeAsync(first, s);
    int f = 0;
    int rc2 = fl.close(&f);
    if (rc) return rc;
    if (rc2) return rc2;
    if ((rc = flags_status(f, true))) return rc;
    for (int a = 0; a < 3; ++a)
        if (h[a] != ~0ull) {
            if (axis) *axis = a;
            if (index) *index = uint64_t(h[a]);
            return RB200_QUALITY_GATE;
        }
    return RB200_OK;
}


extern "C" {

int rb200_abi_version(void) { return RB200_ABI_VERSION; }

const char* rb200_status_string(int status) {
    switch (status) {
        case RB200_OK: return "ok";
        case RB200_UNSUPPORTED: return "unsupported request";
        case RB200_EXECUTION: return "execution failed";
        case RB200_NONFINITE_OUTPUT: return "nonfinite output";
        case RB200_NONZERO_GAUGE: return "nonzero gauge";
        case RB200_QUALITY_GATE: return "quality gate";
        case RB200_CANCELLED: return "cancelled";
        case RB200_ITERATION_LIMIT: return "pressure iteration limit";
        case RB200_BREAKDOWN: return "pressure arithmetic broke down";
        case RB200_OUT_OF_MEMORY: return "device allocation failed";
        case RB200_INVALID_ARGUMENT: return "invalid argument";
        case RB200_INCOMPATIBLE_RHS: return "sealed-domain RHS sum exceeds rounding budget";
        case RB200_NONFINITE_INPUT: return "field contains a nonfinite value";
        case RB200_NONZERO_WALL_VELOCITY: return "fixed wall velocity is nonzero";
        case RB200_ARITHMETIC_FAILURE: return "numerical operation produced a nonfinite value";
        case RB200_DIVERGENCE_LIMIT: return "actual divergence limit";
        case RB200_COURANT_LIMIT: return "Courant limit";
        case RB200_NO_DEVICE: return "no sm_100 device";
        case RB200_LENGTH_MISMATCH: return "field length does not match the grid";
        case RB200_INVALID_INITIAL_PRESSURE: return "initial pressure requires a sealed operator and zero gauge";
        case RB200_DENSE3D_INVALID_STATE: return "dense3D frame: invalid state";
        case RB200_DENSE3D_LIMIT: return "dense3D export limit";
        case RB200_DENSE3D_ABORTED: return "dense3D export aborted";
        case RB200_DENSE3D_IO: return "dense3D output error";
        case RB200_LIQUID_REJECTED: return "liquid volume transport rejected the operation";
        case RB200_BOX_FLUX_REJECTED: return "box flux projection rejected the operation";
        case RB200_SIMULATION_REJECTED: return "simulation rejected the step";
        default: return "unknown status";
    }
}

int rb200_device_count(void) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess) return 0;
    int n = 0;
    for (int d = 0; d < count; ++d) {
        cudaDeviceProp prop;
        if (cudaGetDeviceProperties(&prop, d) == cudaSuccess && prop.major == 10) ++n;
    }
    return n;
}

// ---------------------------------------------------------------- workspace
int rb200_workspace_create(const rb200_grid* grid, double density, int method, uint64_t memory_limit,
                           int device, rb200_workspace** out) {
    if (!out) return RB200_INVALID_ARGUMENT;
    *out = nullptr;
    GridDev g;
    int rc = make_grid_dev(grid, density, &g);
    if (rc) {
        set_error("invalid grid or density");
        return rc;
    }
    if (method < RB200_JACOBI_PCG_V1 || method > RB200_MG_MIXED) {
        set_error("method not available on the device");
        return RB200_UNSUPPORTED;
    }
    // Six f64 cell arrays (b, p, r, two directions, z), q and the FP32
    // hierarchy (about 5.2 bytes per fine cell) for multigrid, plus partials.
    uint64_t need = uint64_t(g.cells) * (method == RB200_MG_MIXED ? 62 : 48);
    if (need > memory_limit) {
        set_error("device buffers exceed the memory limit");
        return RB200_OUT_OF_MEMORY;
    }
    if ((rc = select_device(device))) return rc;
    std::unique_ptr<rb200_workspace> ws(new (std::nothrow) rb200_workspace());
    if (!ws) return RB200_OUT_OF_MEMORY;
    ws->device = device;
    ws->g = g;
    ws->grid = *grid;
    ws->method = method;
    ws->limit = memory_limit;
    RB200_CUDA(cudaStreamCreateWithFlags(&ws->stream, cudaStreamNonBlocking));
    if ((rc = ws->solver.init(g, method, ws->stream))) return rc;
    *out = ws.release();
    return RB200_OK;
}

void rb200_workspace_destroy(rb200_workspace* ws) { delete ws; }

uint64_t rb200_workspace_allocated_bytes(const rb200_workspace* ws) { return ws ? ws->solver.bytes() : 0; }

void* rb200_workspace_stream(rb200_workspace* ws) { return ws ? (void*)ws->stream : nullptr; }

static int workspace_solve(rb200_workspace* ws, const double* rhs, bool on_device, size_t len, double dt,
                           const rb200_settings* settings, rb200_report* report, rb200_cancel_fn cancelled,
                           void* ctx, const double* initial = nullptr) {
    if (!ws || !rhs || !settings) return RB200_INVALID_ARGUMENT;
    if (report) std::memset(report, 0, sizeof(*report));
    if (len != size_t(ws->g.cells)) return RB200_LENGTH_MISMATCH;
    cudaSetDevice(ws->device);
    if (!std::isfinite(dt) || dt <= 0.0 || !settings_valid(settings)) {
        // validate_cells(rhs) precedes the settings check (src/pressure.rs:373).
        if (!on_device)
            for (size_t i = 0; i < len; ++i)
                if (!std::isfinite(rhs[i])) return RB200_NONFINITE_INPUT;
        return RB200_INVALID_ARGUMENT;
    }
    if (cancelled && cancelled(ctx)) return RB200_CANCELLED;
    RB200_CUDA(cudaMemcpyAsync(ws->solver.b(), rhs, len * sizeof(double),
                               on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDefault, ws->stream));
    int rc = ws->solver.solve(dt, *settings, report, cancelled, ctx, initial);
    if (rc == RB200_EXECUTION) ws->err = get_error();
    return rc;
}

int rb200_workspace_solve_rhs(rb200_workspace* ws, const double* rhs, size_t len, double dt,
                              const rb200_settings* settings, rb200_report* report, rb200_cancel_fn cancelled,
                              void* ctx) {
    return workspace_solve(ws, rhs, false, len, dt, settings, report, cancelled, ctx);
}

int rb200_workspace_solve_rhs_initial(rb200_workspace* ws, const double* rhs, const double* initial, size_t len,
                                      double dt, const rb200_settings* settings, rb200_report* report,
                                      rb200_cancel_fn cancelled, void* ctx) {
    if (!initial) return RB200_INVALID_ARGUMENT;
    return workspace_solve(ws, rhs, false, len, dt, settings, report, cancelled, ctx, initial);
}

int rb200_workspace_solve_rhs_device(rb200_workspace* ws, const double* rhs_device, size_t len, double dt,
                                     const rb200_settings* settings, rb200_report* report,
                                     rb200_cancel_fn cancelled, void* ctx) {
    return workspace_solve(ws, rhs_device, true, len, dt, settings, report, cancelled, ctx);
}

int rb200_workspace_pressure(rb200_workspace* ws, double* out, size_t len) {
    if (!ws || !out) return RB200_INVALID_ARGUMENT;
    if (len != size_t(ws->g.cells)) return RB200_LENGTH_MISMATCH;
    cudaSetDevice(ws->device);
    RB200_CUDA(cudaMemcpyAsync(out, ws->solver.p(), len * sizeof(double), cudaMemcpyDeviceToHost, ws->stream));
    RB200_CUDA(cudaStreamSynchronize(ws->stream));
    return RB200_OK;
}

const double* rb200_workspace_pressure_device(rb200_workspace* ws) { return ws ? ws->solver.p() : nullptr; }

int rb200_workspace_set_trace(rb200_workspace* ws, rb200_trace* trace, size_t capacity) {
    if (!ws) return RB200_INVALID_ARGUMENT;
    cudaSetDevice(ws->device);
    return ws->solver.set_trace(trace, capacity);
}

int rb200_workspace_profile(rb200_workspace* ws, int which, int launches, double* avg_ms) {
    if (!ws || !avg_ms) return RB200_INVALID_ARGUMENT;
    cudaSetDevice(ws->device);
    return ws->solver.profile(which, launches, avg_ms);
}

// ---------------------------------------------------------------- provider
static const char* method_id(int method) {
    switch (method) {
        case RB200_JACOBI_PCG_V1: return "b200-jacobi-pcg-v1";
        case RB200_SGS_PCG_V1: return "b200-sgs-pcg-v1";
        case RB200_RBSGS_PCG: return "b200-rbsgs-pcg";
        default: return "b200-mg-mixed";
    }
}

int rb200_provider_create(const rb200_provider_config* config, rb200_provider** out) {
    if (!config || !out) return RB200_INVALID_ARGUMENT;
    *out = nullptr;
    if (!settings_valid(&config->settings)) return RB200_INVALID_ARGUMENT;
    std::unique_ptr<rb200_provider> p(new (std::nothrow) rb200_provider());
    if (!p) return RB200_OUT_OF_MEMORY;
    p->cfg = *config;
    int rc = rb200_workspace_create(&config->grid, config->density, config->method, UINT64_MAX, config->device,
                                    &p->ws);
    if (rc) return rc;
    *out = p.release();
    return RB200_OK;
}

void rb200_provider_destroy(rb200_provider* provider) { delete provider; }

int rb200_provider_metadata(const rb200_provider* provider, rb200_metadata* out) {
    if (!provider || !out) return RB200_INVALID_ARGUMENT;
    // Mirrors the sealed-box metadata of src/solver_provider/modal.rs:93-119.
    out->id = method_id(provider->cfg.method);
    out->version = "1";
    out->stage = "pressure";
    out->input_layout = "x-fastest-cell-centered";
    out->input_scalar = "f64";
    out->input_units = "m^3/s^2";
    out->output_layout = "x-fastest-cell-centered";
    out->output_scalar = "f64";
    out->output_units = "Pa";
    out->domain = "sealed constant-density MAC box";
    for (int d = 0; d < 3; ++d) out->shape_xyz[d] = provider->cfg.grid.counts[d];
    return RB200_OK;
}

int rb200_provider_supports(const rb200_provider* provider, const rb200_request* request) {
    if (!provider || !request) return RB200_INVALID_ARGUMENT;
    if (!same_grid(provider->cfg.grid, request->grid)) return RB200_UNSUPPORTED;
    if (request->density != provider->cfg.density) return RB200_UNSUPPORTED;
    if (request->len != size_t(provider->ws->g.cells)) return RB200_UNSUPPORTED;
    return RB200_OK;
}

int rb200_provider_predict(rb200_provider* provider, const rb200_request* request, double* pressure, size_t len,
                           rb200_cancel_fn cancelled, void* ctx) {
    if (!provider || !request || !pressure || !request->rhs) return RB200_INVALID_ARGUMENT;
    int rc = rb200_provider_supports(provider, request);
    if (rc) {
        provider->err = "request grid, density or length differs from the provider's";
        return rc;
    }
    if (len != request->len) {
        provider->err = "output length differs from the request";
        return RB200_UNSUPPORTED;
    }
    rc = rb200_workspace_solve_rhs(provider->ws, request->rhs, request->len, request->dt, &provider->cfg.settings,
                                   &provider->last, cancelled, ctx);
    provider->last_status = rc;
    if (rc == RB200_CANCELLED) return RB200_CANCELLED;
    if (rc != RB200_OK) {
        provider->err = std::string("device solve: ") + rb200_status_string(rc);
        return rc == RB200_UNSUPPORTED ? RB200_UNSUPPORTED : RB200_EXECUTION;
    }
    rc = rb200_workspace_pressure(provider->ws, pressure, len);
    if (rc) {
        provider->err = get_error();
        return RB200_EXECUTION;
    }
    for (size_t i = 0; i < len; ++i)
        if (!std::isfinite(pressure[i])) return RB200_NONFINITE_OUTPUT;
    provider->err.clear();
    return RB200_OK;
}

const char* rb200_provider_last_error(const rb200_provider* provider) {
    return provider ? provider->err.c_str() : get_error();
}

int rb200_provider_last_report(const rb200_provider* provider, rb200_report* out, int* solve_status) {
    if (!provider || !out) return RB200_INVALID_ARGUMENT;
    *out = provider->last;
    if (solve_status) *solve_status = provider->last_status;
    return RB200_OK;
}

// ---------------------------------------------------------------- primitives
int rb200_apply_full_device(const rb200_grid* grid, double density, const double* pressure, double* out,
                            void* stream) {
    RB200_PRIM_BEGIN(grid, density)
    if ((rc = launch_check_finite(pressure, g.cells, fl.d, s))) return rc;
    if ((rc = launch_apply_full(g, pressure, out, fl.d, s))) return rc;
    int f = 0;
    if ((rc = fl.close(&f))) return rc;
    return flags_status(f, false);
}


int rb200_qualify_pressure_device(const rb200_grid* grid, double density, const double* rhs,
                                  const double* pressure, size_t len, double dt, const rb200_settings* settings,
                                  rb200_report* report, void* stream) {
    if (!rhs || !pressure || !settings) return RB200_INVALID_ARGUMENT;
    if (report) std::memset(report, 0, sizeof(*report));
    if (!std::isfinite(dt) || dt <= 0.0 || !settings_valid(settings)) return RB200_INVALID_ARGUMENT;
    GridDev g;
    int rc = make_grid_dev(grid, density, &g);
    if (rc) return rc;
    if (len != size_t(g.cells)) return RB200_LENGTH_MISMATCH;
    cudaStream_t s = (cudaStream_t)stream;
    const size_t nb = size_t(precondition_partials_blocks());
    const size_t bytes = (4 * nb + 5) * sizeof(double) + sizeof(unsigned);
    char* scratch = nullptr;
    RB200_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&scratch), bytes, s));
    Partials part{reinterpret_cast<double*>(scratch), reinterpret_cast<unsigned*>(scratch + (4 * nb + 5) * 8)};
    double* out = part.data + 4 * nb;
    cudaMemsetAsync(part.ticket, 0, sizeof(unsigned), s);
    rc = launch_qualify_pressure(g, rhs, pressure, part, out, s);
    double h[5] = {0, 0, 0, 0, 0};
    if (!rc && cudaMemcpyAsync(h, out, sizeof(h), cudaMemcpyDeviceToHost, s) != cudaSuccess) rc = RB200_EXECUTION;
    cudaFreeAsync(scratch, s);
    if (!rc && cudaStreamSynchronize(s) != cudaSuccess) rc = RB200_EXECUTION;
    if (rc) return rc;
    // the order of the reference's checks: non-finite output, gauge, product
    if (h[3] == 1.0) return RB200_NONFINITE_OUTPUT;
    if (h[4] != 0.0) return RB200_NONZERO_GAUGE;
    if (h[3] != 0.0) return RB200_NONFINITE_OUTPUT;
    const double l2 = std::sqrt(h[0]);
    const double threshold = std::fmax(settings->absolute_residual, settings->relative_residual * std::sqrt(h[1]));
    const double divergence = h[2] * dt / g.volume;
    if (report) {
        report->true_residual_l2 = l2;
        report->true_residual_max = h[2];
        report->predicted_divergence_max = divergence;
    }
    if (!std::isfinite(l2) || !std::isfinite(divergence) || l2 > threshold || divergence > settings->divergence_limit)
        return RB200_QUALITY_GATE;
    return RB200_OK;
}

int rb200_projection_witness_f32_device(const rb200_grid* grid, double density, const double* pressure, double dt,
                                        const float* u, const float* v, const float* w, const float* su,
                                        const float* sv, const float* sw, int* axis, uint64_t* index, void* stream) {
    return witness_prim<float>(grid, density, pressure, dt, u, v, w, su, sv, sw, axis, index, stream);
}

int rb200_projection_witness_f64_device(const rb200_grid* grid, double density, const double* pressure, double dt,
                                        const double* u, const double* v, const double* w, const double* su,
                                        const double* sv, const double* sw, int* axis, uint64_t* index,
                                        void* stream) {
    return witness_prim<double>(grid, density, pressure, dt, u, v, w, su, sv, sw, axis, index, stream);
}

int rb200_precondition_jacobi_device(const rb200_grid* grid, double density, const double* r, double* z, size_t len,
                                     double* rz, void* stream) {
    if (!r || !z || !rz) return RB200_INVALID_ARGUMENT;
    RB200_PRIM_BEGIN(grid, density)
    if (len != size_t(g.cells)) return RB200_LENGTH_MISMATCH;
    if ((rc = launch_check_finite(r, g.cells, fl.d, s))) return rc;
    // scratch: partials [blocks][2], the result, the ticket
    const size_t nb = size_t(precondition_partials_blocks());
    const size_t bytes = (2 * nb + 1) * sizeof(double) + sizeof(unsigned);
    char* scratch = nullptr;
    RB200_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&scratch), bytes, s));
    Partials part{reinterpret_cast<double*>(scratch), reinterpret_cast<unsigned*>(scratch + (2 * nb + 1) * 8)};
    double* rz_dev = part.data + 2 * nb;
    cudaMemsetAsync(part.ticket, 0, sizeof(unsigned), s);
    rc = launch_precondition_jacobi(g, r, z, part, rz_dev, s);
    double h = 0.0;
    if (!rc && cudaMemcpyAsync(&h, rz_dev, sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess)
        rc = RB200_EXECUTION;
    cudaFreeAsync(scratch, s);
    if (rc) return rc;
    int f = 0;
    if ((rc = fl.close(&f))) return rc;
    *rz = h;
    return flags_status(f, false);
}

int rb200_build_rhs_f32_device(const rb200_grid* grid, double density, const float* u, const float* v,
                               const float* w, double dt, double* rhs, void* stream) {
    return build_rhs_prim<float>(grid, density, u, v, w, dt, rhs, stream);
}
int rb200_build_rhs_f64_device(const rb200_grid* grid, double density, const double* u, const double* v,
                               const double* w, double dt, double* rhs, void* stream) {
    return build_rhs_prim<double>(grid, density, u, v, w, dt, rhs, stream);
}


int rb200_divergence_f32_device(const rb200_grid* grid, const float* u, const float* v, const float* w, double* out,
                                void* stream) {
    return divergence_prim<float>(grid, u, v, w, out, stream);
}
int rb200_divergence_f64_device(const rb200_grid* grid, const double* u, const double* v, const double* w,
                                double* out, void* stream) {
    return divergence_prim<double>(grid, u, v, w, out, stream);
}


int rb200_correct_f32_device(const rb200_grid* grid, double density, const double* pressure, double dt, float* u,
                             float* v, float* w, void* stream) {
    return correct_prim<float>(grid, density, pressure, dt, u, v, w, stream);
}
int rb200_correct_f64_device(const rb200_grid* grid, double density, const double* pressure, double dt, double* u,
                             double* v, double* w, void* stream) {
    return correct_prim<double>(grid, density, pressure, dt, u, v, w, stream);
}


int rb200_advect_velocity_f32_device(const rb200_grid* grid, const float* u, const float* v, const float* w,
                                     double dt, float* ou, float* ov, float* ow, void* stream) {
    return advect_prim<float>(grid, u, v, w, dt, ou, ov, ow, stream);
}
int rb200_advect_velocity_f64_device(const rb200_grid* grid, const double* u, const double* v, const double* w,
                                     double dt, double* ou, double* ov, double* ow, void* stream) {
    return advect_prim<double>(grid, u, v, w, dt, ou, ov, ow, stream);
}

int rb200_advect_tracer_f32_device(const rb200_grid* grid, const float* old, const float* u, const float* v,
                                   const float* w, double dt, float* out, void* stream) {
    if (!std::isfinite(dt) || dt <= 0.0) return RB200_INVALID_ARGUMENT;
    RB200_PRIM_BEGIN(grid, 1.0)
    if ((rc = launch_validate_faces<float>(g, u, v, w, fl.d, s))) return rc;
    int f = 0;
    if ((rc = fl.close(&f))) return rc;
    if (f & VF_NONFINITE) return RB200_NONFINITE_INPUT;
    FlagsScope fl2(s);
    if ((rc = fl2.open())) return rc;
    if ((rc = launch_advect_tracer<float>(g, old, u, v, w, dt, out, fl2.d, s))) return rc;
    if ((rc = fl2.close(&f))) return rc;
    return flags_status(f, false);
}

}  // extern "C"
