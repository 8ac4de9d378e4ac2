/*
 * rheon_b200 — C ABI of the B200 (sm_100a) fixed-box carrier step.
 *
 * Plain pointers and sizes only. Host pointers are borrowed for the duration
 * of a call; device pointers (the *_device entry points) must be CUDA device
 * allocations on the handle's device. Every handle owns one CUDA stream and is
 * not thread-safe: one caller thread at a time, as Rheon's `&mut self` traits.
 *
 * Reference interfaces replaced (paths within the Rheon project):
 *   PressureProvider trait ............ src/solver_provider.rs:67-76
 *   PressureRequest ................... src/solver_provider.rs:47-52
 *   ProviderRejection ................. src/solver_provider.rs:55-62
 *   PressureWorkspace::solve_rhs ...... src/pressure.rs:365-393
 *   PressureWorkspace::solve_velocity . src/pressure.rs:344-361
 *   PressureSettings / PressureReport . src/pressure.rs:34-49
 *   PressureError ..................... src/pressure.rs:52-77
 *   PressureOperator primitives ....... src/operator.rs:378-781
 *   advect_velocity / advect_tracer ... src/advection.rs:28-102
 *   Simulation step owner (composed) .. src/simulation.rs:812-1403
 */
#ifndef RHEON_B200_H
#define RHEON_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RB200_ABI_VERSION 1

#if defined(__GNUC__)
#define RB200_API __attribute__((visibility("default")))
#else
#define RB200_API
#endif

/* Status codes. 1-6 map one to one onto ProviderRejection
 * (src/solver_provider.rs:55-62); 7-11 onto PressureError
 * (src/pressure.rs:52-77); 12-16 onto OperatorError / SimulationError gates. */
typedef enum rb200_status {
    RB200_OK = 0,
    RB200_UNSUPPORTED = 1,           /* ProviderRejection::Unsupported            */
    RB200_EXECUTION = 2,             /* ProviderRejection::Execution (CUDA error) */
    RB200_NONFINITE_OUTPUT = 3,      /* ProviderRejection::NonFiniteOutput        */
    RB200_NONZERO_GAUGE = 4,         /* ProviderRejection::NonZeroGauge           */
    RB200_QUALITY_GATE = 5,          /* ProviderRejection::QualityGate            */
    RB200_CANCELLED = 6,             /* ProviderRejection::Cancelled              */
    RB200_ITERATION_LIMIT = 7,       /* PressureError::IterationLimit             */
    RB200_BREAKDOWN = 8,             /* PressureError::Breakdown                  */
    RB200_OUT_OF_MEMORY = 9,         /* PressureError::AllocationFailed/BufferLimit */
    RB200_INVALID_ARGUMENT = 10,     /* PressureError::InvalidSettings, bad dt... */
    RB200_INCOMPATIBLE_RHS = 11,     /* PressureError::IncompatibleRhs            */
    RB200_NONFINITE_INPUT = 12,      /* OperatorError::NonFiniteInput             */
    RB200_NONZERO_WALL_VELOCITY = 13,/* OperatorError::NonZeroWallVelocity        */
    RB200_ARITHMETIC_FAILURE = 14,   /* OperatorError::ArithmeticFailure          */
    RB200_DIVERGENCE_LIMIT = 15,     /* SimulationError::DivergenceLimit          */
    RB200_COURANT_LIMIT = 16,        /* SimulationError::CourantLimit             */
    RB200_NO_DEVICE = 17,            /* no usable sm_100 device                   */
    RB200_LENGTH_MISMATCH = 18,      /* OperatorError::LengthMismatch             */
    RB200_INVALID_INITIAL_PRESSURE = 22,/* PressureError::InvalidInitialPressure  */
    RB200_DENSE3D_INVALID_STATE = 23,/* Dense3dError::InvalidState (src/dense3d_sequence.rs:21-27) */
    RB200_DENSE3D_LIMIT = 24,        /* Dense3dError::Limit                       */
    RB200_DENSE3D_ABORTED = 25,      /* Dense3dError::Aborted                     */
    RB200_DENSE3D_IO = 26,           /* Dense3dError::Io                          */
    RB200_LIQUID_REJECTED = 27,      /* LiquidVolumeError: see rb200_liquid_report.error */
    RB200_BOX_FLUX_REJECTED = 28,    /* BoxFluxError's own variants: see rb200_box_flux_report.error */
    RB200_SIMULATION_REJECTED = 29   /* SimulationError's own variants: see rb200_forced_step_report.error */
} rb200_status;

/* Pressure methods. JACOBI_PCG_V1 reproduces "jacobi-pcg-v1"
 * (src/pressure.rs:7-29). SGS_PCG_V1 reproduces the exact lexicographic
 * "sgs-pcg-v1" sweep order. RBSGS_PCG is the device-native red-black symmetric
 * Gauss-Seidel preconditioner (new). MG_MIXED is flexible CG with an FP32
 * geometric multigrid V(2,2) preconditioner, FP64 residual/accumulation and an
 * FP64 coarse solve (new). */
typedef enum rb200_method {
    RB200_JACOBI_PCG_V1 = 0,
    RB200_SGS_PCG_V1 = 1,
    RB200_RBSGS_PCG = 2,
    RB200_MG_MIXED = 3
} rb200_method;

/* Face storage of the resident carrier state. F32 is Rheon's own storage
 * (src/simulation.rs:167-172); F64 keeps the same formulas without the casts. */
typedef enum rb200_storage { RB200_FACES_F32 = 0, RB200_FACES_F64 = 1 } rb200_storage;

/* GridGeometry::new(counts, spacing, origin) (src/geometry.rs:114). */
typedef struct rb200_grid {
    uint64_t counts[3];
    double spacing[3];
    double origin[3];
} rb200_grid;

/* PressureSettings (src/pressure.rs:34-39). */
typedef struct rb200_settings {
    double relative_residual;
    double absolute_residual;
    double divergence_limit;
    uint64_t max_iterations;
} rb200_settings;

/* PressureReport (src/pressure.rs:44-49) plus the typed-error payloads. */
typedef struct rb200_report {
    uint64_t iterations;
    double true_residual_l2;
    double true_residual_max;
    double predicted_divergence_max;
    double incompatible_sum;      /* IncompatibleRhs { sum, .. }             */
    double incompatible_budget;   /* IncompatibleRhs { .., rounding_budget } */
    uint64_t breakdown_iteration; /* Breakdown { iteration }                 */
} rb200_report;

/* One PCG iteration's scalars (diagnostics / per-iteration parity). */
typedef struct rb200_trace {
    double curvature;
    double alpha;
    double recursive_l2;
    double rz;
    double beta;
    uint32_t replaced;
    uint32_t checked;
} rb200_trace;

/* Cancellation predicate, polled on the caller thread between device chunks.
 * Nonzero return cancels (never falls back), as `cancelled: &mut dyn FnMut()
 * -> bool` in src/solver_provider.rs:70-75. */
typedef int (*rb200_cancel_fn)(void* ctx);

/* ------------------------------------------------------------------ library */
RB200_API int rb200_abi_version(void);
/* Static message for a status code. */
RB200_API const char* rb200_status_string(int status);
/* Number of visible sm_100 devices (0 when none). */
RB200_API int rb200_device_count(void);

/* ------------------------------------------------- PressureProvider drop-in
 * rb200_provider_* are the four trait methods of PressureProvider
 * (src/solver_provider.rs:67-76) over the C ABI. */
typedef struct rb200_provider rb200_provider;

typedef struct rb200_provider_config {
    rb200_grid grid;          /* the only grid this provider accepts        */
    double density;           /* sealed-box density                         */
    int method;               /* rb200_method                               */
    rb200_settings settings;  /* stopping rule used inside predict()        */
    int device;               /* CUDA ordinal                               */
} rb200_provider_config;

/* PressureRequest (src/solver_provider.rs:47-52): RHS of the full, ungauged
 * integrated operator, x-fastest, m^3/s^2. */
typedef struct rb200_request {
    rb200_grid grid;
    double density;
    double dt;
    const double* rhs;
    size_t len;
} rb200_request;

/* SolverMetadata (src/solver_provider.rs:18-33), as static strings. */
typedef struct rb200_metadata {
    const char* id;
    const char* version;
    const char* stage;
    const char* input_layout;
    const char* input_scalar;
    const char* input_units;
    const char* output_layout;
    const char* output_scalar;
    const char* output_units;
    const char* domain;
    uint64_t shape_xyz[3];
} rb200_metadata;

/* Allocates every device buffer for the grid; predict() allocates nothing. */
RB200_API int rb200_provider_create(const rb200_provider_config* config, rb200_provider** out);
RB200_API void rb200_provider_destroy(rb200_provider* provider);
/* PressureProvider::metadata */
RB200_API int rb200_provider_metadata(const rb200_provider* provider, rb200_metadata* out);
/* PressureProvider::supports: RB200_OK or RB200_UNSUPPORTED. */
RB200_API int rb200_provider_supports(const rb200_provider* provider, const rb200_request* request);
/* PressureProvider::predict: writes all len cells of pressure (p[0] == 0).
 * Returns RB200_OK, RB200_UNSUPPORTED, RB200_EXECUTION, RB200_CANCELLED or
 * RB200_NONFINITE_OUTPUT; an unconverged solve (iteration limit, breakdown,
 * incompatible RHS) is RB200_EXECUTION with the detail in last_error and
 * last_report. The caller re-qualifies the output, as Rheon does. */
RB200_API int rb200_provider_predict(rb200_provider* provider, const rb200_request* request, double* pressure,
                           size_t len, rb200_cancel_fn cancelled, void* ctx);
RB200_API const char* rb200_provider_last_error(const rb200_provider* provider);
RB200_API int rb200_provider_last_report(const rb200_provider* provider, rb200_report* out, int* solve_status);

/* -------------------------------------------------- PressureWorkspace mirror */
typedef struct rb200_workspace rb200_workspace;

/* PressureWorkspace::with_implementation(grid, limit, implementation)
 * (src/pressure.rs:265-314). memory_limit bounds the device bytes. */
RB200_API int rb200_workspace_create(const rb200_grid* grid, double density, int method,
                           uint64_t memory_limit, int device, rb200_workspace** out);
RB200_API void rb200_workspace_destroy(rb200_workspace* ws);
RB200_API uint64_t rb200_workspace_allocated_bytes(const rb200_workspace* ws);
/* Opaque cudaStream_t of the workspace. */
RB200_API void* rb200_workspace_stream(rb200_workspace* ws);
/* PressureWorkspace::solve_rhs on host buffers. On RB200_ITERATION_LIMIT the
 * iterate stays readable through rb200_workspace_pressure, as in Rheon. */
RB200_API int rb200_workspace_solve_rhs(rb200_workspace* ws, const double* rhs, size_t len, double dt,
                              const rb200_settings* settings, rb200_report* report,
                              rb200_cancel_fn cancelled, void* ctx);
/* PressureWorkspace::solve_rhs_with_initial_pressure (src/pressure.rs:415-430,
 * feature "accepted-pressure-warm-start"): PCG seeded by `initial` (len
 * values, finite, initial[0] == 0, else RB200_NONFINITE_INPUT or
 * RB200_INVALID_INITIAL_PRESSURE). rhs and initial may be host or device
 * memory (the copy direction is inferred). */
RB200_API int rb200_workspace_solve_rhs_initial(rb200_workspace* ws, const double* rhs, const double* initial,
                                                size_t len, double dt, const rb200_settings* settings,
                                                rb200_report* report, rb200_cancel_fn cancelled, void* ctx);
/* Same on a device-resident RHS (len doubles on the workspace's device). The
 * workspace works on its own stream: the RHS must be complete when called. */
RB200_API int rb200_workspace_solve_rhs_device(rb200_workspace* ws, const double* rhs_device, size_t len,
                                     double dt, const rb200_settings* settings,
                                     rb200_report* report, rb200_cancel_fn cancelled, void* ctx);
/* Last pressure to host / device memory. */
RB200_API int rb200_workspace_pressure(rb200_workspace* ws, double* out, size_t len);
RB200_API const double* rb200_workspace_pressure_device(rb200_workspace* ws);
/* Per-iteration scalars of the next solves (NULL disables). trace points to
 * capacity rb200_trace records in host memory, filled at the end of a solve. */
RB200_API int rb200_workspace_set_trace(rb200_workspace* ws, rb200_trace* trace, size_t capacity);
/* Diagnostics: average device milliseconds of one PCG pass (which = 0: the
 * fused direction update + operator + curvature pass, 1: the fused update +
 * preconditioner + dots pass), over `launches` back-to-back launches timed with
 * CUDA events on the handle's stream, on the current vectors; or (which = 2)
 * of one iteration of the persistent Jacobi-PCG kernel, run for `launches`
 * iterations in one launch (RB200_UNSUPPORTED when the handle does not use
 * it). Leaves the solver's scalars in a timing state; the next solve resets
 * them. */
RB200_API int rb200_workspace_profile(rb200_workspace* ws, int which, int launches, double* avg_ms);

/* Allocation-free Jacobi-PCG solve. No counterpart in the reference.
 *
 * For callers that must not allocate device memory: a host application whose
 * device memory is owned by its own allocator under a fixed budget, so that a
 * plug-in may not grow the process's device footprint while it runs. It solves like rb200_workspace_solve_rhs_device with
 * RB200_JACOBI_PCG_V1 (same kernels, same results) on caller-owned device
 * buffers: rhs_device (read) and pressure_device (written, len doubles).
 * It calls no cudaMalloc/cudaFree or allocating routine. Its scratch is one
 * fixed device array of about 1.2 MB inside the library, which every GPU that
 * loads the library holds until the process exits; grids of more than 32768
 * cells (32^3) are rejected with RB200_UNSUPPORTED.
 *   - The first call on a device looks up that array's device address (once
 *     per device, with the device current); make that first call before any
 *     stream capture begins. The address is kept for the process: do not call
 *     this entry point on a device after cudaDeviceReset on it.
 *   - Every call shares the one array and leaves its contents behind; calls
 *     whose work overlaps on the GPU (other threads, other streams) race and
 *     corrupt each other. Serialize them.
 *   - The call is synchronous: it polls the solver state from the host.
 * `stream` is a cudaStream_t (NULL = legacy default stream). */
RB200_API int rb200_pressure_solve_static(const rb200_grid* grid, double density, const double* rhs_device,
                                          double* pressure_device, size_t len, double dt,
                                          const rb200_settings* settings, rb200_report* report, void* stream);

/* ----------------------------------------- PressureOperator device primitives
 * All pointers are device pointers; `stream` is a cudaStream_t (NULL = legacy).
 * These validate like the reference (walls, finiteness) and return its errors. */
RB200_API int rb200_apply_full_device(const rb200_grid* grid, double density, const double* pressure,
                            double* out, void* stream);
/* precondition_jacobi (src/pressure.rs:534-575): z = r/D on every row but the
 * eliminated gauge row (z[0] = 0); *rz receives r.z over rows >= 1
 * (compensated). Returns RB200_NONFINITE_INPUT for a non-finite r. */
RB200_API int rb200_precondition_jacobi_device(const rb200_grid* grid, double density, const double* r, double* z,
                                               size_t len, double* rz, void* stream);
/* ProviderWorkspace's qualification of a candidate pressure on the device
 * (src/solver_provider.rs:239-270): RB200_NONFINITE_OUTPUT for a non-finite
 * pressure or product K p, RB200_NONZERO_GAUGE for pressure[0] != 0,
 * RB200_QUALITY_GATE when |b - K p|_2 exceeds max(absolute, relative |b|_2)
 * or max|b - K p| dt / V exceeds settings.divergence_limit, else RB200_OK.
 * report (may be NULL) receives the candidate's residual l2, max and
 * predicted divergence (iterations 0). Synchronous on `stream`. */
RB200_API int rb200_qualify_pressure_device(const rb200_grid* grid, double density, const double* rhs,
                                            const double* pressure, size_t len, double dt,
                                            const rb200_settings* settings, rb200_report* report, void* stream);
/* The momentum witness of a supplied projection
 * (solver_provider/composition/projection.rs:515-542): the supplied velocity
 * (su, sv, sw) must equal, bit for bit, the input velocity (u, v, w)
 * corrected with the supplied pressure. RB200_OK, or RB200_QUALITY_GATE with
 * *axis (0, 1, 2) and *index the first mismatching face (MomentumWitness);
 * field validation errors as the primitives above. Synchronous on `stream`. */
RB200_API int rb200_projection_witness_f32_device(const rb200_grid* grid, double density, const double* pressure,
                                                  double dt, const float* u, const float* v, const float* w,
                                                  const float* su, const float* sv, const float* sw, int* axis,
                                                  uint64_t* index, void* stream);
RB200_API int rb200_projection_witness_f64_device(const rb200_grid* grid, double density, const double* pressure,
                                                  double dt, const double* u, const double* v, const double* w,
                                                  const double* su, const double* sv, const double* sw, int* axis,
                                                  uint64_t* index, void* stream);
RB200_API int rb200_build_rhs_f32_device(const rb200_grid* grid, double density, const float* u,
                               const float* v, const float* w, double dt, double* rhs,
                               void* stream);
RB200_API int rb200_build_rhs_f64_device(const rb200_grid* grid, double density, const double* u,
                               const double* v, const double* w, double dt, double* rhs,
                               void* stream);
RB200_API int rb200_divergence_f32_device(const rb200_grid* grid, const float* u, const float* v,
                                const float* w, double* out, void* stream);
RB200_API int rb200_divergence_f64_device(const rb200_grid* grid, const double* u, const double* v,
                                const double* w, double* out, void* stream);
RB200_API int rb200_correct_f32_device(const rb200_grid* grid, double density, const double* pressure,
                             double dt, float* u, float* v, float* w, void* stream);
RB200_API int rb200_correct_f64_device(const rb200_grid* grid, double density, const double* pressure,
                             double dt, double* u, double* v, double* w, void* stream);
RB200_API int rb200_advect_velocity_f32_device(const rb200_grid* grid, const float* u, const float* v,
                                     const float* w, double dt, float* out_u, float* out_v,
                                     float* out_w, void* stream);
RB200_API int rb200_advect_velocity_f64_device(const rb200_grid* grid, const double* u, const double* v,
                                     const double* w, double dt, double* out_u, double* out_v,
                                     double* out_w, void* stream);
RB200_API int rb200_advect_tracer_f32_device(const rb200_grid* grid, const float* old, const float* u,
                                   const float* v, const float* w, double dt, float* out,
                                   void* stream);

/* ---------------------------------------------- resident carrier step owner
 * Device-resident accepted state, composed as Rheon's step owner orders it
 * (src/simulation.rs:812-1403): dt policy -> advect_velocity -> optional
 * buoyancy -> build_rhs -> PCG -> correct_candidate -> actual divergence gate
 * -> Courant gate -> advect_tracer -> commit. A failed step leaves the
 * accepted state untouched (transactional, src/simulation.rs:805-811). */
typedef struct rb200_carrier rb200_carrier;

typedef struct rb200_carrier_config {
    rb200_grid grid;
    double density;
    int storage;                   /* rb200_storage                        */
    int method;                    /* rb200_method                         */
    rb200_settings settings;
    double actual_divergence_limit;/* SimulationConfig (simulation.rs:11)  */
    double max_courant;
    int with_tracer;               /* allocate a cell tracer (f32)         */
    int device;
    int fp32_advection;            /* sample/backtrace in FP32 arithmetic  */
    int warm_start;                /* PressureInitializationPolicy: 0 Cold, 1 AcceptedPreviousV1
                                      (src/pressure_initialization.rs:7-12): seed each
                                      solve with the last accepted step's pressure */
} rb200_carrier_config;

typedef struct rb200_step_params {
    double requested_dt;   /* upper bound on dt                              */
    double cfl;            /* dt <= cfl / velocity_rate when > 0 (0 = off)   */
    double buoyancy;       /* g_b on Y faces from the tracer (0 = off)       */
    int iteration_limit_ok;/* accept an exact-iteration-count solve          */
    int skip_gates;        /* do not reject on divergence/Courant gates      */
} rb200_step_params;

/* StepReport (src/simulation.rs:44-53) subset plus solver diagnostics. */
typedef struct rb200_step_report {
    double dt;
    double time;
    uint64_t generation;
    rb200_report pressure;
    int pressure_status;
    double actual_divergence_max;
    double courant;
    double velocity_rate;
    double pressure_ms;    /* device time of the pressure solve (CUDA events) */
    uint64_t kernel_launches; /* kernels this step launched (graph nodes included) */
    int pressure_initialization; /* the policy this step's solve actually used: 0 cold,
                                    1 seeded by the accepted previous pressure */
} rb200_step_report;

RB200_API int rb200_carrier_create(const rb200_carrier_config* config, rb200_carrier** out);
RB200_API void rb200_carrier_destroy(rb200_carrier* carrier);
RB200_API uint64_t rb200_carrier_allocated_bytes(const rb200_carrier* carrier);
RB200_API void* rb200_carrier_stream(rb200_carrier* carrier);
/* Faces in the configured storage type (float* or double*), in host memory or
 * in this device's memory (the copy direction is inferred); tracer may be
 * NULL. Validates the fixed-box wall contract. rb200_carrier_download copies
 * the accepted state out the same way. */
RB200_API int rb200_carrier_upload(rb200_carrier* carrier, const void* u, const void* v, const void* w,
                         const float* tracer);
RB200_API int rb200_carrier_download(rb200_carrier* carrier, void* u, void* v, void* w, float* tracer);
/* Random-Fourier accepted state generated on the device: u_d(x) = amplitude *
 * sum_m amp[m][d] sin(2 pi k_m.x/L + phase[m]) + noise * U(-1,1) at the face
 * centres (x in cell units, L the cell counts), wall-normal faces 0; k and amp
 * are modes x 3 row-major, modes <= 8. U is SplitMix64 stream 16+d of `seed`,
 * as the host generator. The tracer, if any, is cleared. */
RB200_API int rb200_carrier_init_fourier(rb200_carrier* carrier, uint64_t seed, int modes, const double* k,
                                         const double* phase, const double* amp, double amplitude, double noise);
/* Device pointers of the accepted state (valid until the next step). */
RB200_API int rb200_carrier_state_device(rb200_carrier* carrier, void** u, void** v, void** w,
                               float** tracer);
/* One step as one CUDA graph (dt policy, advection, RHS, the pressure solve
 * as a device-controlled WHILE loop, correction, gates, tracer, commit), then
 * a wait for its report. Cancellation is polled before the step. Returns the
 * step status (RB200_OK when the step was accepted and published). */
RB200_API int rb200_carrier_step(rb200_carrier* carrier, const rb200_step_params* params,
                                 rb200_step_report* report, rb200_cancel_fn cancelled, void* ctx);
/* Launch a step without waiting (one per carrier in flight); carriers on
 * different streams overlap on the device. rb200_carrier_step_wait blocks for
 * the report and returns the step status. */
RB200_API int rb200_carrier_step_async(rb200_carrier* carrier, const rb200_step_params* params);
/* A projection of the accepted state (ProjectionStepWorkspace::project,
 * src/projection_step.rs:863-1033): the accepted faces (as uploaded) are the
 * provisional velocity; build_rhs with dt = params->requested_dt, the pressure
 * solve, correction, the actual divergence gate and the commit run as in a
 * step, without advection and without the Courant gate. cfl and buoyancy must
 * be 0, and the carrier must carry no tracer or liquid state. The async form
 * pairs with rb200_carrier_step_wait / rb200_carrier_step_poll. */
RB200_API int rb200_carrier_project(rb200_carrier* carrier, const rb200_step_params* params,
                                    rb200_step_report* report);
RB200_API int rb200_carrier_project_async(rb200_carrier* carrier, const rb200_step_params* params);
RB200_API int rb200_carrier_step_wait(rb200_carrier* carrier, rb200_step_report* report);
/* Nonblocking: 1 when the launched step has finished on the device (its
 * report is ready for rb200_carrier_step_wait), 0 while it runs or when no
 * step is in flight. */
RB200_API int rb200_carrier_step_poll(const rb200_carrier* carrier);
/* Batched instances: launch one step of every carrier, then wait for all.
 * statuses[i] receives each step's status; returns the first launch error. */
RB200_API int rb200_carriers_step(rb200_carrier* const* carriers, size_t count, const rb200_step_params* params,
                                  rb200_step_report* reports, int* statuses);
/* ------------------------------------------------- packed batch of carriers
 * Many independent fixed boxes of uneven sizes stepped together with the
 * mixed-precision pressure method (f32 faces, FP32 multigrid V(2,2) inside
 * FP64 flexible CG). No counterpart in the reference, which steps one box at a
 * time (src/simulation.rs:812-1403); every instance follows that step owner's
 * order, gates and transactional commit. All instances live in one device
 * arena, every stage of the step is one launch over all of them, and a step of
 * the whole batch is one CUDA graph (the solve a device-controlled WHILE node
 * that runs while any instance's solve runs). An instance's results do not
 * depend on the other instances: a batch of one gives the same bits. Each
 * instance needs a hierarchy of at least two levels whose non-coarsest levels
 * have an x extent that is a multiple of 4 (RB200_UNSUPPORTED otherwise), and
 * carries no tracer. */
typedef struct rb200_batch rb200_batch;

typedef struct rb200_batch_config {
    double density;
    rb200_settings settings;
    double actual_divergence_limit;/* SimulationConfig (simulation.rs:11)  */
    double max_courant;
    int device;
    int fp32_advection;            /* sample/backtrace in FP32 arithmetic  */
} rb200_batch_config;

/* At most 128 instances. */
RB200_API int rb200_batch_create(const rb200_grid* grids, size_t count, const rb200_batch_config* config,
                                 rb200_batch** out);
RB200_API void rb200_batch_destroy(rb200_batch* batch);
RB200_API uint64_t rb200_batch_allocated_bytes(const rb200_batch* batch);
RB200_API void* rb200_batch_stream(rb200_batch* batch);
RB200_API const char* rb200_batch_last_error(const rb200_batch* batch);
/* f32 faces of instance `index` from host or device memory (validated like
 * rb200_carrier_upload); rb200_batch_download copies its accepted state out. */
RB200_API int rb200_batch_upload(rb200_batch* batch, size_t index, const float* u, const float* v, const float* w);
RB200_API int rb200_batch_download(rb200_batch* batch, size_t index, float* u, float* v, float* w);
/* The last pressure of instance `index` (host or device memory). */
RB200_API int rb200_batch_pressure(rb200_batch* batch, size_t index, double* out, size_t len);
/* One step of every instance: params, reports and statuses hold one entry per
 * instance (buoyancy must be 0). rb200_batch_step waits for the reports; the
 * async form launches the step graph, rb200_batch_step_poll tells whether it
 * has finished and rb200_batch_step_wait collects it. */
RB200_API int rb200_batch_step(rb200_batch* batch, const rb200_step_params* params, rb200_step_report* reports,
                               int* statuses);
RB200_API int rb200_batch_step_async(rb200_batch* batch, const rb200_step_params* params);
RB200_API int rb200_batch_step_poll(const rb200_batch* batch);
RB200_API int rb200_batch_step_wait(rb200_batch* batch, rb200_step_report* reports, int* statuses);
/* A profiling aid: one step of every instance like rb200_batch_step (the state
 * advances), issued eagerly with an event after every launch instead of as the
 * step graph, the solve loop decided on the host after each trip. Per kernel
 * kind (kinds >= rb200_batch_profile_kinds() entries): the summed device time
 * in ms, the launches and a static name. */
RB200_API int rb200_batch_profile_step(rb200_batch* batch, const rb200_step_params* params,
                                       rb200_step_report* reports, int* statuses, double* kernel_ms,
                                       int* kernel_launches, const char** kernel_names, int kinds);
RB200_API int rb200_batch_profile_kinds(void);

/* rb200_workspace_profile on the carrier's pressure solver. */
RB200_API int rb200_carrier_profile(rb200_carrier* carrier, int which, int launches, double* avg_ms);
/* Last pressure of the carrier (host copy). */
RB200_API int rb200_carrier_pressure(rb200_carrier* carrier, double* out, size_t len);
/* The carrier's accepted state as dense3D frame fields (device pointers,
 * valid until the next step or upload): faces, tracer (NULL without one),
 * the liquid fraction (NULL without a liquid state), and the pressure of the
 * last accepted step (NULL, i.e.
 * zeros, before the first accepted step after an upload). Without the
 * warm-start copy of the accepted pressure, a carrier whose last step was
 * rejected holds no accepted pressure: RB200_DENSE3D_INVALID_STATE. */
struct rb200_dense3d_fields;
RB200_API int rb200_carrier_dense3d_fields(rb200_carrier* carrier, struct rb200_dense3d_fields* fields);

/* ------------------------------------------------------------------------
 * dense3D accepted-state frames (src/dense3d_sequence.rs). A frame is one
 * JSON line, byte-identical to write_dense3d_frame (:412-564): header
 * (frame, time_s, dt_s, carrier/liquid stamps), the fields velocity_x/y/z and
 * tracer as Rust `{:.9e}` f32 text, fraction and pressure as `{:.17e}` f64
 * text, then the diagnostics object or null. The encoder formats a
 * device-resident state on the device; the writer streams frames to a file
 * descriptor with the limits and terminal errors of Dense3dSequence
 * (:42-120, :224-341).
 * ------------------------------------------------------------------------ */
typedef struct rb200_dense3d_encoder rb200_dense3d_encoder;
typedef struct rb200_dense3d_writer rb200_dense3d_writer;

/* The frame's scalars: LiquidTransportView clocks/stamps and, for accepted
 * steps, the LiquidStepReport diagnostics (src/dense3d_sequence.rs:494-556).
 * has_diagnostics = 0 is the constructor frame (frame 0, time 0, carrier
 * stamp version 0; "diagnostics":null, dt_s printed as 0). */
typedef struct rb200_dense3d_frame {
    uint64_t frame;
    double time_s;
    double dt_s;
    uint64_t carrier_stamp_id, carrier_stamp_version;
    uint64_t liquid_stamp_id, liquid_stamp_version;
    int has_diagnostics;
    uint64_t pressure_iterations;
    double pressure_residual_m3_s2, carrier_divergence_s_inv, liquid_divergence_s_inv;
    double volume_before_m3, volume_after_m3, mass_after_kg;
    double inward_m3, outward_m3, source_m3, balance_m3, rounding_budget_m3;
} rb200_dense3d_frame;

/* Device pointers of one state. u, v, w: face velocities in
 * velocity_storage (RB200_FACES_F32, or RB200_FACES_F64 printed as the f32
 * each value rounds to). tracer (f32), fraction (f64) and pressure (f64) may
 * be NULL (zeros: the constructor pressure is zero). */
typedef struct rb200_dense3d_fields {
    int velocity_storage;
    const void* u;
    const void* v;
    const void* w;
    const float* tracer;
    const double* fraction;
    const double* pressure;
} rb200_dense3d_fields;

/* Dense3dLimits (src/dense3d_sequence.rs:13-19). */
typedef struct rb200_dense3d_limits {
    uint64_t max_cells;
    uint64_t max_frames;  /* includes the constructor frame */
    uint64_t max_bytes;   /* total bytes of all lines     */
} rb200_dense3d_limits;

RB200_API int rb200_dense3d_encoder_create(const rb200_grid* grid, int device, rb200_dense3d_encoder** out);
RB200_API void rb200_dense3d_encoder_destroy(rb200_dense3d_encoder* encoder);
/* Upper bound on the bytes of one frame line of this grid. */
RB200_API uint64_t rb200_dense3d_frame_bound(const rb200_dense3d_encoder* encoder);
RB200_API const char* rb200_dense3d_encoder_error(const rb200_dense3d_encoder* encoder);
/* Encode one frame into device memory `out` (capacity bytes) on `stream`,
 * then wait; *length receives the line's bytes. The preflight of
 * src/dense3d_sequence.rs:419-494 (finite fields, fraction in [0, 1], clocks,
 * report) fails with RB200_DENSE3D_INVALID_STATE before any byte is written;
 * a too small buffer gives RB200_DENSE3D_LIMIT. */
RB200_API int rb200_dense3d_encode(rb200_dense3d_encoder* encoder, const rb200_dense3d_frame* frame,
                                   const rb200_dense3d_fields* fields, void* out, uint64_t capacity,
                                   uint64_t* length, void* stream);
/* The text of one number as Rust's `{:.17e}` (f64) / `{:.9e}` (f32) prints
 * it, computed on the host by the encoder's own routine; returns the length
 * (a NUL follows) or RB200_INVALID_ARGUMENT (capacity < 26 / 17). */
RB200_API int rb200_dense3d_text_f64(double value, char* out, size_t capacity);
RB200_API int rb200_dense3d_text_f32(float value, char* out, size_t capacity);

/* Frame stream on an open file descriptor. Creation fails with
 * RB200_DENSE3D_LIMIT like Dense3dSequence::new (zero frames or bytes, too
 * many cells). Frames must come in order 0, 1, 2, ... (frame 0: the
 * constructor frame). rb200_dense3d_writer_frame encodes the frame on
 * `stream` and waits for the encode; the device-to-host copy and the write(2)
 * then run on the writer's own stream and thread, overlapping the caller's
 * next step (two frames in flight at most). Any failure is terminal (later
 * calls give RB200_DENSE3D_ABORTED): the frame limit (RB200_DENSE3D_LIMIT), a
 * frame longer than the byte budget left (RB200_DENSE3D_IO, nothing of that
 * frame is written), the preflight, and a failed copy or write
 * (RB200_DENSE3D_IO, reported by the next frame, flush or sync call). */
RB200_API int rb200_dense3d_writer_create(const rb200_grid* grid, const rb200_dense3d_limits* limits, int fd,
                                          int device, rb200_dense3d_writer** out);
RB200_API void rb200_dense3d_writer_destroy(rb200_dense3d_writer* writer);
RB200_API int rb200_dense3d_writer_frame(rb200_dense3d_writer* writer, const rb200_dense3d_frame* frame,
                                         const rb200_dense3d_fields* fields, void* stream);
/* Dense3dSequence::flush (src/dense3d_sequence.rs:332-341): returns once
 * every accepted frame is written; terminal on failure. */
RB200_API int rb200_dense3d_writer_flush(rb200_dense3d_writer* writer);
/* flush, then fsync of the descriptor (a failure aborts the stream). */
RB200_API int rb200_dense3d_writer_sync(rb200_dense3d_writer* writer);
/* Frames accepted (encoded and queued), and bytes written so far. */
RB200_API uint64_t rb200_dense3d_writer_frames(const rb200_dense3d_writer* writer);
RB200_API uint64_t rb200_dense3d_writer_bytes(const rb200_dense3d_writer* writer);
RB200_API int rb200_dense3d_writer_aborted(const rb200_dense3d_writer* writer);
RB200_API const char* rb200_dense3d_writer_error(const rb200_dense3d_writer* writer);

/* ------------------------------------------------------------------------
 * Liquid-volume transport (src/liquid_volume.rs): the represented liquid
 * fraction moved through the carrier's face velocities by first-order
 * shared-face donor transfer, on the device. LiquidVolumeState with an inlet
 * boundary and the all-cells divergence domain.
 * ------------------------------------------------------------------------ */
typedef struct rb200_liquid_volume rb200_liquid_volume;

/* LiquidVolumeError (src/liquid_volume.rs:27-72), the payload in the report. */
typedef enum rb200_liquid_error {
    RB200_LIQUID_OK = 0,
    RB200_LIQUID_INVALID_DENSITY = 1,
    RB200_LIQUID_INVALID_FRACTION = 2,    /* error_cell */
    RB200_LIQUID_INVALID_INLET = 3,
    RB200_LIQUID_INVALID_SOURCE = 4,
    RB200_LIQUID_INVALID_SETTINGS = 5,
    RB200_LIQUID_INVALID_TIME_STEP = 6,
    RB200_LIQUID_TIME_RESOLUTION = 7,
    RB200_LIQUID_TIME_MISMATCH = 8,
    RB200_LIQUID_LENGTH_MISMATCH = 9,
    RB200_LIQUID_NONFINITE_VELOCITY = 10,
    RB200_LIQUID_VERSION_OVERFLOW = 11,
    RB200_LIQUID_BUFFER_LIMIT = 12,       /* error_actual = required, error_limit = limit */
    RB200_LIQUID_COURANT_LIMIT = 13,      /* error_cell, error_actual, error_limit */
    RB200_LIQUID_DIVERGENCE_LIMIT = 14,   /* error_actual, error_limit */
    RB200_LIQUID_FRACTION_BOUNDS = 15,    /* error_cell, error_actual = fraction */
    RB200_LIQUID_BALANCE_LIMIT = 16,      /* error_actual = error, error_limit = rounding budget */
    RB200_LIQUID_ARITHMETIC_FAILURE = 17,
    RB200_LIQUID_CANCELLED = 18,
    RB200_LIQUID_GEOMETRY_MISMATCH = 19,
    RB200_LIQUID_PERIODIC_VELOCITY_MISMATCH = 20  /* error_cell = the seam's lower face, error_actual = the axis */
} rb200_liquid_error;

/* VolumeStamp (src/liquid_volume.rs:6-10). */
typedef struct rb200_liquid_stamp {
    uint64_t id;
    uint64_t version;
} rb200_liquid_stamp;

/* LiquidFlowInterval (src/liquid_volume.rs:111-150): f32 face velocities
 * (device pointers, x-fastest) held over [start, start + dt]. */
typedef struct rb200_liquid_flow {
    rb200_liquid_stamp stamp;
    const float* u;
    const float* v;
    const float* w;
    double start;
    double dt;
} rb200_liquid_flow;

/* LiquidInlet (src/liquid_volume.rs:76-96): fraction[2 d + s] is the outside
 * fraction of axis d, side s (0 lower, 1 upper), used on inflow only. */
typedef struct rb200_liquid_inlet {
    rb200_liquid_stamp stamp;
    double fraction[6];
} rb200_liquid_inlet;

/* LiquidVolumeSource (src/liquid_volume.rs:174-190): m^3/s per cell (device). */
typedef struct rb200_liquid_source {
    rb200_liquid_stamp stamp;
    const double* rate;
} rb200_liquid_source;

/* LiquidVolumeSettings (src/liquid_volume.rs:192-199). */
typedef struct rb200_liquid_settings {
    double max_outward_courant;
    double actual_divergence_limit;
} rb200_liquid_settings;

/* LiquidVolumeReport (src/liquid_volume.rs:200-229) plus the error. */
typedef struct rb200_liquid_report {
    rb200_liquid_stamp stamp, flow, inlet, source;  /* inlet: the boundary's stamp */
    int has_source;
    int periodic;         /* advance_periodic */
    double dt, time;
    double liquid_volume_before, liquid_volume_after;
    double inward_boundary_volume, outward_boundary_volume, source_volume;
    double volume_balance_error, volume_rounding_budget;
    double liquid_mass_before, liquid_mass_after;
    double max_outward_courant, actual_divergence_max;
    double fraction_min, fraction_max;
    uint64_t dry_cells, mixed_cells, full_cells;
    int error;            /* rb200_liquid_error */
    uint64_t error_cell;
    double error_actual, error_limit;
} rb200_liquid_report;

/* LiquidVolumeState::new (src/liquid_volume.rs:276-351): fraction is host or
 * device memory of cell_len values; limit bounds the device bytes (two
 * fraction arrays). RB200_LIQUID_REJECTED with *error filled on a rejected
 * density, fraction, arithmetic or buffer limit. */
RB200_API int rb200_liquid_create(const rb200_grid* grid, double density, rb200_liquid_stamp stamp,
                                  const double* fraction, uint64_t limit, int device, rb200_liquid_volume** out,
                                  rb200_liquid_report* error);
RB200_API void rb200_liquid_destroy(rb200_liquid_volume* liquid);
RB200_API uint64_t rb200_liquid_allocated_bytes(const rb200_liquid_volume* liquid);
/* The accepted state: fraction (device pointer, valid until the next
 * advance), stamp and time. */
RB200_API int rb200_liquid_state(const rb200_liquid_volume* liquid, const double** fraction,
                                 rb200_liquid_stamp* stamp, double* time);
RB200_API int rb200_liquid_download(rb200_liquid_volume* liquid, double* out, size_t len);
/* LiquidVolumeState::advance (src/liquid_volume.rs:376-387, 520-776): one
 * explicit interval on `stream` (NULL: the state's own), waited for. On
 * success the candidate becomes the accepted state (time = start + dt,
 * version + 1); on RB200_LIQUID_REJECTED the accepted state is unchanged and
 * report->error names the failure. source may be NULL. */
RB200_API int rb200_liquid_advance(rb200_liquid_volume* liquid, const rb200_liquid_flow* flow,
                                   const rb200_liquid_inlet* inlet, const rb200_liquid_source* source,
                                   const rb200_liquid_settings* settings, rb200_liquid_report* report,
                                   void* stream);
/* VolumeStage (src/liquid_volume.rs:18-23): the cancellation points of an
 * interval, asked in the reference's order (prepare_with_boundary,
 * src/liquid_volume.rs:558-830): BeforeFlux once; FaceFluxSlice once per z
 * plane of each axis's faces (for the periodic seam check, then for the face
 * transfers); CellUpdateSlice once per z plane of cells; BeforeCommit once,
 * after every check. A nonzero return cancels: RB200_LIQUID_REJECTED with
 * report->error = RB200_LIQUID_CANCELLED and report->error_cell = the stage,
 * the accepted state unchanged. The transport runs on the device before the
 * points are asked, so an error the reference meets before a point ends the
 * sequence there, as in the reference. */
typedef enum rb200_volume_stage {
    RB200_VOLUME_BEFORE_FLUX = 0,
    RB200_VOLUME_FACE_FLUX_SLICE = 1,
    RB200_VOLUME_CELL_UPDATE_SLICE = 2,
    RB200_VOLUME_BEFORE_COMMIT = 3
} rb200_volume_stage;
typedef int (*rb200_liquid_cancel_fn)(void* ctx, int stage);
/* rb200_liquid_advance with the cancellation callback (NULL: never cancel). */
RB200_API int rb200_liquid_advance_cancellable(rb200_liquid_volume* liquid, const rb200_liquid_flow* flow,
                                               const rb200_liquid_inlet* inlet, const rb200_liquid_source* source,
                                               const rb200_liquid_settings* settings, rb200_liquid_cancel_fn cancel,
                                               void* ctx, rb200_liquid_report* report, void* stream);
/* LiquidVolumeState::advance_periodic (src/liquid_volume.rs:389-406): the box
 * wraps around on every axis. The two faces of each seam must carry the same
 * velocity (else RB200_LIQUID_PERIODIC_VELOCITY_MISMATCH), inflow through a
 * seam takes the fraction of the cell across it, and no boundary volume is
 * counted; `boundary` is reported as the report's inlet stamp. */
RB200_API int rb200_liquid_advance_periodic(rb200_liquid_volume* liquid, const rb200_liquid_flow* flow,
                                            rb200_liquid_stamp boundary, const rb200_liquid_source* source,
                                            const rb200_liquid_settings* settings, rb200_liquid_report* report,
                                            void* stream);
RB200_API int rb200_liquid_advance_periodic_cancellable(rb200_liquid_volume* liquid, const rb200_liquid_flow* flow,
                                                        rb200_liquid_stamp boundary,
                                                        const rb200_liquid_source* source,
                                                        const rb200_liquid_settings* settings,
                                                        rb200_liquid_cancel_fn cancel, void* ctx,
                                                        rb200_liquid_report* report, void* stream);

/* The liquid step on the resident carrier (LiquidTransportSimulation,
 * src/liquid_step.rs:828-900): the carrier owns a liquid-volume state, and
 * every step advances it through the step's corrected faces over
 * [time, time + dt] before the step commits; a rejected transport rejects the
 * step (status RB200_LIQUID_REJECTED, details in rb200_carrier_liquid_report)
 * and neither state changes. Needs f32 face storage. The flow intervals are
 * stamped {flow_id, candidate generation}. An upload or device
 * initialisation of the carrier restarts both clocks at zero. */
RB200_API int rb200_carrier_attach_liquid(rb200_carrier* carrier, double density, rb200_liquid_stamp stamp,
                                          uint64_t flow_id, const double* fraction, uint64_t limit,
                                          rb200_liquid_report* error);
/* The inlet, source (NULL: none; device memory kept valid while steps run)
 * and volume settings of the following steps (LiquidStepInputs). */
RB200_API int rb200_carrier_liquid_inputs(rb200_carrier* carrier, const rb200_liquid_inlet* inlet,
                                          const rb200_liquid_source* source, const rb200_liquid_settings* settings);
/* The liquid report of the last step (its error when the transport rejected it). */
RB200_API int rb200_carrier_liquid_report(const rb200_carrier* carrier, rb200_liquid_report* report);
/* The accepted liquid state: fraction (device), stamp, time. */
RB200_API int rb200_carrier_liquid_state(const rb200_carrier* carrier, const double** fraction,
                                         rb200_liquid_stamp* stamp, double* time);
/* Host (or device) copy of the accepted liquid fraction. */
RB200_API int rb200_carrier_liquid_download(rb200_carrier* carrier, double* out, size_t len);

/* ------------------------------------------------------------------ box flux
 * Prescribed outward speeds on the six sides of the fixed box
 * (src/box_flux.rs): BoxFluxWorkspace holds the pressure workspace of the
 * projection; project() imposes the sides' speeds on the provisional f32 faces,
 * rejects a net boundary flux above its rounding budget, solves the sealed
 * pressure system for the imposed field, corrects the interior faces into the
 * output, gates the stored field's divergence and reports the energy ledger.
 * Operator and pressure errors keep their own statuses (RB200_NONFINITE_INPUT,
 * RB200_LENGTH_MISMATCH, RB200_INVALID_ARGUMENT for InvalidTimeStep, the
 * PressureError statuses 6-11); BoxFluxError's own variants return
 * RB200_BOX_FLUX_REJECTED with rb200_box_flux_report.error set. */
typedef enum rb200_box_flux_error {
    RB200_BOX_FLUX_NONE = 0,
    RB200_BOX_FLUX_INVALID_BOUNDARY = 1,   /* a non-finite outward speed           */
    RB200_BOX_FLUX_INVALID_SETTINGS = 2,   /* actual_divergence_limit              */
    RB200_BOX_FLUX_INVALID_MASS = 3,       /* density * cell volume                */
    RB200_BOX_FLUX_BUFFER_LIMIT = 4,       /* {required, limit}                    */
    RB200_BOX_FLUX_INCOMPATIBLE_FLUX = 5,  /* {net, rounding_budget}: actual, limit */
    RB200_BOX_FLUX_CANCELLED = 6,          /* {stage}                              */
    RB200_BOX_FLUX_DIVERGENCE_LIMIT = 7,   /* {actual, limit}                      */
    RB200_BOX_FLUX_ARITHMETIC_FAILURE = 8
} rb200_box_flux_error;

/* BoxFluxStage (src/box_flux.rs:53-59): where the cancellation predicate is asked. */
typedef enum rb200_box_flux_stage {
    RB200_BOX_FLUX_BEFORE_SOLVE = 0,
    RB200_BOX_FLUX_PRESSURE_ITERATION = 1,
    RB200_BOX_FLUX_CORRECTION_SLICE = 2,
    RB200_BOX_FLUX_BEFORE_ACCEPTANCE = 3
} rb200_box_flux_stage;

/* PrescribedBoxFlux (src/box_flux.rs:15-46): outward[2*d] is the lower side of
 * axis d (outward normal -d), outward[2*d+1] the upper side, in m/s. */
typedef struct rb200_box_flux_boundary {
    uint64_t id, version;
    float outward[6];
} rb200_box_flux_boundary;

/* BoxFluxReport and BoxFluxWork (src/box_flux.rs:91-116) plus the error payloads. */
typedef struct rb200_box_flux_report {
    uint64_t boundary_id, boundary_version;
    rb200_report pressure;
    double actual_divergence_max;
    double net_outward_flux;
    double flux_rounding_budget;
    double kinetic_before;
    double kinetic_after;
    double correction_energy;
    double boundary_pressure_work;    /* -dt sum p Q                          */
    double divergence_residual_work;  /* dt sum p cell_volume div             */
    double correction_residual_work;  /* sum (m (v - u) + dt area dp) v       */
    double budget_error;
    int error;                        /* rb200_box_flux_error                 */
    int stage;                        /* rb200_box_flux_stage of a cancel     */
    double error_actual, error_limit; /* IncompatibleFlux / DivergenceLimit   */
    uint64_t required, limit;         /* BufferLimit                          */
} rb200_box_flux_report;

/* Cancellation predicate with the stage it is asked at (nonzero cancels). */
typedef int (*rb200_box_flux_cancel_fn)(void* ctx, int stage);

typedef struct rb200_box_flux rb200_box_flux;

/* BoxFluxWorkspace::new (src/box_flux.rs:132-186): limit covers 56 bytes per
 * cell, as the reference's (a pressure workspace and one f64 cell array);
 * `error` (optional) receives InvalidMass / BufferLimit. */
RB200_API int rb200_box_flux_create(const rb200_grid* grid, double density, uint64_t limit, int method, int device,
                                    rb200_box_flux** out, rb200_box_flux_report* error);
RB200_API void rb200_box_flux_destroy(rb200_box_flux* workspace);
RB200_API uint64_t rb200_box_flux_allocated_bytes(const rb200_box_flux* workspace);
RB200_API void* rb200_box_flux_stream(rb200_box_flux* workspace);
/* BoxFluxWorkspace::project (src/box_flux.rs:213-397) on device face arrays
 * (old and out, lengths in elements). Inputs are never written; the output is
 * written from the first correction slice on, so a failure after that leaves
 * it partial. The predicate is asked at BeforeSolve, between pressure
 * iterations, once per face slice of the correction (3 nz + 1 times: the
 * first before the device pass, the others once it is under way) and
 * BeforeAcceptance. Ordered on the workspace's stream; returns after it. */
RB200_API int rb200_box_flux_project_device(rb200_box_flux* workspace, const float* const old[3],
                                            const size_t old_len[3], double dt,
                                            const rb200_box_flux_boundary* boundary,
                                            const rb200_settings* pressure_settings,
                                            double actual_divergence_limit, float* const out[3],
                                            const size_t out_len[3], rb200_box_flux_report* report,
                                            rb200_box_flux_cancel_fn cancelled, void* ctx);
/* The same with host arrays: the old faces are copied in and the output out
 * (device staging allocated on the first call). */
RB200_API int rb200_box_flux_project(rb200_box_flux* workspace, const float* const old[3], const size_t old_len[3],
                                     double dt, const rb200_box_flux_boundary* boundary,
                                     const rb200_settings* pressure_settings, double actual_divergence_limit,
                                     float* const out[3], const size_t out_len[3], rb200_box_flux_report* report,
                                     rb200_box_flux_cancel_fn cancelled, void* ctx);
/* BoxFluxWorkspace::divergence (src/box_flux.rs:201-206, 405-434): the measured
 * divergence of a full f32 face field (device arrays), outer samples included. */
RB200_API int rb200_box_flux_divergence_device(rb200_box_flux* workspace, const float* const faces[3],
                                               const size_t len[3], double* out, size_t out_len);
/* BoxFluxWorkspace::pressure: the last pressure (host copy / device pointer). */
RB200_API int rb200_box_flux_pressure(rb200_box_flux* workspace, double* out, size_t len);
RB200_API const double* rb200_box_flux_pressure_device(rb200_box_flux* workspace);
/* Average device time (CUDA events on the workspace's stream) of `launches`
 * back-to-back repeats of the last projection's RHS pass (which = 0) or its
 * correction pass (which = 1). */
RB200_API int rb200_box_flux_profile(rb200_box_flux* workspace, int which, int launches, double* avg_ms);
/* Device times (CUDA events on the workspace's stream) of the RHS pass and the
 * correction pass inside the last projection that reached them (-1: not run). */
RB200_API int rb200_box_flux_last_pass_ms(rb200_box_flux* workspace, double* rhs_ms, double* correct_ms);

/* ------------------------------------------------------------------ forced step
 * The step owner with its forcing and boundary domains on the resident
 * carrier: Simulation::step / step_with_forces / step_with_box_flux
 * (src/simulation.rs:393-581, prepare_impl :812-1403). Host-driven: the
 * stages run as device passes on the carrier's stream in the reference's
 * order, with its cancellation points, and the accepted state is published
 * only by the final commit. Needs f32 face storage and a tracer. With a
 * liquid state attached (rb200_carrier_attach_liquid, inputs set) this is the
 * liquid step (LiquidTransportSimulation::step / step_with_box_flux,
 * src/liquid_step.rs:517-567): the transport runs through the candidate faces
 * and a rejected transport (RB200_LIQUID_REJECTED, rb200_carrier_liquid_report)
 * rejects the step. */
typedef struct rb200_smoke_source {      /* SmokeSource (src/simulation.rs:19-27) */
    double lower[3];
    double upper[3];
    double tracer_rate;                  /* concentration per second, saturated at one */
    double vertical_acceleration;        /* on the interior Y faces inside the box     */
} rb200_smoke_source;

typedef enum rb200_force_units { RB200_FORCE_ACCELERATION = 0, RB200_FORCE_DENSITY = 1 } rb200_force_units;

typedef struct rb200_body_force {        /* BodyForce (src/forces.rs:11-45) */
    double value[3];
    int units;                           /* rb200_force_units                         */
    int has_region;                      /* 0: the whole box                          */
    double lower[3];                     /* half-open support lower <= x < upper      */
    double upper[3];
} rb200_body_force;

/* StepStage (src/simulation.rs:28-42), the stage a cancellation is asked at. */
typedef enum rb200_step_stage {
    RB200_STAGE_BEFORE_ADVECTION = 0,
    RB200_STAGE_VELOCITY_SLICE = 1,
    RB200_STAGE_BEFORE_FORCES = 2,
    RB200_STAGE_FORCE_SLICE = 3,
    RB200_STAGE_VISCOSITY = 4,
    RB200_STAGE_BEFORE_PRESSURE = 5,
    RB200_STAGE_PRESSURE_ITERATION = 6,
    RB200_STAGE_PROJECTION_SLICE = 7,
    RB200_STAGE_BEFORE_PROJECTION_ACCEPTANCE = 8,
    RB200_STAGE_BEFORE_TRACER = 9,
    RB200_STAGE_TRACER_SLICE = 10,
    RB200_STAGE_BEFORE_COMMIT = 11,
    RB200_STAGE_LIQUID_BEFORE_COMMIT = 12   /* LiquidStepStage::BeforeCommit (src/liquid_step.rs:918) */
} rb200_step_stage;

typedef int (*rb200_step_cancel_fn)(void* ctx, int stage);

/* SimulationError's own variants (src/simulation.rs:55-83) under RB200_SIMULATION_REJECTED. */
typedef enum rb200_simulation_error {
    RB200_SIMULATION_NONE = 0,
    RB200_SIMULATION_INVALID_SOURCE = 1,
    RB200_SIMULATION_INVALID_FORCE = 2,
    RB200_SIMULATION_TIME_RESOLUTION = 3,
    RB200_SIMULATION_BOUNDARY_WORKSPACE_MISMATCH = 4,
    RB200_SIMULATION_CANCELLED = 5        /* report.stage */
} rb200_simulation_error;

typedef struct rb200_forced_step_params {
    double requested_dt;
    const rb200_smoke_source* source;    /* NULL: none                                */
    const rb200_body_force* forces;      /* force_count entries                       */
    size_t force_count;
    rb200_box_flux* box_flux;            /* NULL: the sealed box; else the boundary's
                                            projection workspace (same grid, density,
                                            method as the carrier)                    */
    const rb200_box_flux_boundary* boundary;
    int tracer_policy;                   /* BoxFluxTracerPolicy: 0 ClampedAppearance  */
} rb200_forced_step_params;

/* ForcedStepReport / BoxFluxStepReport (src/forces.rs:51-61,
 * src/box_flux_step.rs:26-57) plus the error payloads. */
typedef struct rb200_forced_step_report {
    double dt, time;
    uint64_t generation;
    rb200_report pressure;
    double actual_divergence_max, courant, tracer_integral, kinetic_energy;
    int has_forces;                      /* ForceReport present                       */
    int has_boundary;                    /* box-flux step: projection and work below  */
    double force_kinetic_before, force_kinetic_after, force_applied_work;
    rb200_box_flux_report projection;
    double kinetic_old, kinetic_after_advection, kinetic_after_smoke_force, kinetic_before_projection,
        kinetic_accepted, advection_change, smoke_force_work, external_force_work, budget_error,
        boundary_volume_imbalance, tracer_old_integral, tracer_transport_change, tracer_source_change;
    int tracer_policy;
    int error;                           /* rb200_simulation_error                    */
    int stage;                           /* rb200_step_stage of a cancellation        */
    int pad;
    double error_actual, error_limit;    /* DivergenceLimit / CourantLimit            */
    uint64_t simulation_array_bytes, boundary_workspace_array_bytes;
} rb200_forced_step_report;

RB200_API int rb200_carrier_step_forced(rb200_carrier* carrier, const rb200_forced_step_params* params,
                                        rb200_forced_step_report* report, rb200_step_cancel_fn cancelled,
                                        void* ctx);

#ifdef __cplusplus
}
#endif
#endif
