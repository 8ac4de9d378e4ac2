/*
 * Oracle for the fixed-box carrier step: a CPU restatement of Rheon's Rust
 * arithmetic for this path. TEST INFRASTRUCTURE ONLY. It is the checker that
 * the CUDA library is compared against, and the CPU baseline that bench.py
 * times. Nothing in the product (rheon_b200/, include/) links or calls it.
 *
 * Every routine keeps the reference's operation order and its serial
 * Neumaier-compensated reductions, and is compiled with -ffp-contract=off
 * (Rust never fuses a multiply and an add). The reference itself is Rust and
 * cannot be compiled in this image (no cargo/rustc), so parity is pinned by
 * porting the reference's own known-answer tests onto this restatement.
 *
 * Reference files (paths within the Rheon project):
 *   src/geometry.rs    GridGeometry::new :114-191, cell/face indexing :250-258
 *   src/sampling.rs    ScalarSampler::sample :74-122, backtrace :151-175
 *   src/advection.rs   advect_velocity :28-68, advect_tracer :72-102
 *   src/operator.rs    new :58-97, apply_full :378-456, build_rhs :460-509,
 *                      divergence :513-568, correct_candidate_in_place :627-668,
 *                      build_rhs_f64 :672-708, divergence_f64 :711-742,
 *                      correct_candidate_f64 :746-781, diagonal :813-838
 *   src/pressure.rs    compensated_sum :135-148, true_report :432-456,
 *                      precondition_sgs :467-532, precondition_jacobi :534-575,
 *                      solve_loaded :577-740
 *   src/solver_provider.rs  ProviderWorkspace::solve_observed :160-327
 *   src/simulation.rs  velocity_rate :1415-1429, apply_force :1449-1472
 */
#ifndef RHEON_B200_ORACLE_H
#define RHEON_B200_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes share their numeric values with include/rheon_b200.h. */
enum {
    ORC_OK = 0,
    ORC_UNSUPPORTED = 1,
    ORC_EXECUTION = 2,
    ORC_NONFINITE_OUTPUT = 3,
    ORC_NONZERO_GAUGE = 4,
    ORC_QUALITY_GATE = 5,
    ORC_CANCELLED = 6,
    ORC_ITERATION_LIMIT = 7,
    ORC_BREAKDOWN = 8,
    ORC_OUT_OF_MEMORY = 9,
    ORC_INVALID_ARGUMENT = 10,
    ORC_INCOMPATIBLE_RHS = 11,
    ORC_NONFINITE_INPUT = 12,
    ORC_NONZERO_WALL_VELOCITY = 13,
    ORC_ARITHMETIC_FAILURE = 14,
    ORC_DIVERGENCE_LIMIT = 15,
    ORC_COURANT_LIMIT = 16,
    ORC_LENGTH_MISMATCH = 18,
    ORC_INVALID_GEOMETRY = 19,
    ORC_INVALID_TIME_STEP = 20,
    ORC_NONFINITE_POSITION = 21,
    ORC_INVALID_INITIAL_PRESSURE = 22,  /* PressureError::InvalidInitialPressure */
};

typedef struct orc_grid {
    uint64_t counts[3];
    double spacing[3];
    double origin[3];
} orc_grid;

typedef struct orc_settings {
    double relative_residual;
    double absolute_residual;
    double divergence_limit;
    uint64_t max_iterations;
} orc_settings;

typedef struct orc_report {
    uint64_t iterations;
    double true_residual_l2;
    double true_residual_max;
    double predicted_divergence_max;
    /* IncompatibleRhs payload (sum, rounding_budget); Breakdown iteration. */
    double incompatible_sum;
    double incompatible_budget;
    uint64_t breakdown_iteration;
} orc_report;

/* Per-iteration scalars of the PCG recurrence (for per-iteration parity). */
typedef struct orc_trace {
    double curvature;   /* d.Kd                       */
    double alpha;       /* rz / curvature             */
    double recursive_l2;/* sqrt(r.r) after the update */
    double rz;          /* r.z after preconditioning  */
    double beta;        /* next_rz / rz (0 if replaced)*/
    uint32_t replaced;  /* 1 when the true residual replaced r */
    uint32_t checked;   /* 1 when a true residual was evaluated */
} orc_trace;

enum { ORC_JACOBI_PCG_V1 = 0, ORC_SGS_PCG_V1 = 1 };

int orc_grid_validate(const orc_grid* g);

/* Sampling (sampling.rs). axis 0..2 samples that face field, 3 samples cells. */
int orc_sample(const orc_grid* g, int axis, const float* values, const double position[3],
               double* out);
int orc_backtrace(const orc_grid* g, const float* u, const float* v, const float* w,
                  const double position[3], double dt, double out[3]);

/* Advection (advection.rs). f32 storage is the reference; f64 storage keeps
 * the same formulas with the `as f32` casts removed. */
int orc_advect_velocity_f32(const orc_grid* g, const float* u, const float* v, const float* w,
                            double dt, float* ou, float* ov, float* ow, int threads);
int orc_advect_velocity_f64(const orc_grid* g, const double* u, const double* v, const double* w,
                            double dt, double* ou, double* ov, double* ow, int threads);
int orc_advect_tracer_f32(const orc_grid* g, const float* old, const float* u, const float* v,
                          const float* w, double dt, float* out, int threads);

/* Operator (operator.rs). */
int orc_apply_full(const orc_grid* g, double density, const double* p, double* out, int threads);
int orc_build_rhs_f32(const orc_grid* g, double density, const float* u, const float* v,
                      const float* w, double dt, double* out);
int orc_build_rhs_f64(const orc_grid* g, double density, const double* u, const double* v,
                      const double* w, double dt, double* out);
int orc_divergence_f32(const orc_grid* g, const float* u, const float* v, const float* w,
                       double* out);
int orc_divergence_f64(const orc_grid* g, const double* u, const double* v, const double* w,
                       double* out);
int orc_correct_f32(const orc_grid* g, double density, const double* p, double dt, float* u,
                    float* v, float* w);
int orc_correct_f64(const orc_grid* g, double density, const double* p, double dt, double* u,
                    double* v, double* w);
double orc_diagonal(const orc_grid* g, double density, const uint64_t coordinate[3]);

/* Reductions (pressure.rs). */
double orc_compensated_sum(const double* values, size_t n);
double orc_dot(const double* a, const double* b, size_t n);

/* Preconditioners on a residual r (r[0] is zeroed); z receives M^-1 r.
 * Returns r.z through *rz. */
int orc_precondition(const orc_grid* g, double density, int method, double* r, double* z,
                     double* rz);

/* PressureWorkspace::solve_rhs. pressure_out holds the iterate on every exit
 * that reaches the loop (including ITERATION_LIMIT). trace (optional) gets one
 * entry per iteration, up to trace_capacity. */
int orc_solve_rhs(const orc_grid* g, double density, int method, const double* rhs, double dt,
                  const orc_settings* s, double* pressure_out, orc_report* report,
                  orc_trace* trace, size_t trace_capacity, int threads);
/* solve_rhs_with_initial_pressure (seeded PCG); initial == NULL is solve_rhs. */
int orc_solve_rhs_initial(const orc_grid* g, double density, int method, const double* rhs,
                          const double* initial, double dt, const orc_settings* s, double* pressure_out,
                          orc_report* report, orc_trace* trace, size_t trace_capacity, int threads);

/* ProviderWorkspace host qualification of a supplied pressure candidate.
 * Returns ORC_OK, ORC_NONFINITE_OUTPUT, ORC_NONZERO_GAUGE or ORC_QUALITY_GATE;
 * the recomputed diagnostics go to *report either way. */
int orc_qualify_pressure(const orc_grid* g, double density, const double* rhs, double dt,
                         const orc_settings* s, const double* pressure, orc_report* report);

/* simulation.rs helpers. */
int orc_velocity_rate_f32(const orc_grid* g, const float* u, const float* v, const float* w,
                          double* rate);
int orc_velocity_rate_f64(const orc_grid* g, const double* u, const double* v, const double* w,
                          double* rate);
double orc_max_abs(const double* values, size_t n);

/* One carrier step on f32 or f64 faces, composed from the public primitives
 * exactly as Rheon's step owner orders them: advect -> (optional Y-face
 * buoyancy from the tracer) -> build_rhs -> PCG -> correct -> actual divergence
 * -> Courant -> tracer advection with the corrected velocity.
 * faces[0..2] hold the accepted velocity on entry and the corrected candidate on
 * exit (also on failure, as scratch). tracer may be NULL.
 * If iteration_limit_ok is nonzero, an IterationLimit from the PCG still
 * proceeds to the correction with the iterate (exact-iteration-count mode). */
typedef struct orc_step_params {
    double dt;
    double density;
    int method;
    orc_settings settings;
    double buoyancy;          /* g_b; 0 disables the buoyancy hook */
    int iteration_limit_ok;
    int threads;
} orc_step_params;

typedef struct orc_step_report {
    orc_report pressure;
    int pressure_status;
    double actual_divergence_max;
    double courant;
    double rate_before;
} orc_step_report;

int orc_carrier_step_f32(const orc_grid* g, const orc_step_params* prm, float* u, float* v,
                         float* w, float* tracer, orc_step_report* rep);
int orc_carrier_step_f64(const orc_grid* g, const orc_step_params* prm, double* u, double* v,
                         double* w, float* tracer, orc_step_report* rep);
/* The same step with the solve seeded by `initial` (NULL: cold), the step's
 * pressure copied to `pressure_out` (NULL: not kept). */
int orc_carrier_step_seeded_f32(const orc_grid* g, const orc_step_params* prm, float* u, float* v,
                                float* w, float* tracer, const double* initial, double* pressure_out,
                                orc_step_report* rep);
int orc_carrier_step_seeded_f64(const orc_grid* g, const orc_step_params* prm, double* u, double* v,
                                double* w, float* tracer, const double* initial, double* pressure_out,
                                orc_step_report* rep);

/* dense3D accepted-state frame (src/dense3d_sequence.rs:412-564): one JSON
 * line with Rust's `{:.9e}` text for the f32 fields (velocity_x/y/z, tracer)
 * and `{:.17e}` for the f64 fields (fraction, pressure) and the clocks and
 * diagnostics. Numbers come from the C library's exact "%.*e" conversion
 * (round half to even on the exact binary value), with the exponent rewritten
 * the Rust way (no '+', no leading zeros). tracer / fraction may be NULL
 * (zeros). Returns 0, or 23 (invalid state: the preflight of
 * src/dense3d_sequence.rs:419-494 failed; nothing is written), or 24 when
 * `capacity` is too small; *length receives the line's byte count. */
typedef struct orc_dense3d_frame {
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
} orc_dense3d_frame;

int orc_dense3d_frame_text(const orc_grid* g, const orc_dense3d_frame* frame, const float* u, const float* v,
                           const float* w, const float* tracer, const double* fraction, const double* pressure,
                           char* out, size_t capacity, size_t* length);

/* Liquid-volume transport, LiquidVolumeState::prepare_with_boundary with an
 * inlet boundary, the all-cells divergence domain and no reconstructed
 * columns (src/liquid_volume.rs:520-776), plus the flow-interval, inlet and
 * source validations (:123-150, :84-96, :185-190) and validate_advance
 * (:485-506). `accepted` is the state's fraction (x-fastest), `candidate`
 * receives the new fraction on success. inlet[2 d + s]: the outside fraction
 * of axis d, side s (0 lower, 1 upper). source may be NULL. periodic != 0 is
 * advance_periodic (src/liquid_volume.rs:389-406): the inlet is unused, seams
 * must carry equal velocities (PeriodicVelocityMismatch: error_cell = the
 * lower seam face, error_actual = the axis), the upper seam face repeats the
 * lower one's transfer, and no boundary volume is counted. Returns 0 or the
 * rb200_liquid_error code of the first failure, with its payload in the
 * report. */
typedef struct orc_liquid_report {
    double dt, time;
    double liquid_volume_before, liquid_volume_after;
    double inward_boundary_volume, outward_boundary_volume, source_volume;
    double volume_balance_error, volume_rounding_budget;
    double liquid_mass_before, liquid_mass_after;
    double max_outward_courant, actual_divergence_max;
    double fraction_min, fraction_max;
    uint64_t dry_cells, mixed_cells, full_cells;
    uint64_t error_cell;     /* CourantLimit, FractionBounds, InvalidFraction */
    double error_actual;     /* CourantLimit/DivergenceLimit actual, FractionBounds fraction, BalanceLimit error */
    double error_limit;      /* CourantLimit/DivergenceLimit limit, BalanceLimit rounding budget */
} orc_liquid_report;

int orc_liquid_advance(const orc_grid* g, double density, double state_time, uint64_t state_version,
                       const double* accepted, double* candidate, const float* u, const float* v, const float* w,
                       double start, double dt, const double inlet[6], const double* source_rate,
                       double max_outward_courant, double actual_divergence_limit, int periodic,
                       orc_liquid_report* rep);
/* LiquidVolumeState::new validation (src/liquid_volume.rs:276-305): 0 or the
 * error code (InvalidDensity, InvalidFraction with *cell, ArithmeticFailure). */
int orc_liquid_validate_state(const orc_grid* g, double density, const double* fraction, uint64_t* cell);

/* Box-flux projection, BoxFluxWorkspace::project (src/box_flux.rs:213-397):
 * the provisional faces' boundary samples are replaced by the prescribed
 * outward speeds outward[2 d + s] (s = 0 lower, 1 upper side of axis d), the
 * known net outward flux must vanish within 64 eps of its magnitude, the
 * pressure is solved with the RHS of the imposed field, interior faces are
 * corrected, and the interior energy ledger is formed (plain serial sums, as
 * the reference). Returns 0, an orc status (12 NonFiniteInput, 14
 * ArithmeticFailure, 10 invalid dt or settings, a PressureError code of the
 * solve), 28 IncompatibleFlux (net, rounding budget in the report) or 15
 * DivergenceLimit. out_* receive the projected faces (untouched before the
 * correction), pressure_out the pressure. */
typedef struct orc_box_flux_report {
    orc_report pressure;
    int pressure_status;
    double actual_divergence_max;
    double net_outward_flux, flux_rounding_budget;
    double kinetic_before, kinetic_after, correction_energy;
    double boundary_pressure_work, divergence_residual_work, correction_residual_work, budget_error;
} orc_box_flux_report;

int orc_box_flux_project(const orc_grid* g, double density, int method, const float* u, const float* v,
                         const float* w, double dt, const float outward[6], const orc_settings* pressure,
                         double actual_divergence_limit, float* out_u, float* out_v, float* out_w,
                         double* pressure_out, orc_box_flux_report* rep);

/* The step owner with its forcing and boundary domains
 * (Simulation::step / step_with_forces / step_with_box_flux,
 * src/simulation.rs:393-581, prepare_impl :812-1403) on f32 faces and an f32
 * tracer: dt policy with the smoke and body-force accelerations, advection,
 * the smoke source's Y-face force (apply_force :1449-1472), the body forces
 * (src/forces.rs:144-212), the sealed projection or the box-flux projection
 * (outward != NULL), the divergence and Courant gates, tracer advection, the
 * smoke source's tracer (apply_source :1473-1496), the tracer range check and
 * the box-flux step's work ledger (src/box_flux_step.rs). The state is
 * updated only on success. Returns 0, an orc status, or 29 with
 * report.error = 1 InvalidSource, 2 InvalidForce, 3 TimeResolution. */
typedef struct orc_smoke_source {
    double lower[3], upper[3];
    double tracer_rate, vertical_acceleration;
} orc_smoke_source;

typedef struct orc_body_force {
    double value[3];
    int units;       /* 0 Acceleration, 1 ForceDensity */
    int has_region;
    double lower[3], upper[3];
} orc_body_force;

typedef struct orc_sim_config {
    double density;
    int method;
    orc_settings pressure;
    double actual_divergence_limit, max_courant;
} orc_sim_config;

typedef struct orc_sim_state {
    float *u, *v, *w, *tracer;
    double time;
    uint64_t generation;
} orc_sim_state;

typedef struct orc_sim_report {
    double dt, time;
    uint64_t generation;
    orc_report pressure;
    double actual_divergence_max, courant, tracer_integral, kinetic_energy;
    int has_forces;
    double force_kinetic_before, force_kinetic_after, force_applied_work;
    orc_box_flux_report projection;
    double kinetic_old, kinetic_after_advection, kinetic_after_smoke_force, kinetic_before_projection,
        kinetic_accepted, advection_change, smoke_force_work, external_force_work, budget_error,
        boundary_volume_imbalance, tracer_old_integral, tracer_transport_change, tracer_source_change;
    int error;
    double error_actual, error_limit;
} orc_sim_report;

int orc_sim_step(const orc_grid* g, const orc_sim_config* config, orc_sim_state* state, double requested_dt,
                 const orc_smoke_source* source, const orc_body_force* forces, size_t force_count,
                 const float* outward, orc_sim_report* rep);

#ifdef __cplusplus
}
#endif
#endif
