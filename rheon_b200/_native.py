"""ctypes declarations for librheon_b200.so (the C ABI of include/rheon_b200.h).

There is no fallback: importing the package on a machine without the built
library raises ImportError, and every compute call goes to the CUDA library.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librheon_b200.so")

OK = 0
UNSUPPORTED = 1
EXECUTION = 2
NONFINITE_OUTPUT = 3
NONZERO_GAUGE = 4
QUALITY_GATE = 5
CANCELLED = 6
ITERATION_LIMIT = 7
BREAKDOWN = 8
OUT_OF_MEMORY = 9
INVALID_ARGUMENT = 10
INCOMPATIBLE_RHS = 11
NONFINITE_INPUT = 12
NONZERO_WALL_VELOCITY = 13
ARITHMETIC_FAILURE = 14
DIVERGENCE_LIMIT = 15
COURANT_LIMIT = 16
NO_DEVICE = 17
LENGTH_MISMATCH = 18
INVALID_INITIAL_PRESSURE = 22
DENSE3D_INVALID_STATE = 23
DENSE3D_LIMIT = 24
DENSE3D_ABORTED = 25
DENSE3D_IO = 26
LIQUID_REJECTED = 27
BOX_FLUX_REJECTED = 28
SIMULATION_REJECTED = 29

STATUS_NAMES = {
    0: "Ok", 1: "Unsupported", 2: "Execution", 3: "NonFiniteOutput", 4: "NonZeroGauge", 5: "QualityGate",
    6: "Cancelled", 7: "IterationLimit", 8: "Breakdown", 9: "AllocationFailed", 10: "InvalidArgument",
    11: "IncompatibleRhs", 12: "NonFiniteInput", 13: "NonZeroWallVelocity", 14: "ArithmeticFailure",
    15: "DivergenceLimit", 16: "CourantLimit", 17: "NoDevice", 18: "LengthMismatch",
    22: "InvalidInitialPressure", 23: "InvalidState", 24: "Limit", 25: "Aborted", 26: "Io", 27: "LiquidRejected",
    28: "BoxFluxRejected", 29: "SimulationRejected",
}

# rb200_liquid_error: LiquidVolumeError variants (src/liquid_volume.rs:27-72)
LIQUID_ERRORS = {0: "Ok", 1: "InvalidDensity", 2: "InvalidFraction", 3: "InvalidInlet", 4: "InvalidSource",
                 5: "InvalidSettings", 6: "InvalidTimeStep", 7: "TimeResolution", 8: "TimeMismatch",
                 9: "LengthMismatch", 10: "NonFiniteVelocity", 11: "VersionOverflow", 12: "BufferLimit",
                 13: "CourantLimit", 14: "DivergenceLimit", 15: "FractionBounds", 16: "BalanceLimit",
                 17: "ArithmeticFailure", 18: "Cancelled", 19: "GeometryMismatch", 20: "PeriodicVelocityMismatch"}

# rb200_volume_stage: VolumeStage (src/liquid_volume.rs:18-23)
VOLUME_STAGES = ("BeforeFlux", "FaceFluxSlice", "CellUpdateSlice", "BeforeCommit")

# rb200_box_flux_error: BoxFluxError's own variants (src/box_flux.rs:60-72)
BOX_FLUX_ERRORS = {0: "Ok", 1: "InvalidBoundary", 2: "InvalidSettings", 3: "InvalidMass", 4: "BufferLimit",
                   5: "IncompatibleFlux", 6: "Cancelled", 7: "DivergenceLimit", 8: "ArithmeticFailure"}
# rb200_box_flux_stage: BoxFluxStage (src/box_flux.rs:53-59)
BOX_FLUX_STAGES = ("BeforeSolve", "PressureIteration", "CorrectionSlice", "BeforeAcceptance")


class Grid(C.Structure):
    _fields_ = [("counts", C.c_uint64 * 3), ("spacing", C.c_double * 3), ("origin", C.c_double * 3)]


class Settings(C.Structure):
    _fields_ = [("relative_residual", C.c_double), ("absolute_residual", C.c_double),
                ("divergence_limit", C.c_double), ("max_iterations", C.c_uint64)]


class Report(C.Structure):
    _fields_ = [("iterations", C.c_uint64), ("true_residual_l2", C.c_double), ("true_residual_max", C.c_double),
                ("predicted_divergence_max", C.c_double), ("incompatible_sum", C.c_double),
                ("incompatible_budget", C.c_double), ("breakdown_iteration", C.c_uint64)]


class Trace(C.Structure):
    _fields_ = [("curvature", C.c_double), ("alpha", C.c_double), ("recursive_l2", C.c_double),
                ("rz", C.c_double), ("beta", C.c_double), ("replaced", C.c_uint32), ("checked", C.c_uint32)]


class ProviderConfig(C.Structure):
    _fields_ = [("grid", Grid), ("density", C.c_double), ("method", C.c_int), ("settings", Settings),
                ("device", C.c_int)]


class Request(C.Structure):
    _fields_ = [("grid", Grid), ("density", C.c_double), ("dt", C.c_double), ("rhs", C.c_void_p),
                ("len", C.c_size_t)]


class Metadata(C.Structure):
    _fields_ = [(n, C.c_char_p) for n in ("id", "version", "stage", "input_layout", "input_scalar", "input_units",
                                          "output_layout", "output_scalar", "output_units", "domain")] + [
        ("shape_xyz", C.c_uint64 * 3)]


class CarrierConfig(C.Structure):
    _fields_ = [("grid", Grid), ("density", C.c_double), ("storage", C.c_int), ("method", C.c_int),
                ("settings", Settings), ("actual_divergence_limit", C.c_double), ("max_courant", C.c_double),
                ("with_tracer", C.c_int), ("device", C.c_int), ("fp32_advection", C.c_int),
                ("warm_start", C.c_int)]


class BatchConfig(C.Structure):
    _fields_ = [("density", C.c_double), ("settings", Settings), ("actual_divergence_limit", C.c_double),
                ("max_courant", C.c_double), ("device", C.c_int), ("fp32_advection", C.c_int)]


class StepParams(C.Structure):
    _fields_ = [("requested_dt", C.c_double), ("cfl", C.c_double), ("buoyancy", C.c_double),
                ("iteration_limit_ok", C.c_int), ("skip_gates", C.c_int)]


class StepReport(C.Structure):
    _fields_ = [("dt", C.c_double), ("time", C.c_double), ("generation", C.c_uint64), ("pressure", Report),
                ("pressure_status", C.c_int), ("actual_divergence_max", C.c_double), ("courant", C.c_double),
                ("velocity_rate", C.c_double), ("pressure_ms", C.c_double),
                ("kernel_launches", C.c_uint64), ("pressure_initialization", C.c_int)]


CANCEL_FN = C.CFUNCTYPE(C.c_int, C.c_void_p)

class Dense3dFrame(C.Structure):
    _fields_ = [("frame", C.c_uint64), ("time_s", C.c_double), ("dt_s", C.c_double),
                ("carrier_stamp_id", C.c_uint64), ("carrier_stamp_version", C.c_uint64),
                ("liquid_stamp_id", C.c_uint64), ("liquid_stamp_version", C.c_uint64),
                ("has_diagnostics", C.c_int), ("pressure_iterations", C.c_uint64),
                ("pressure_residual_m3_s2", C.c_double), ("carrier_divergence_s_inv", C.c_double),
                ("liquid_divergence_s_inv", C.c_double), ("volume_before_m3", C.c_double),
                ("volume_after_m3", C.c_double), ("mass_after_kg", C.c_double), ("inward_m3", C.c_double),
                ("outward_m3", C.c_double), ("source_m3", C.c_double), ("balance_m3", C.c_double),
                ("rounding_budget_m3", C.c_double)]


class Dense3dFields(C.Structure):
    _fields_ = [("velocity_storage", C.c_int), ("u", C.c_void_p), ("v", C.c_void_p), ("w", C.c_void_p),
                ("tracer", C.c_void_p), ("fraction", C.c_void_p), ("pressure", C.c_void_p)]


class Dense3dLimits(C.Structure):
    _fields_ = [("max_cells", C.c_uint64), ("max_frames", C.c_uint64), ("max_bytes", C.c_uint64)]


class LiquidStamp(C.Structure):
    _fields_ = [("id", C.c_uint64), ("version", C.c_uint64)]


class LiquidFlow(C.Structure):
    _fields_ = [("stamp", LiquidStamp), ("u", C.c_void_p), ("v", C.c_void_p), ("w", C.c_void_p),
                ("start", C.c_double), ("dt", C.c_double)]


class LiquidInlet(C.Structure):
    _fields_ = [("stamp", LiquidStamp), ("fraction", C.c_double * 6)]


class LiquidSource(C.Structure):
    _fields_ = [("stamp", LiquidStamp), ("rate", C.c_void_p)]


class LiquidSettings(C.Structure):
    _fields_ = [("max_outward_courant", C.c_double), ("actual_divergence_limit", C.c_double)]


class LiquidReport(C.Structure):
    _fields_ = ([("stamp", LiquidStamp), ("flow", LiquidStamp), ("inlet", LiquidStamp), ("source", LiquidStamp),
                 ("has_source", C.c_int), ("periodic", C.c_int)] +
                [(n, C.c_double) for n in ("dt", "time", "liquid_volume_before", "liquid_volume_after",
                                           "inward_boundary_volume", "outward_boundary_volume", "source_volume",
                                           "volume_balance_error", "volume_rounding_budget", "liquid_mass_before",
                                           "liquid_mass_after", "max_outward_courant", "actual_divergence_max",
                                           "fraction_min", "fraction_max")] +
                [(n, C.c_uint64) for n in ("dry_cells", "mixed_cells", "full_cells")] +
                [("error", C.c_int), ("error_cell", C.c_uint64), ("error_actual", C.c_double),
                 ("error_limit", C.c_double)])


class BoxFluxBoundary(C.Structure):
    _fields_ = [("id", C.c_uint64), ("version", C.c_uint64), ("outward", C.c_float * 6)]


class BoxFluxReport(C.Structure):
    _fields_ = ([("boundary_id", C.c_uint64), ("boundary_version", C.c_uint64), ("pressure", Report)] +
                [(n, C.c_double) for n in ("actual_divergence_max", "net_outward_flux", "flux_rounding_budget",
                                           "kinetic_before", "kinetic_after", "correction_energy",
                                           "boundary_pressure_work", "divergence_residual_work",
                                           "correction_residual_work", "budget_error")] +
                [("error", C.c_int), ("stage", C.c_int), ("error_actual", C.c_double),
                 ("error_limit", C.c_double), ("required", C.c_uint64), ("limit", C.c_uint64)])


BOX_FLUX_CANCEL_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int)

# rb200_step_stage: StepStage (src/simulation.rs:28-42)
STEP_STAGES = ("BeforeAdvection", "VelocitySlice", "BeforeForces", "ForceSlice", "Viscosity", "BeforePressure",
               "PressureIteration", "ProjectionSlice", "BeforeProjectionAcceptance", "BeforeTracer", "TracerSlice",
               "BeforeCommit", "LiquidBeforeCommit")
# rb200_simulation_error: SimulationError's own variants
SIMULATION_ERRORS = {0: "Ok", 1: "InvalidSource", 2: "InvalidForce", 3: "TimeResolution",
                     4: "BoundaryWorkspaceMismatch", 5: "Cancelled"}
STEP_CANCEL_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int)


class SmokeSourceC(C.Structure):
    _fields_ = [("lower", C.c_double * 3), ("upper", C.c_double * 3), ("tracer_rate", C.c_double),
                ("vertical_acceleration", C.c_double)]


class BodyForceC(C.Structure):
    _fields_ = [("value", C.c_double * 3), ("units", C.c_int), ("has_region", C.c_int),
                ("lower", C.c_double * 3), ("upper", C.c_double * 3)]


class ForcedStepParams(C.Structure):
    _fields_ = [("requested_dt", C.c_double), ("source", C.POINTER(SmokeSourceC)),
                ("forces", C.POINTER(BodyForceC)), ("force_count", C.c_size_t), ("box_flux", C.c_void_p),
                ("boundary", C.POINTER(BoxFluxBoundary)), ("tracer_policy", C.c_int)]


FORCED_WORK = ("kinetic_old", "kinetic_after_advection", "kinetic_after_smoke_force", "kinetic_before_projection",
               "kinetic_accepted", "advection_change", "smoke_force_work", "external_force_work", "budget_error",
               "boundary_volume_imbalance", "tracer_old_integral", "tracer_transport_change",
               "tracer_source_change")


class ForcedStepReport(C.Structure):
    _fields_ = ([("dt", C.c_double), ("time", C.c_double), ("generation", C.c_uint64), ("pressure", Report)] +
                [(n, C.c_double) for n in ("actual_divergence_max", "courant", "tracer_integral", "kinetic_energy")] +
                [("has_forces", C.c_int), ("has_boundary", C.c_int)] +
                [(n, C.c_double) for n in ("force_kinetic_before", "force_kinetic_after", "force_applied_work")] +
                [("projection", BoxFluxReport)] + [(n, C.c_double) for n in FORCED_WORK] +
                [("tracer_policy", C.c_int), ("error", C.c_int), ("stage", C.c_int), ("pad", C.c_int),
                 ("error_actual", C.c_double), ("error_limit", C.c_double),
                 ("simulation_array_bytes", C.c_uint64), ("boundary_workspace_array_bytes", C.c_uint64)])

_P = C.c_void_p
_I = C.c_int
_D = C.c_double
_S = C.c_size_t

# name -> (restype, argtypes); every symbol here is declared in include/rheon_b200.h
SIGNATURES = {
    "rb200_abi_version": (_I, []),
    "rb200_status_string": (C.c_char_p, [_I]),
    "rb200_device_count": (_I, []),
    "rb200_provider_create": (_I, [C.POINTER(ProviderConfig), C.POINTER(_P)]),
    "rb200_provider_destroy": (None, [_P]),
    "rb200_provider_metadata": (_I, [_P, C.POINTER(Metadata)]),
    "rb200_provider_supports": (_I, [_P, C.POINTER(Request)]),
    "rb200_provider_predict": (_I, [_P, C.POINTER(Request), _P, _S, CANCEL_FN, _P]),
    "rb200_provider_last_error": (C.c_char_p, [_P]),
    "rb200_provider_last_report": (_I, [_P, C.POINTER(Report), C.POINTER(_I)]),
    "rb200_workspace_create": (_I, [C.POINTER(Grid), _D, _I, C.c_uint64, _I, C.POINTER(_P)]),
    "rb200_workspace_destroy": (None, [_P]),
    "rb200_workspace_allocated_bytes": (C.c_uint64, [_P]),
    "rb200_workspace_stream": (_P, [_P]),
    "rb200_workspace_solve_rhs": (_I, [_P, _P, _S, _D, C.POINTER(Settings), C.POINTER(Report), CANCEL_FN, _P]),
    "rb200_workspace_solve_rhs_initial": (_I, [_P, _P, _P, _S, _D, C.POINTER(Settings), C.POINTER(Report),
                                               CANCEL_FN, _P]),
    "rb200_workspace_solve_rhs_device": (_I, [_P, _P, _S, _D, C.POINTER(Settings), C.POINTER(Report), CANCEL_FN,
                                              _P]),
    "rb200_workspace_pressure": (_I, [_P, _P, _S]),
    "rb200_workspace_pressure_device": (_P, [_P]),
    "rb200_workspace_set_trace": (_I, [_P, _P, _S]),
    "rb200_workspace_profile": (_I, [_P, _I, _I, C.POINTER(_D)]),
    "rb200_pressure_solve_static": (_I, [C.POINTER(Grid), _D, _P, _P, _S, _D, C.POINTER(Settings),
                                         C.POINTER(Report), _P]),
    "rb200_apply_full_device": (_I, [C.POINTER(Grid), _D, _P, _P, _P]),
    "rb200_qualify_pressure_device": (_I, [C.POINTER(Grid), _D, _P, _P, C.c_size_t, _D, C.POINTER(Settings),
                                           C.POINTER(Report), _P]),
    "rb200_projection_witness_f32_device": (_I, [C.POINTER(Grid), _D, _P, _D, _P, _P, _P, _P, _P, _P,
                                                 C.POINTER(C.c_int), C.POINTER(C.c_uint64), _P]),
    "rb200_projection_witness_f64_device": (_I, [C.POINTER(Grid), _D, _P, _D, _P, _P, _P, _P, _P, _P,
                                                 C.POINTER(C.c_int), C.POINTER(C.c_uint64), _P]),
    "rb200_precondition_jacobi_device": (_I, [C.POINTER(Grid), _D, _P, _P, C.c_size_t, C.POINTER(_D), _P]),
    "rb200_build_rhs_f32_device": (_I, [C.POINTER(Grid), _D, _P, _P, _P, _D, _P, _P]),
    "rb200_build_rhs_f64_device": (_I, [C.POINTER(Grid), _D, _P, _P, _P, _D, _P, _P]),
    "rb200_divergence_f32_device": (_I, [C.POINTER(Grid), _P, _P, _P, _P, _P]),
    "rb200_divergence_f64_device": (_I, [C.POINTER(Grid), _P, _P, _P, _P, _P]),
    "rb200_correct_f32_device": (_I, [C.POINTER(Grid), _D, _P, _D, _P, _P, _P, _P]),
    "rb200_correct_f64_device": (_I, [C.POINTER(Grid), _D, _P, _D, _P, _P, _P, _P]),
    "rb200_advect_velocity_f32_device": (_I, [C.POINTER(Grid), _P, _P, _P, _D, _P, _P, _P, _P]),
    "rb200_advect_velocity_f64_device": (_I, [C.POINTER(Grid), _P, _P, _P, _D, _P, _P, _P, _P]),
    "rb200_advect_tracer_f32_device": (_I, [C.POINTER(Grid), _P, _P, _P, _P, _D, _P, _P]),
    "rb200_carrier_create": (_I, [C.POINTER(CarrierConfig), C.POINTER(_P)]),
    "rb200_carrier_destroy": (None, [_P]),
    "rb200_carrier_allocated_bytes": (C.c_uint64, [_P]),
    "rb200_carrier_stream": (_P, [_P]),
    "rb200_carrier_upload": (_I, [_P, _P, _P, _P, _P]),
    "rb200_carrier_download": (_I, [_P, _P, _P, _P, _P]),
    "rb200_carrier_init_fourier": (_I, [_P, C.c_uint64, _I, _P, _P, _P, _D, _D]),
    "rb200_carrier_state_device": (_I, [_P, C.POINTER(_P), C.POINTER(_P), C.POINTER(_P), C.POINTER(_P)]),
    "rb200_carrier_step": (_I, [_P, C.POINTER(StepParams), C.POINTER(StepReport), CANCEL_FN, _P]),
    "rb200_carrier_step_async": (_I, [_P, C.POINTER(StepParams)]),
    "rb200_carrier_project": (_I, [_P, C.POINTER(StepParams), C.POINTER(StepReport)]),
    "rb200_carrier_project_async": (_I, [_P, C.POINTER(StepParams)]),
    "rb200_carrier_step_wait": (_I, [_P, C.POINTER(StepReport)]),
    "rb200_carrier_step_poll": (_I, [_P]),
    "rb200_carriers_step": (_I, [C.POINTER(_P), _S, C.POINTER(StepParams), C.POINTER(StepReport), C.POINTER(_I)]),
    "rb200_batch_create": (_I, [C.POINTER(Grid), _S, C.POINTER(BatchConfig), C.POINTER(_P)]),
    "rb200_batch_destroy": (None, [_P]),
    "rb200_batch_allocated_bytes": (C.c_uint64, [_P]),
    "rb200_batch_stream": (_P, [_P]),
    "rb200_batch_last_error": (C.c_char_p, [_P]),
    "rb200_batch_upload": (_I, [_P, _S, _P, _P, _P]),
    "rb200_batch_download": (_I, [_P, _S, _P, _P, _P]),
    "rb200_batch_pressure": (_I, [_P, _S, _P, _S]),
    "rb200_batch_step": (_I, [_P, C.POINTER(StepParams), C.POINTER(StepReport), C.POINTER(_I)]),
    "rb200_batch_step_async": (_I, [_P, C.POINTER(StepParams)]),
    "rb200_batch_step_poll": (_I, [_P]),
    "rb200_batch_step_wait": (_I, [_P, C.POINTER(StepReport), C.POINTER(_I)]),
    "rb200_batch_profile_step": (_I, [_P, C.POINTER(StepParams), C.POINTER(StepReport), C.POINTER(_I),
                                      C.POINTER(_D), C.POINTER(_I), C.POINTER(C.c_char_p), _I]),
    "rb200_batch_profile_kinds": (_I, []),
    "rb200_carrier_profile": (_I, [_P, _I, _I, C.POINTER(_D)]),
    "rb200_carrier_pressure": (_I, [_P, _P, _S]),
    "rb200_carrier_dense3d_fields": (_I, [_P, C.POINTER(Dense3dFields)]),
    "rb200_dense3d_encoder_create": (_I, [C.POINTER(Grid), _I, C.POINTER(_P)]),
    "rb200_dense3d_encoder_destroy": (None, [_P]),
    "rb200_dense3d_frame_bound": (C.c_uint64, [_P]),
    "rb200_dense3d_encoder_error": (C.c_char_p, [_P]),
    "rb200_dense3d_encode": (_I, [_P, C.POINTER(Dense3dFrame), C.POINTER(Dense3dFields), _P, C.c_uint64,
                                  C.POINTER(C.c_uint64), _P]),
    "rb200_dense3d_text_f64": (_I, [_D, C.c_char_p, _S]),
    "rb200_dense3d_text_f32": (_I, [C.c_float, C.c_char_p, _S]),
    "rb200_dense3d_writer_create": (_I, [C.POINTER(Grid), C.POINTER(Dense3dLimits), _I, _I, C.POINTER(_P)]),
    "rb200_dense3d_writer_destroy": (None, [_P]),
    "rb200_dense3d_writer_frame": (_I, [_P, C.POINTER(Dense3dFrame), C.POINTER(Dense3dFields), _P]),
    "rb200_dense3d_writer_flush": (_I, [_P]),
    "rb200_dense3d_writer_sync": (_I, [_P]),
    "rb200_dense3d_writer_frames": (C.c_uint64, [_P]),
    "rb200_dense3d_writer_bytes": (C.c_uint64, [_P]),
    "rb200_dense3d_writer_aborted": (_I, [_P]),
    "rb200_dense3d_writer_error": (C.c_char_p, [_P]),
    "rb200_liquid_create": (_I, [C.POINTER(Grid), _D, LiquidStamp, _P, C.c_uint64, _I, C.POINTER(_P),
                                 C.POINTER(LiquidReport)]),
    "rb200_liquid_destroy": (None, [_P]),
    "rb200_liquid_allocated_bytes": (C.c_uint64, [_P]),
    "rb200_liquid_state": (_I, [_P, C.POINTER(_P), C.POINTER(LiquidStamp), C.POINTER(_D)]),
    "rb200_liquid_download": (_I, [_P, _P, _S]),
    "rb200_liquid_advance": (_I, [_P, C.POINTER(LiquidFlow), C.POINTER(LiquidInlet), C.POINTER(LiquidSource),
                                  C.POINTER(LiquidSettings), C.POINTER(LiquidReport), _P]),
    "rb200_liquid_advance_periodic": (_I, [_P, C.POINTER(LiquidFlow), LiquidStamp, C.POINTER(LiquidSource),
                                           C.POINTER(LiquidSettings), C.POINTER(LiquidReport), _P]),
    "rb200_liquid_advance_cancellable": (_I, [_P, C.POINTER(LiquidFlow), C.POINTER(LiquidInlet),
                                              C.POINTER(LiquidSource), C.POINTER(LiquidSettings), STEP_CANCEL_FN, _P,
                                              C.POINTER(LiquidReport), _P]),
    "rb200_liquid_advance_periodic_cancellable": (_I, [_P, C.POINTER(LiquidFlow), LiquidStamp,
                                                       C.POINTER(LiquidSource), C.POINTER(LiquidSettings),
                                                       STEP_CANCEL_FN, _P, C.POINTER(LiquidReport), _P]),
    "rb200_carrier_attach_liquid": (_I, [_P, _D, LiquidStamp, C.c_uint64, _P, C.c_uint64, C.POINTER(LiquidReport)]),
    "rb200_carrier_liquid_inputs": (_I, [_P, C.POINTER(LiquidInlet), C.POINTER(LiquidSource),
                                         C.POINTER(LiquidSettings)]),
    "rb200_carrier_liquid_report": (_I, [_P, C.POINTER(LiquidReport)]),
    "rb200_carrier_liquid_state": (_I, [_P, C.POINTER(_P), C.POINTER(LiquidStamp), C.POINTER(_D)]),
    "rb200_carrier_liquid_download": (_I, [_P, _P, _S]),
    "rb200_box_flux_create": (_I, [C.POINTER(Grid), _D, C.c_uint64, _I, _I, C.POINTER(_P),
                                   C.POINTER(BoxFluxReport)]),
    "rb200_box_flux_destroy": (None, [_P]),
    "rb200_box_flux_allocated_bytes": (C.c_uint64, [_P]),
    "rb200_box_flux_stream": (_P, [_P]),
    "rb200_box_flux_project_device": (_I, [_P, _P * 3, _S * 3, _D, C.POINTER(BoxFluxBoundary), C.POINTER(Settings),
                                           _D, _P * 3, _S * 3, C.POINTER(BoxFluxReport), BOX_FLUX_CANCEL_FN, _P]),
    "rb200_box_flux_project": (_I, [_P, _P * 3, _S * 3, _D, C.POINTER(BoxFluxBoundary), C.POINTER(Settings),
                                    _D, _P * 3, _S * 3, C.POINTER(BoxFluxReport), BOX_FLUX_CANCEL_FN, _P]),
    "rb200_box_flux_divergence_device": (_I, [_P, _P * 3, _S * 3, _P, _S]),
    "rb200_box_flux_pressure": (_I, [_P, _P, _S]),
    "rb200_box_flux_pressure_device": (_P, [_P]),
    "rb200_box_flux_profile": (_I, [_P, _I, _I, C.POINTER(_D)]),
    "rb200_box_flux_last_pass_ms": (_I, [_P, C.POINTER(_D), C.POINTER(_D)]),
    "rb200_carrier_step_forced": (_I, [_P, C.POINTER(ForcedStepParams), C.POINTER(ForcedStepReport),
                                       STEP_CANCEL_FN, _P]),
}

_lib = None


def lib():
    """Load librheon_b200.so; raise if it is not built (no fallback path)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is not built; run `python -m rheon_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


NO_CANCEL = CANCEL_FN()
