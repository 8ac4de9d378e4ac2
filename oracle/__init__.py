"""Oracle: ctypes binding of the CPU restatement of Rheon's carrier arithmetic.

TEST INFRASTRUCTURE ONLY. Imported by tests/, by ``__graft_entry__.smoke()`` and
by bench.py's CPU-baseline/reference arm, as the checker and the timed CPU
baseline. The product package ``rheon_b200`` never imports it.

The C++ source (oracle.cpp) restates, with the reference's operation order and
serial Neumaier reductions, src/{geometry,sampling,advection,operator,
pressure}.rs of the Rheon project; see oracle.h for the file:line map.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")

OK = 0
UNSUPPORTED = 1
NONFINITE_OUTPUT = 3
NONZERO_GAUGE = 4
QUALITY_GATE = 5
CANCELLED = 6
ITERATION_LIMIT = 7
BREAKDOWN = 8
INVALID_ARGUMENT = 10
INCOMPATIBLE_RHS = 11
NONFINITE_INPUT = 12
NONZERO_WALL_VELOCITY = 13
ARITHMETIC_FAILURE = 14
DIVERGENCE_LIMIT = 15
COURANT_LIMIT = 16
LENGTH_MISMATCH = 18
INVALID_GEOMETRY = 19
INVALID_TIME_STEP = 20
NONFINITE_POSITION = 21
INVALID_INITIAL_PRESSURE = 22

JACOBI_PCG_V1 = 0
SGS_PCG_V1 = 1


class Grid(C.Structure):
    _fields_ = [("counts", C.c_uint64 * 3), ("spacing", C.c_double * 3), ("origin", C.c_double * 3)]


class Settings(C.Structure):
    _fields_ = [
        ("relative_residual", C.c_double),
        ("absolute_residual", C.c_double),
        ("divergence_limit", C.c_double),
        ("max_iterations", C.c_uint64),
    ]


class Report(C.Structure):
    _fields_ = [
        ("iterations", C.c_uint64),
        ("true_residual_l2", C.c_double),
        ("true_residual_max", C.c_double),
        ("predicted_divergence_max", C.c_double),
        ("incompatible_sum", C.c_double),
        ("incompatible_budget", C.c_double),
        ("breakdown_iteration", C.c_uint64),
    ]


class Trace(C.Structure):
    _fields_ = [
        ("curvature", C.c_double),
        ("alpha", C.c_double),
        ("recursive_l2", C.c_double),
        ("rz", C.c_double),
        ("beta", C.c_double),
        ("replaced", C.c_uint32),
        ("checked", C.c_uint32),
    ]


class StepParams(C.Structure):
    _fields_ = [
        ("dt", C.c_double),
        ("density", C.c_double),
        ("method", C.c_int),
        ("settings", Settings),
        ("buoyancy", C.c_double),
        ("iteration_limit_ok", C.c_int),
        ("threads", C.c_int),
    ]


class StepReport(C.Structure):
    _fields_ = [
        ("pressure", Report),
        ("pressure_status", C.c_int),
        ("actual_divergence_max", C.c_double),
        ("courant", C.c_double),
        ("rate_before", C.c_double),
    ]


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


class LiquidReport(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "dt", "time", "liquid_volume_before", "liquid_volume_after", "inward_boundary_volume",
        "outward_boundary_volume", "source_volume", "volume_balance_error", "volume_rounding_budget",
        "liquid_mass_before", "liquid_mass_after", "max_outward_courant", "actual_divergence_max", "fraction_min",
        "fraction_max")] + [(n, C.c_uint64) for n in ("dry_cells", "mixed_cells", "full_cells", "error_cell")] + [
        ("error_actual", C.c_double), ("error_limit", C.c_double)]


# rb200_liquid_error (include/rheon_b200.h)
LIQUID_ERRORS = {0: "Ok", 1: "InvalidDensity", 2: "InvalidFraction", 3: "InvalidInlet", 4: "InvalidSource",
                 5: "InvalidSettings", 6: "InvalidTimeStep", 7: "TimeResolution", 8: "TimeMismatch",
                 9: "LengthMismatch", 10: "NonFiniteVelocity", 11: "VersionOverflow", 12: "BufferLimit",
                 13: "CourantLimit", 14: "DivergenceLimit", 15: "FractionBounds", 16: "BalanceLimit",
                 17: "ArithmeticFailure", 18: "Cancelled", 19: "GeometryMismatch", 20: "PeriodicVelocityMismatch"}


class BoxFluxReport(C.Structure):
    _fields_ = [("pressure", Report), ("pressure_status", C.c_int)] + [(n, C.c_double) for n in (
        "actual_divergence_max", "net_outward_flux", "flux_rounding_budget", "kinetic_before", "kinetic_after",
        "correction_energy", "boundary_pressure_work", "divergence_residual_work", "correction_residual_work",
        "budget_error")]


class SmokeSource(C.Structure):
    _fields_ = [("lower", C.c_double * 3), ("upper", C.c_double * 3), ("tracer_rate", C.c_double),
                ("vertical_acceleration", C.c_double)]


class BodyForce(C.Structure):
    _fields_ = [("value", C.c_double * 3), ("units", C.c_int), ("has_region", C.c_int),
                ("lower", C.c_double * 3), ("upper", C.c_double * 3)]


class SimConfig(C.Structure):
    _fields_ = [("density", C.c_double), ("method", C.c_int), ("pressure", Settings),
                ("actual_divergence_limit", C.c_double), ("max_courant", C.c_double)]


class SimState(C.Structure):
    _fields_ = [("u", C.c_void_p), ("v", C.c_void_p), ("w", C.c_void_p), ("tracer", C.c_void_p),
                ("time", C.c_double), ("generation", C.c_uint64)]


SIM_WORK = ("kinetic_old", "kinetic_after_advection", "kinetic_after_smoke_force", "kinetic_before_projection",
            "kinetic_accepted", "advection_change", "smoke_force_work", "external_force_work", "budget_error",
            "boundary_volume_imbalance", "tracer_old_integral", "tracer_transport_change", "tracer_source_change")


class SimReport(C.Structure):
    _fields_ = ([("dt", C.c_double), ("time", C.c_double), ("generation", C.c_uint64), ("pressure", Report)] +
                [(n, C.c_double) for n in ("actual_divergence_max", "courant", "tracer_integral", "kinetic_energy")] +
                [("has_forces", C.c_int)] +
                [(n, C.c_double) for n in ("force_kinetic_before", "force_kinetic_after", "force_applied_work")] +
                [("projection", BoxFluxReport)] + [(n, C.c_double) for n in SIM_WORK] +
                [("error", C.c_int), ("error_actual", C.c_double), ("error_limit", C.c_double)])


def build() -> str:
    """Compile the oracle with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = C.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


_P = C.c_void_p


def _declare(L):
    L.orc_grid_validate.argtypes = [C.POINTER(Grid)]
    L.orc_sample.argtypes = [C.POINTER(Grid), C.c_int, _P, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.orc_backtrace.argtypes = [C.POINTER(Grid), _P, _P, _P, C.POINTER(C.c_double), C.c_double, C.POINTER(C.c_double)]
    L.orc_advect_velocity_f32.argtypes = [C.POINTER(Grid), _P, _P, _P, C.c_double, _P, _P, _P, C.c_int]
    L.orc_advect_velocity_f64.argtypes = [C.POINTER(Grid), _P, _P, _P, C.c_double, _P, _P, _P, C.c_int]
    L.orc_advect_tracer_f32.argtypes = [C.POINTER(Grid), _P, _P, _P, _P, C.c_double, _P, C.c_int]
    L.orc_apply_full.argtypes = [C.POINTER(Grid), C.c_double, _P, _P, C.c_int]
    L.orc_build_rhs_f32.argtypes = [C.POINTER(Grid), C.c_double, _P, _P, _P, C.c_double, _P]
    L.orc_build_rhs_f64.argtypes = [C.POINTER(Grid), C.c_double, _P, _P, _P, C.c_double, _P]
    L.orc_divergence_f32.argtypes = [C.POINTER(Grid), _P, _P, _P, _P]
    L.orc_divergence_f64.argtypes = [C.POINTER(Grid), _P, _P, _P, _P]
    L.orc_correct_f32.argtypes = [C.POINTER(Grid), C.c_double, _P, C.c_double, _P, _P, _P]
    L.orc_correct_f64.argtypes = [C.POINTER(Grid), C.c_double, _P, C.c_double, _P, _P, _P]
    L.orc_diagonal.argtypes = [C.POINTER(Grid), C.c_double, C.POINTER(C.c_uint64)]
    L.orc_diagonal.restype = C.c_double
    L.orc_compensated_sum.argtypes = [_P, C.c_size_t]
    L.orc_compensated_sum.restype = C.c_double
    L.orc_dot.argtypes = [_P, _P, C.c_size_t]
    L.orc_dot.restype = C.c_double
    L.orc_precondition.argtypes = [C.POINTER(Grid), C.c_double, C.c_int, _P, _P, C.POINTER(C.c_double)]
    L.orc_solve_rhs.argtypes = [C.POINTER(Grid), C.c_double, C.c_int, _P, C.c_double, C.POINTER(Settings), _P,
                                C.POINTER(Report), _P, C.c_size_t, C.c_int]
    L.orc_qualify_pressure.argtypes = [C.POINTER(Grid), C.c_double, _P, C.c_double, C.POINTER(Settings), _P,
                                       C.POINTER(Report)]
    L.orc_velocity_rate_f32.argtypes = [C.POINTER(Grid), _P, _P, _P, C.POINTER(C.c_double)]
    L.orc_velocity_rate_f64.argtypes = [C.POINTER(Grid), _P, _P, _P, C.POINTER(C.c_double)]
    L.orc_max_abs.argtypes = [_P, C.c_size_t]
    L.orc_max_abs.restype = C.c_double
    L.orc_carrier_step_f32.argtypes = [C.POINTER(Grid), C.POINTER(StepParams), _P, _P, _P, _P, C.POINTER(StepReport)]
    L.orc_carrier_step_f64.argtypes = [C.POINTER(Grid), C.POINTER(StepParams), _P, _P, _P, _P, C.POINTER(StepReport)]
    L.orc_solve_rhs_initial.argtypes = [C.POINTER(Grid), C.c_double, C.c_int, _P, _P, C.c_double,
                                        C.POINTER(Settings), _P, C.POINTER(Report), _P, C.c_size_t, C.c_int]
    L.orc_liquid_advance.argtypes = [C.POINTER(Grid), C.c_double, C.c_double, C.c_uint64, _P, _P, _P, _P, _P,
                                     C.c_double, C.c_double, C.POINTER(C.c_double), _P, C.c_double, C.c_double,
                                     C.c_int, C.POINTER(LiquidReport)]
    L.orc_liquid_validate_state.argtypes = [C.POINTER(Grid), C.c_double, _P, C.POINTER(C.c_uint64)]
    L.orc_box_flux_project.argtypes = [C.POINTER(Grid), C.c_double, C.c_int, _P, _P, _P, C.c_double,
                                       C.POINTER(C.c_float), C.POINTER(Settings), C.c_double, _P, _P, _P, _P,
                                       C.POINTER(BoxFluxReport)]
    L.orc_dense3d_frame_text.argtypes = [C.POINTER(Grid), C.POINTER(Dense3dFrame), _P, _P, _P, _P, _P, _P,
                                         C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]
    L.orc_sim_step.argtypes = [C.POINTER(Grid), C.POINTER(SimConfig), C.POINTER(SimState), C.c_double,
                               C.POINTER(SmokeSource), C.POINTER(BodyForce), C.c_size_t, _P, C.POINTER(SimReport)]
    for name in ("orc_carrier_step_seeded_f32", "orc_carrier_step_seeded_f64"):
        getattr(L, name).argtypes = [C.POINTER(Grid), C.POINTER(StepParams), _P, _P, _P, _P, _P, _P,
                                     C.POINTER(StepReport)]


def grid(counts, spacing=(1.0, 1.0, 1.0), origin=(0.0, 0.0, 0.0)) -> Grid:
    g = Grid()
    for d in range(3):
        g.counts[d] = int(counts[d])
        g.spacing[d] = float(spacing[d])
        g.origin[d] = float(origin[d])
    return g


def settings(rel=1e-11, abs_=1e-12, div=1e-9, max_iterations=1000) -> Settings:
    return Settings(rel, abs_, div, max_iterations)


def face_counts(g: Grid, axis: int):
    n = [int(g.counts[d]) for d in range(3)]
    n[axis] += 1
    return n


def face_len(g: Grid, axis: int) -> int:
    f = face_counts(g, axis)
    return f[0] * f[1] * f[2]


def cell_len(g: Grid) -> int:
    return int(g.counts[0]) * int(g.counts[1]) * int(g.counts[2])


def _ptr(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.c_void_p)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


# ------------------------------------------------------------------ wrappers
def sample(g, axis, values, position):
    values = _f32(values)
    pos = (C.c_double * 3)(*position)
    out = C.c_double()
    st = lib().orc_sample(C.byref(g), axis, _ptr(values), pos, C.byref(out))
    return st, out.value


def backtrace(g, u, v, w, position, dt):
    u, v, w = _f32(u), _f32(v), _f32(w)
    pos = (C.c_double * 3)(*position)
    out = (C.c_double * 3)()
    st = lib().orc_backtrace(C.byref(g), _ptr(u), _ptr(v), _ptr(w), pos, dt, out)
    return st, [out[0], out[1], out[2]]


def advect_velocity(g, faces, dt, threads=1):
    dtype = faces[0].dtype
    ins = [np.ascontiguousarray(f) for f in faces]
    outs = [np.zeros_like(f) for f in ins]
    fn = lib().orc_advect_velocity_f32 if dtype == np.float32 else lib().orc_advect_velocity_f64
    st = fn(C.byref(g), *[_ptr(a) for a in ins], dt, *[_ptr(a) for a in outs], threads)
    return st, outs


def advect_tracer(g, old, faces, dt, threads=1):
    old = _f32(old)
    faces = [_f32(f) for f in faces]
    out = np.zeros(cell_len(g), np.float32)
    st = lib().orc_advect_tracer_f32(C.byref(g), _ptr(old), *[_ptr(f) for f in faces], dt, _ptr(out), threads)
    return st, out


def apply_full(g, density, p, threads=1):
    p = _f64(p)
    out = np.zeros(cell_len(g), np.float64)
    st = lib().orc_apply_full(C.byref(g), density, _ptr(p), _ptr(out), threads)
    return st, out


def build_rhs(g, density, faces, dt):
    out = np.zeros(cell_len(g), np.float64)
    if faces[0].dtype == np.float32:
        fs = [_f32(f) for f in faces]
        st = lib().orc_build_rhs_f32(C.byref(g), density, *[_ptr(f) for f in fs], dt, _ptr(out))
    else:
        fs = [_f64(f) for f in faces]
        st = lib().orc_build_rhs_f64(C.byref(g), density, *[_ptr(f) for f in fs], dt, _ptr(out))
    return st, out


def divergence(g, faces):
    out = np.zeros(cell_len(g), np.float64)
    if faces[0].dtype == np.float32:
        fs = [_f32(f) for f in faces]
        st = lib().orc_divergence_f32(C.byref(g), *[_ptr(f) for f in fs], _ptr(out))
    else:
        fs = [_f64(f) for f in faces]
        st = lib().orc_divergence_f64(C.byref(g), *[_ptr(f) for f in fs], _ptr(out))
    return st, out


def correct(g, density, p, dt, faces):
    """Returns (status, corrected copies of faces)."""
    p = _f64(p)
    fs = [np.array(f, copy=True, order="C") for f in faces]
    fn = lib().orc_correct_f32 if fs[0].dtype == np.float32 else lib().orc_correct_f64
    st = fn(C.byref(g), density, _ptr(p), dt, *[_ptr(f) for f in fs])
    return st, fs


def diagonal(g, density, coordinate):
    c = (C.c_uint64 * 3)(*coordinate)
    return lib().orc_diagonal(C.byref(g), density, c)


def compensated_sum(values):
    values = _f64(values)
    return lib().orc_compensated_sum(_ptr(values), values.size)


def dot(a, b):
    a, b = _f64(a), _f64(b)
    return lib().orc_dot(_ptr(a), _ptr(b), a.size)


def precondition(g, density, method, r):
    r = np.array(r, dtype=np.float64, copy=True)
    z = np.zeros_like(r)
    rz = C.c_double()
    st = lib().orc_precondition(C.byref(g), density, method, _ptr(r), _ptr(z), C.byref(rz))
    return st, z, rz.value


@dataclass
class SolveResult:
    status: int
    pressure: np.ndarray
    report: Report
    trace: list


def solve_rhs(g, density, method, rhs, dt, s: Settings, trace=False, threads=1, initial=None) -> SolveResult:
    """solve_rhs, or solve_rhs_with_initial_pressure when `initial` is given."""
    rhs = _f64(rhs)
    p = np.zeros(cell_len(g), np.float64)
    rep = Report()
    cap = int(s.max_iterations) if trace else 0
    tr = (Trace * max(cap, 1))()
    init = None if initial is None else _f64(initial)
    if init is not None and init.size != rhs.size:
        return SolveResult(LENGTH_MISMATCH, p, rep, [])
    st = lib().orc_solve_rhs_initial(C.byref(g), density, method, _ptr(rhs), _ptr(init) if init is not None else None,
                                     dt, C.byref(s), _ptr(p), C.byref(rep), C.cast(tr, C.c_void_p) if cap else None,
                                     cap, threads)
    return SolveResult(st, p, rep, [tr[i] for i in range(cap)] if cap else [])


def qualify_pressure(g, density, rhs, dt, s: Settings, pressure):
    rhs, pressure = _f64(rhs), _f64(pressure)
    rep = Report()
    st = lib().orc_qualify_pressure(C.byref(g), density, _ptr(rhs), dt, C.byref(s), _ptr(pressure), C.byref(rep))
    return st, rep


def velocity_rate(g, faces):
    out = C.c_double()
    if faces[0].dtype == np.float32:
        fs = [_f32(f) for f in faces]
        st = lib().orc_velocity_rate_f32(C.byref(g), *[_ptr(f) for f in fs], C.byref(out))
    else:
        fs = [_f64(f) for f in faces]
        st = lib().orc_velocity_rate_f64(C.byref(g), *[_ptr(f) for f in fs], C.byref(out))
    return st, out.value


def carrier_step(g, faces, params: StepParams, tracer=None, initial=None, keep_pressure=False):
    """One carrier step in place on copies; returns (status, faces, tracer,
    StepReport), plus the step's pressure when keep_pressure. `initial` seeds
    the solve (solve_rhs_with_initial_pressure)."""
    fs = [np.array(f, copy=True, order="C") for f in faces]
    tr = None if tracer is None else np.array(tracer, dtype=np.float32, copy=True)
    rep = StepReport()
    init = None if initial is None else _f64(initial)
    pout = np.zeros(cell_len(g), np.float64) if keep_pressure else None
    fn = lib().orc_carrier_step_seeded_f32 if fs[0].dtype == np.float32 else lib().orc_carrier_step_seeded_f64
    st = fn(C.byref(g), C.byref(params), *[_ptr(f) for f in fs], _ptr(tr) if tr is not None else None,
            _ptr(init) if init is not None else None, _ptr(pout) if pout is not None else None, C.byref(rep))
    if keep_pressure:
        return st, fs, tr, rep, pout
    return st, fs, tr, rep


DENSE3D_DIAGNOSTICS = ("pressure_residual_m3_s2", "carrier_divergence_s_inv", "liquid_divergence_s_inv",
                       "volume_before_m3", "volume_after_m3", "mass_after_kg", "inward_m3", "outward_m3",
                       "source_m3", "balance_m3", "rounding_budget_m3")


def dense3d_frame_text(g, frame=0, time_s=0.0, dt_s=0.0, carrier_stamp=(0, 0), liquid_stamp=(0, 0),
                       diagnostics=None, faces=None, tracer=None, fraction=None, pressure=None):
    """write_dense3d_frame (src/dense3d_sequence.rs:412-564) of host arrays:
    (status, bytes). faces: three f32 arrays; tracer f32, fraction and
    pressure f64 (None: zeros). Status 0, or 23 for a failed preflight."""
    f = Dense3dFrame()
    f.frame = frame
    f.time_s = time_s
    f.dt_s = dt_s
    f.carrier_stamp_id, f.carrier_stamp_version = carrier_stamp
    f.liquid_stamp_id, f.liquid_stamp_version = liquid_stamp
    if diagnostics is not None:
        f.has_diagnostics = 1
        f.pressure_iterations = int(diagnostics.get("pressure_iterations", 0))
        for k in DENSE3D_DIAGNOSTICS:
            setattr(f, k, float(diagnostics.get(k, 0.0)))
    fs = [_f32(a) for a in faces]
    tr = _f32(tracer) if tracer is not None else None
    fr = _f64(fraction) if fraction is not None else None
    p = _f64(pressure) if pressure is not None else np.zeros(cell_len(g))
    cap = (sum(a.size for a in fs) + cell_len(g)) * 17 + 2 * cell_len(g) * 26 + 4096
    buf = C.create_string_buffer(cap)
    n = C.c_size_t()
    st = lib().orc_dense3d_frame_text(C.byref(g), C.byref(f), _ptr(fs[0]), _ptr(fs[1]), _ptr(fs[2]),
                                      _ptr(tr) if tr is not None else None, _ptr(fr) if fr is not None else None,
                                      _ptr(p), buf, cap, C.byref(n))
    return st, (buf.raw[:n.value] if st == 0 else b"")


def liquid_validate_state(g, density, fraction):
    """LiquidVolumeState::new validation: (error name, cell)."""
    f = _f64(fraction)
    cell = C.c_uint64()
    code = lib().orc_liquid_validate_state(C.byref(g), density, _ptr(f), C.byref(cell))
    return LIQUID_ERRORS[code], cell.value


def liquid_advance(g, density, fraction, faces, start, dt, inlet, source=None, max_outward_courant=1.0,
                   actual_divergence_limit=1e-9, state_time=None, version=0, periodic=False):
    """LiquidVolumeState::advance with an inlet boundary, or advance_periodic
    (src/liquid_volume.rs:376-406, 520-776): (error name, candidate fraction or
    None, report dict). inlet is ignored when periodic."""
    acc = _f64(fraction)
    cand = np.zeros_like(acc)
    fs = [_f32(a) for a in faces]
    inl = (C.c_double * 6)(*[float(x) for pair in inlet for x in pair])
    src = _f64(source) if source is not None else None
    rep = LiquidReport()
    code = lib().orc_liquid_advance(C.byref(g), density, start if state_time is None else state_time, version,
                                    _ptr(acc), _ptr(cand), _ptr(fs[0]), _ptr(fs[1]), _ptr(fs[2]), start, dt, inl,
                                    _ptr(src) if src is not None else None, max_outward_courant,
                                    actual_divergence_limit, 1 if periodic else 0, C.byref(rep))
    out = {name: getattr(rep, name) for name, _ in LiquidReport._fields_}
    return LIQUID_ERRORS[code], (cand if code == 0 else None), out


def box_flux_project(g, density, method, faces, dt, outward, s: Settings, actual_divergence_limit, out=None):
    """BoxFluxWorkspace::project (src/box_flux.rs:213-397): (status, projected
    faces, pressure, report dict). outward: [[lower, upper]] per axis (f32).
    out: optional initial output arrays (left untouched before the correction)."""
    fs = [_f32(a) for a in faces]
    outs = [np.array(o, dtype=np.float32) for o in out] if out is not None else [np.zeros_like(a) for a in fs]
    p = np.zeros(cell_len(g))
    ow = (C.c_float * 6)(*[float(x) for pair in outward for x in pair])
    rep = BoxFluxReport()
    st = lib().orc_box_flux_project(C.byref(g), density, method, _ptr(fs[0]), _ptr(fs[1]), _ptr(fs[2]), dt, ow,
                                    C.byref(s), actual_divergence_limit, _ptr(outs[0]), _ptr(outs[1]),
                                    _ptr(outs[2]), _ptr(p), C.byref(rep))
    d = {n: getattr(rep, n) for n, _ in BoxFluxReport._fields_ if n not in ("pressure",)}
    d["iterations"] = rep.pressure.iterations
    return st, outs, p, d


class Simulation:
    """The step owner of the oracle (Simulation::step / step_with_forces /
    step_with_box_flux, src/simulation.rs:393-581): f32 faces and tracer,
    updated by step() only when it succeeds."""

    def __init__(self, g, density, method, pressure: Settings, actual_divergence_limit, max_courant, faces=None,
                 tracer=None):
        self.g = g
        self.config = SimConfig(density, method, pressure, actual_divergence_limit, max_courant)
        self.faces = [np.zeros(face_len(g, d), np.float32) if faces is None else np.array(faces[d], np.float32)
                      for d in range(3)]
        self.tracer = np.zeros(cell_len(g), np.float32) if tracer is None else np.array(tracer, np.float32)
        self.time = 0.0
        self.generation = 0

    def step(self, requested_dt, source=None, forces=(), outward=None):
        """(status, report). source: dict(lower, upper, tracer_rate, vertical_acceleration);
        forces: dicts (value, units 0/1, region=(lower, upper) or None); outward: [[lo, hi]] per axis."""
        st_ = SimState(_ptr(self.faces[0]), _ptr(self.faces[1]), _ptr(self.faces[2]), _ptr(self.tracer),
                       self.time, self.generation)
        src = None
        if source is not None:
            src = SmokeSource((C.c_double * 3)(*source["lower"]), (C.c_double * 3)(*source["upper"]),
                              source["tracer_rate"], source["vertical_acceleration"])
        fa = (BodyForce * max(1, len(forces)))()
        for i, f in enumerate(forces):
            fa[i].value = (C.c_double * 3)(*f["value"])
            fa[i].units = int(f.get("units", 0))
            region = f.get("region")
            fa[i].has_region = 1 if region is not None else 0
            if region is not None:
                fa[i].lower = (C.c_double * 3)(*region[0])
                fa[i].upper = (C.c_double * 3)(*region[1])
        ow = None if outward is None else (C.c_float * 6)(*[float(x) for pair in outward for x in pair])
        rep = SimReport()
        st = lib().orc_sim_step(C.byref(self.g), C.byref(self.config), C.byref(st_), requested_dt,
                                C.byref(src) if src is not None else None, fa, len(forces), ow, C.byref(rep))
        if st == 0:
            self.time = st_.time
            self.generation = st_.generation
        return st, rep
