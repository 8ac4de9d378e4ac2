"""rheon_b200: Rheon's fixed-box carrier step on the B200 (sm_100a).

The host-side mirror of Rheon's interfaces for this path, over the C ABI of
include/rheon_b200.h (librheon_b200.so). Names follow the Rust crate:
GridGeometry, PressureOperator, PressureWorkspace, PressureImplementation,
PressureSettings, PressureReport, PressureError, the PressureProvider trait
(B200PressureProvider) and a resident step owner (CarrierSimulation).
Every compute call runs the CUDA library; there is no CPU path.

Device arrays are anything with ``data_ptr()`` (torch CUDA tensors) or raw
integer device pointers. Host arrays are numpy arrays.
"""
from __future__ import annotations

import ctypes as C
import enum
from dataclasses import dataclass, field
from typing import Callable, Optional, Sequence

import numpy as np

from . import _native as N
from ._native import lib

__all__ = [
    "GridGeometry", "PressureImplementation", "PressureSettings", "PressureReport", "PressureError",
    "OperatorError", "ProviderRejection", "PressureOperator", "PressureWorkspace", "PressureRequest",
    "B200PressureProvider", "CarrierSimulation", "CarrierConfig", "StepParams", "StepReport",
    "SimulationError", "advect_velocity", "advect_tracer", "device_count", "status_name", "step_all",
]


def status_name(code: int) -> str:
    return N.STATUS_NAMES.get(code, f"Status{code}")


def device_count() -> int:
    return int(lib().rb200_device_count())


# ------------------------------------------------------------------ geometry
class GridGeometry:
    """GridGeometry::new(counts, spacing, origin) (src/geometry.rs:114)."""

    def __init__(self, counts, spacing=(1.0, 1.0, 1.0), origin=(0.0, 0.0, 0.0)):
        self.counts = tuple(int(c) for c in counts)
        self.spacing = tuple(float(h) for h in spacing)
        self.origin = tuple(float(o) for o in origin)
        if any(c <= 0 for c in self.counts):
            raise ValueError("cell count is zero")
        if any(not (h > 0.0 and np.isfinite(h)) for h in self.spacing):
            raise ValueError("spacing must be finite and positive")

    def c(self) -> N.Grid:
        g = N.Grid()
        for d in range(3):
            g.counts[d] = self.counts[d]
            g.spacing[d] = self.spacing[d]
            g.origin[d] = self.origin[d]
        return g

    def cell_len(self) -> int:
        return self.counts[0] * self.counts[1] * self.counts[2]

    def face_counts(self, axis: int):
        f = list(self.counts)
        f[axis] += 1
        return tuple(f)

    def face_len(self, axis: int) -> int:
        f = self.face_counts(axis)
        return f[0] * f[1] * f[2]

    def cell_volume(self) -> float:
        return self.spacing[0] * self.spacing[1] * self.spacing[2]

    def upper(self):
        return tuple(self.origin[d] + self.counts[d] * self.spacing[d] for d in range(3))

    def __eq__(self, other):
        return isinstance(other, GridGeometry) and (self.counts, self.spacing, self.origin) == (
            other.counts, other.spacing, other.origin)

    def __repr__(self):
        return f"GridGeometry({self.counts}, {self.spacing}, {self.origin})"


# ------------------------------------------------------------------ pressure types
class PressureImplementation(enum.IntEnum):
    """PressureImplementation (src/pressure.rs:7-29) plus the device-native methods."""

    JACOBI_PCG_V1 = 0
    SGS_PCG_V1 = 1
    RBSGS_PCG = 2
    MG_MIXED = 3

    def id(self) -> str:
        return {0: "jacobi-pcg-v1", 1: "sgs-pcg-v1", 2: "rbsgs-pcg-b200", 3: "mg-mixed-b200"}[int(self)]

    @classmethod
    def from_id(cls, ident: str):
        for m in cls:
            if m.id() == ident:
                return m
        return None


@dataclass
class PressureSettings:
    """PressureSettings (src/pressure.rs:34-39)."""

    relative_residual: float
    absolute_residual: float
    divergence_limit: float
    max_iterations: int

    def c(self) -> N.Settings:
        return N.Settings(self.relative_residual, self.absolute_residual, self.divergence_limit,
                          int(self.max_iterations))


@dataclass
class PressureReport:
    """PressureReport (src/pressure.rs:44-49)."""

    iterations: int
    true_residual_l2: float
    true_residual_max: float
    predicted_divergence_max: float

    @staticmethod
    def from_c(r: N.Report) -> "PressureReport":
        return PressureReport(int(r.iterations), r.true_residual_l2, r.true_residual_max,
                              r.predicted_divergence_max)


class PressureError(Exception):
    """PressureError (src/pressure.rs:52-77): kind is the variant name."""

    def __init__(self, status: int, report: Optional[N.Report] = None, detail: str = ""):
        self.status = status
        self.kind = status_name(status)
        self.report = PressureReport.from_c(report) if report is not None else None
        self.iterations = int(report.iterations) if report is not None else 0
        self.residual_max = report.true_residual_max if report is not None else None
        self.sum = report.incompatible_sum if report is not None else None
        self.rounding_budget = report.incompatible_budget if report is not None else None
        self.breakdown_iteration = int(report.breakdown_iteration) if report is not None else None
        super().__init__(f"{self.kind}" + (f": {detail}" if detail else ""))


class OperatorError(Exception):
    """OperatorError (src/operator.rs:7-17): kind is the variant name."""

    def __init__(self, status: int):
        self.status = status
        self.kind = status_name(status)
        super().__init__(self.kind)


class ProviderRejection(Exception):
    """ProviderRejection (src/solver_provider.rs:55-62)."""

    def __init__(self, status: int, detail: str = ""):
        self.status = status
        self.kind = status_name(status)
        super().__init__(self.kind + (f": {detail}" if detail else ""))


class SimulationError(Exception):
    def __init__(self, status: int, report=None, detail: str = ""):
        self.status = status
        self.kind = status_name(status)
        self.report = report
        super().__init__(self.kind + (f": {detail}" if detail else ""))


def _cancel_cb(cancelled: Optional[Callable[[], bool]]):
    if cancelled is None:
        return N.NO_CANCEL
    return N.CANCEL_FN(lambda _ctx: 1 if cancelled() else 0)


def _ptr(x) -> int:
    if x is None:
        return 0
    if isinstance(x, int):
        return x
    return int(x.data_ptr())


def _stream_of(*tensors) -> int:
    for t in tensors:
        if t is not None and hasattr(t, "device"):
            import torch

            return int(torch.cuda.current_stream(t.device).cuda_stream)
    return 0


def _f64_host(a, n: int) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float64)
    if a.size != n:
        raise OperatorError(N.LENGTH_MISMATCH)
    return a


# ------------------------------------------------------------------ operator primitives
class PressureOperator:
    """Sealed-box PressureOperator (src/operator.rs:46-97) on device arrays."""

    def __init__(self, grid: GridGeometry, density: float):
        if not (np.isfinite(density) and density > 0.0):
            raise OperatorError(N.INVALID_ARGUMENT)
        self.grid = grid
        self.density = float(density)
        h = grid.spacing
        self.face_area = (h[1] * h[2], h[0] * h[2], h[0] * h[1])
        self.acceleration_factor = tuple(1.0 / (self.density * h[d]) for d in range(3))

    def _check(self, st):
        if st != N.OK:
            raise OperatorError(st)

    def apply_full(self, pressure, out):
        self._check(lib().rb200_apply_full_device(C.byref(self.grid.c()), self.density, _ptr(pressure), _ptr(out),
                                                  _stream_of(pressure)))

    def qualify_pressure(self, rhs, pressure, dt: float, settings: "PressureSettings") -> "PressureReport":
        """ProviderWorkspace's qualification of a candidate pressure
        (src/solver_provider.rs:239-270) on device arrays; raises
        ProviderRejection (NonFiniteOutput, NonZeroGauge, QualityGate) with the
        candidate's report attached."""
        rep = N.Report()
        n = int(pressure.numel()) if hasattr(pressure, "numel") else int(pressure.size)
        st = lib().rb200_qualify_pressure_device(C.byref(self.grid.c()), self.density, _ptr(rhs), _ptr(pressure), n,
                                                 dt, C.byref(settings.c()), C.byref(rep), _stream_of(pressure))
        report = PressureReport.from_c(rep)
        if st != N.OK:
            err = ProviderRejection(st)
            err.report = report
            raise err
        return report

    def projection_witness(self, pressure, dt: float, velocity: Sequence, supplied: Sequence):
        """The momentum witness of a supplied projection
        (composition/projection.rs:515-542): None when `supplied` equals
        `velocity` corrected with `pressure` bit for bit, else (axis, index)
        of the first mismatching face."""
        u, v, w = velocity
        su, sv, sw = supplied
        fn = lib().rb200_projection_witness_f32_device if _is_f32(u) else lib().rb200_projection_witness_f64_device
        axis, index = C.c_int(), C.c_uint64()
        st = fn(C.byref(self.grid.c()), self.density, _ptr(pressure), dt, _ptr(u), _ptr(v), _ptr(w), _ptr(su),
                _ptr(sv), _ptr(sw), C.byref(axis), C.byref(index), _stream_of(u))
        if st == N.QUALITY_GATE:
            return int(axis.value), int(index.value)
        self._check(st)
        return None

    def precondition_jacobi(self, residual, out) -> float:
        """precondition_jacobi (src/pressure.rs:534-575): out = r/D with
        out[0] = 0 (eliminated gauge row); returns r.z over rows >= 1."""
        rz = C.c_double()
        n = int(residual.numel()) if hasattr(residual, "numel") else int(residual.size)
        self._check(lib().rb200_precondition_jacobi_device(C.byref(self.grid.c()), self.density, _ptr(residual),
                                                           _ptr(out), n, C.byref(rz), _stream_of(residual)))
        return rz.value

    def build_rhs(self, velocity: Sequence, dt: float, out):
        u, v, w = velocity
        fn = lib().rb200_build_rhs_f32_device if _is_f32(u) else lib().rb200_build_rhs_f64_device
        self._check(fn(C.byref(self.grid.c()), self.density, _ptr(u), _ptr(v), _ptr(w), dt, _ptr(out),
                       _stream_of(u)))

    def divergence(self, velocity: Sequence, out):
        u, v, w = velocity
        fn = lib().rb200_divergence_f32_device if _is_f32(u) else lib().rb200_divergence_f64_device
        self._check(fn(C.byref(self.grid.c()), _ptr(u), _ptr(v), _ptr(w), _ptr(out), _stream_of(u)))

    def correct_candidate_in_place(self, pressure, dt: float, candidate: Sequence):
        u, v, w = candidate
        fn = lib().rb200_correct_f32_device if _is_f32(u) else lib().rb200_correct_f64_device
        self._check(fn(C.byref(self.grid.c()), self.density, _ptr(pressure), dt, _ptr(u), _ptr(v), _ptr(w),
                       _stream_of(u)))


def _is_f32(t) -> bool:
    return str(getattr(t, "dtype", "")).endswith("float32")


def advect_velocity(grid: GridGeometry, old: Sequence, dt: float, output: Sequence):
    """advect_velocity (src/advection.rs:28-68) on device face arrays."""
    u, v, w = old
    ou, ov, ow = output
    fn = lib().rb200_advect_velocity_f32_device if _is_f32(u) else lib().rb200_advect_velocity_f64_device
    st = fn(C.byref(grid.c()), _ptr(u), _ptr(v), _ptr(w), dt, _ptr(ou), _ptr(ov), _ptr(ow), _stream_of(u))
    if st != N.OK:
        raise OperatorError(st)


def advect_tracer(grid: GridGeometry, old, velocity: Sequence, dt: float, output):
    """advect_tracer (src/advection.rs:72-102) on device arrays (f32 faces)."""
    u, v, w = velocity
    st = lib().rb200_advect_tracer_f32_device(C.byref(grid.c()), _ptr(old), _ptr(u), _ptr(v), _ptr(w), dt,
                                              _ptr(output), _stream_of(old))
    if st != N.OK:
        raise OperatorError(st)


# ------------------------------------------------------------------ workspace
class PressureWorkspace:
    """PressureWorkspace (src/pressure.rs:247-741) with device-resident buffers.

    ``solve_rhs`` raises PressureError like the Rust Result; after an
    IterationLimit the iterate remains readable through ``pressure()``.
    """

    def __init__(self, grid: GridGeometry, limit: int, implementation=PressureImplementation.JACOBI_PCG_V1,
                 density: float = 1.0, device: int = 0):
        self.grid = grid
        self.limit = int(limit)
        self.implementation = PressureImplementation(implementation)
        self.device = device
        self._handle = None
        self._density = None
        self._trace = None
        self._create(density)

    @classmethod
    def with_implementation(cls, grid, limit, implementation, density=1.0, device=0):
        return cls(grid, limit, implementation, density, device)

    def _create(self, density: float):
        self.close()
        h = C.c_void_p()
        st = lib().rb200_workspace_create(C.byref(self.grid.c()), float(density), int(self.implementation),
                                          self.limit, self.device, C.byref(h))
        if st != N.OK:
            raise PressureError(st)
        self._handle = h
        self._density = float(density)
        if self._trace is not None:
            self.set_trace(len(self._trace))

    def close(self):
        if self._handle is not None:
            lib().rb200_workspace_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def allocated_bytes(self) -> int:
        return int(lib().rb200_workspace_allocated_bytes(self._handle))

    def stream(self) -> int:
        return int(lib().rb200_workspace_stream(self._handle) or 0)

    def set_trace(self, capacity: int):
        """Record per-iteration PCG scalars of the following solves."""
        self._trace = (N.Trace * max(int(capacity), 1))()
        st = lib().rb200_workspace_set_trace(self._handle, C.cast(self._trace, C.c_void_p), int(capacity))
        if st != N.OK:
            raise PressureError(st)

    def trace(self, count: int):
        return [self._trace[i] for i in range(min(count, len(self._trace)))]

    def solve_rhs(self, operator: PressureOperator, rhs, dt: float, settings: PressureSettings,
                  cancelled: Optional[Callable[[], bool]] = None, initial=None) -> PressureReport:
        """solve_rhs (src/pressure.rs:365-393); with `initial`,
        solve_rhs_with_initial_pressure (:415-430): PCG seeded by the given
        pressure (finite, initial[0] == 0)."""
        if operator.density != self._density:
            self._create(operator.density)
        rep = N.Report()
        cb = _cancel_cb(cancelled)
        if initial is not None:
            keep = []

            def ptr(a):
                if hasattr(a, "data_ptr"):
                    if hasattr(a, "device"):
                        import torch

                        torch.cuda.current_stream(a.device).synchronize()
                    return _ptr(a), int(a.numel())
                h = np.ascontiguousarray(a, dtype=np.float64)
                keep.append(h)
                return h.ctypes.data_as(C.c_void_p), h.size

            (rp, n), (ip, ni) = ptr(rhs), ptr(initial)
            if ni != n:
                raise PressureError(N.LENGTH_MISMATCH)
            st = lib().rb200_workspace_solve_rhs_initial(self._handle, rp, ip, n, dt, C.byref(settings.c()),
                                                         C.byref(rep), cb, None)
            self.last_report = PressureReport.from_c(rep)
            if st != N.OK:
                raise PressureError(st, rep)
            return self.last_report
        if hasattr(rhs, "data_ptr"):
            # The workspace runs on its own stream: the producer of rhs must be done.
            if hasattr(rhs, "device"):
                import torch

                torch.cuda.current_stream(rhs.device).synchronize()
            st = lib().rb200_workspace_solve_rhs_device(self._handle, _ptr(rhs), int(rhs.numel()), dt,
                                                        C.byref(settings.c()), C.byref(rep), cb, None)
        else:
            a = np.ascontiguousarray(rhs, dtype=np.float64)
            st = lib().rb200_workspace_solve_rhs(self._handle, a.ctypes.data_as(C.c_void_p), a.size, dt,
                                                 C.byref(settings.c()), C.byref(rep), cb, None)
        self.last_report = PressureReport.from_c(rep)
        if st != N.OK:
            raise PressureError(st, rep)
        return self.last_report

    def pressure(self) -> np.ndarray:
        out = np.empty(self.grid.cell_len(), np.float64)
        st = lib().rb200_workspace_pressure(self._handle, out.ctypes.data_as(C.c_void_p), out.size)
        if st != N.OK:
            raise PressureError(st)
        return out

    def profile(self, which: int, launches: int = 20) -> float:
        ms = C.c_double()
        st = lib().rb200_workspace_profile(self._handle, which, launches, C.byref(ms))
        if st != N.OK:
            raise PressureError(st)
        return ms.value

    def pressure_device_ptr(self) -> int:
        return int(lib().rb200_workspace_pressure_device(self._handle) or 0)


# ------------------------------------------------------------------ provider
@dataclass
class PressureRequest:
    """PressureRequest (src/solver_provider.rs:47-52)."""

    grid: GridGeometry
    density: float
    dt: float
    rhs: np.ndarray

    def c(self) -> N.Request:
        self._rhs = np.ascontiguousarray(self.rhs, dtype=np.float64)
        return N.Request(self.grid.c(), self.density, self.dt, self._rhs.ctypes.data_as(C.c_void_p), self._rhs.size)


@dataclass
class SolverMetadata:
    id: str
    version: str
    stage: str
    input: dict = field(default_factory=dict)
    output: dict = field(default_factory=dict)
    domain: str = ""


class B200PressureProvider:
    """A PressureProvider (src/solver_provider.rs:67-76) backed by the B200.

    metadata() / supports() / predict() are the trait's three methods; predict
    writes every cell with pressure[0] == 0 and raises ProviderRejection on
    failure. Rheon's ProviderWorkspace re-qualifies the output on the host.
    """

    def __init__(self, grid: GridGeometry, density: float, settings: PressureSettings,
                 implementation=PressureImplementation.JACOBI_PCG_V1, device: int = 0):
        cfg = N.ProviderConfig(grid.c(), float(density), int(implementation), settings.c(), device)
        h = C.c_void_p()
        st = lib().rb200_provider_create(C.byref(cfg), C.byref(h))
        if st != N.OK:
            raise ProviderRejection(st, "provider construction")
        self._handle = h
        self.grid = grid

    def close(self):
        if getattr(self, "_handle", None) is not None:
            lib().rb200_provider_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def metadata(self) -> SolverMetadata:
        m = N.Metadata()
        lib().rb200_provider_metadata(self._handle, C.byref(m))
        shape = [int(m.shape_xyz[d]) for d in range(3)]
        return SolverMetadata(
            m.id.decode(), m.version.decode(), m.stage.decode(),
            {"shape_xyz": shape, "layout": m.input_layout.decode(), "scalar": m.input_scalar.decode(),
             "units": m.input_units.decode()},
            {"shape_xyz": shape, "layout": m.output_layout.decode(), "scalar": m.output_scalar.decode(),
             "units": m.output_units.decode()},
            m.domain.decode())

    def supports(self, request: PressureRequest) -> None:
        st = lib().rb200_provider_supports(self._handle, C.byref(request.c()))
        if st != N.OK:
            raise ProviderRejection(st)

    def predict(self, request: PressureRequest, pressure: np.ndarray,
                cancelled: Optional[Callable[[], bool]] = None) -> None:
        if pressure.dtype != np.float64 or not pressure.flags["C_CONTIGUOUS"]:
            raise ProviderRejection(N.UNSUPPORTED, "pressure must be contiguous f64")
        req = request.c()
        st = lib().rb200_provider_predict(self._handle, C.byref(req), pressure.ctypes.data_as(C.c_void_p),
                                          pressure.size, _cancel_cb(cancelled), None)
        if st != N.OK:
            raise ProviderRejection(st, (lib().rb200_provider_last_error(self._handle) or b"").decode())

    def last_report(self):
        r = N.Report()
        s = C.c_int()
        lib().rb200_provider_last_report(self._handle, C.byref(r), C.byref(s))
        return s.value, PressureReport.from_c(r)


# ------------------------------------------------------------------ resident step owner
@dataclass
class CarrierConfig:
    """SimulationConfig (src/simulation.rs:11-18) for the resident device step."""

    density: float = 1.0
    pressure: PressureSettings = field(default_factory=lambda: PressureSettings(1e-8, 0.0, 1.7976931348623157e308,
                                                                                100000))
    actual_divergence_limit: float = 1.7976931348623157e308
    max_courant: float = 1.0
    storage: str = "f64"
    implementation: PressureImplementation = PressureImplementation.JACOBI_PCG_V1
    with_tracer: bool = False
    device: int = 0
    fp32_advection: bool = False
    # PressureInitializationPolicy (src/pressure_initialization.rs:7-12):
    # False = Cold, True = AcceptedPreviousV1 (seed each solve with the last
    # accepted step's pressure).
    warm_start: bool = False

    @staticmethod
    def mixed(**kw) -> "CarrierConfig":
        """The mixed-precision carrier: FP32 faces and FP32 advection
        arithmetic, FP32 multigrid V(2,2) smoothing inside FP64 flexible CG
        (FP64 residual, pressure accumulation and coarsest solve)."""
        kw.setdefault("storage", "f32")
        kw.setdefault("implementation", PressureImplementation.MG_MIXED)
        kw.setdefault("fp32_advection", True)
        return CarrierConfig(**kw)


@dataclass
class StepParams:
    requested_dt: float
    cfl: float = 0.0
    buoyancy: float = 0.0
    iteration_limit_ok: bool = False
    skip_gates: bool = False


@dataclass
class StepReport:
    """StepReport (src/simulation.rs:44-53) subset."""

    dt: float
    time: float
    generation: int
    pressure: PressureReport
    pressure_status: int
    actual_divergence_max: float
    courant: float
    velocity_rate: float
    pressure_ms: float = 0.0
    kernel_launches: int = 0
    pressure_initialization: int = 0   # the policy actually used: 0 cold, 1 accepted previous


class CarrierSimulation:
    """Device-resident fixed-box carrier state and its transactional step."""

    def __init__(self, grid: GridGeometry, config: CarrierConfig):
        self.grid = grid
        self.config = config
        self.dtype = np.float32 if config.storage == "f32" else np.float64
        c = N.CarrierConfig(grid.c(), config.density, 0 if config.storage == "f32" else 1,
                            int(config.implementation), config.pressure.c(), config.actual_divergence_limit,
                            config.max_courant, 1 if config.with_tracer else 0, config.device,
                            1 if config.fp32_advection else 0, 1 if config.warm_start else 0)
        h = C.c_void_p()
        st = lib().rb200_carrier_create(C.byref(c), C.byref(h))
        if st != N.OK:
            raise SimulationError(st, detail="carrier construction")
        self._handle = h

    def close(self):
        if getattr(self, "_handle", None) is not None:
            lib().rb200_carrier_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def allocated_bytes(self) -> int:
        return int(lib().rb200_carrier_allocated_bytes(self._handle))

    def stream(self) -> int:
        return int(lib().rb200_carrier_stream(self._handle) or 0)

    def upload(self, faces: Sequence[np.ndarray], tracer: Optional[np.ndarray] = None):
        fs = [np.ascontiguousarray(f, dtype=self.dtype) for f in faces]
        for d in range(3):
            if fs[d].size != self.grid.face_len(d):
                raise SimulationError(N.LENGTH_MISMATCH)
        tr = None if tracer is None else np.ascontiguousarray(tracer, dtype=np.float32)
        st = lib().rb200_carrier_upload(self._handle, *[f.ctypes.data_as(C.c_void_p) for f in fs],
                                        tr.ctypes.data_as(C.c_void_p) if tr is not None else None)
        if st != N.OK:
            raise SimulationError(st)

    def init_fourier(self, seed: int, modes: int = 8, kmax: int = 8, amplitude: float = 1.0, noise: float = 0.05):
        """Random-Fourier accepted state generated on the device (the same
        modes and noise stream as workloads.fourier_faces)."""
        from . import workloads as W

        k, phase, amp = W.fourier_modes(seed, modes, kmax)
        k = np.ascontiguousarray(k, dtype=np.float64)
        phase = np.ascontiguousarray(phase, dtype=np.float64)
        amp = np.ascontiguousarray(amp, dtype=np.float64)
        st = lib().rb200_carrier_init_fourier(self._handle, seed & 0xFFFFFFFFFFFFFFFF, modes,
                                              k.ctypes.data_as(C.c_void_p), phase.ctypes.data_as(C.c_void_p),
                                              amp.ctypes.data_as(C.c_void_p), amplitude, noise)
        if st != N.OK:
            raise SimulationError(st)

    def upload_ptrs(self, u: int, v: int, w: int, tracer: int = 0):
        """Upload from host pointers (e.g. pinned buffers)."""
        st = lib().rb200_carrier_upload(self._handle, u, v, w, tracer or None)
        if st != N.OK:
            raise SimulationError(st)

    def download(self, with_tracer: bool = False):
        fs = [np.empty(self.grid.face_len(d), self.dtype) for d in range(3)]
        tr = np.empty(self.grid.cell_len(), np.float32) if with_tracer else None
        st = lib().rb200_carrier_download(self._handle, *[f.ctypes.data_as(C.c_void_p) for f in fs],
                                          tr.ctypes.data_as(C.c_void_p) if tr is not None else None)
        if st != N.OK:
            raise SimulationError(st)
        return (fs, tr) if with_tracer else fs

    def download_ptrs(self, u: int, v: int, w: int, tracer: int = 0):
        st = lib().rb200_carrier_download(self._handle, u, v, w, tracer or None)
        if st != N.OK:
            raise SimulationError(st)

    def state_device_ptrs(self):
        p = [C.c_void_p() for _ in range(4)]
        lib().rb200_carrier_state_device(self._handle, *[C.byref(x) for x in p])
        return [x.value or 0 for x in p]

    def profile(self, which: int, launches: int = 20) -> float:
        """Average device ms of one PCG pass (0: direction+apply, 1: update),
        or of one iteration of the persistent Jacobi-PCG kernel (2)."""
        ms = C.c_double()
        st = lib().rb200_carrier_profile(self._handle, which, launches, C.byref(ms))
        if st != N.OK:
            raise SimulationError(st)
        return ms.value

    def pressure(self) -> np.ndarray:
        out = np.empty(self.grid.cell_len(), np.float64)
        st = lib().rb200_carrier_pressure(self._handle, out.ctypes.data_as(C.c_void_p), out.size)
        if st != N.OK:
            raise SimulationError(st)
        return out

    @staticmethod
    def _params(params: StepParams) -> N.StepParams:
        return N.StepParams(params.requested_dt, params.cfl, params.buoyancy, int(params.iteration_limit_ok),
                            int(params.skip_gates))

    @staticmethod
    def _report(r: N.StepReport) -> StepReport:
        return StepReport(r.dt, r.time, int(r.generation), PressureReport.from_c(r.pressure), r.pressure_status,
                          r.actual_divergence_max, r.courant, r.velocity_rate, r.pressure_ms,
                          int(r.kernel_launches), int(r.pressure_initialization))

    def step(self, params: StepParams, cancelled: Optional[Callable[[], bool]] = None) -> StepReport:
        """One step (one CUDA graph); raises SimulationError if it is rejected."""
        r = N.StepReport()
        st = lib().rb200_carrier_step(self._handle, C.byref(self._params(params)), C.byref(r),
                                      _cancel_cb(cancelled), None)
        rep = self._report(r)
        if st != N.OK:
            raise SimulationError(st, rep)
        return rep

    def step_async(self, params: StepParams) -> None:
        """Launch one step without waiting; pair with step_wait()."""
        st = lib().rb200_carrier_step_async(self._handle, C.byref(self._params(params)))
        if st != N.OK:
            raise SimulationError(st)

    def project(self, dt: float) -> StepReport:
        """ProjectionStepWorkspace::project (src/projection_step.rs:863-1033)
        of the accepted state: the uploaded faces are projected with `dt`
        (no advection, no Courant gate) and become the accepted state."""
        r = N.StepReport()
        st = lib().rb200_carrier_project(self._handle, C.byref(self._params(StepParams(dt))), C.byref(r))
        rep = self._report(r)
        if st != N.OK:
            raise SimulationError(st, rep)
        return rep

    def project_async(self, dt: float) -> None:
        """Launch a projection without waiting; pair with step_wait()."""
        st = lib().rb200_carrier_project_async(self._handle, C.byref(self._params(StepParams(dt))))
        if st != N.OK:
            raise SimulationError(st)

    def step_done(self) -> bool:
        """Nonblocking: has the step launched by step_async finished?"""
        return bool(lib().rb200_carrier_step_poll(self._handle))

    def step_wait(self) -> StepReport:
        r = N.StepReport()
        st = lib().rb200_carrier_step_wait(self._handle, C.byref(r))
        rep = self._report(r)
        if st != N.OK:
            raise SimulationError(st, rep)
        return rep


def step_all(sims: Sequence["CarrierSimulation"], params: Sequence[StepParams]):
    """Batched instances: one step of every carrier, launched together so that
    they overlap on the device; returns [(status, StepReport)]."""
    n = len(sims)
    handles = (C.c_void_p * n)(*[s._handle.value for s in sims])
    prm = (N.StepParams * n)(*[CarrierSimulation._params(p) for p in params])
    reps = (N.StepReport * n)()
    sts = (C.c_int * n)()
    lib().rb200_carriers_step(handles, n, prm, reps, sts)
    return [(int(sts[i]), CarrierSimulation._report(reps[i])) for i in range(n)]


class BatchedCarriers:
    """Many independent fixed boxes of uneven sizes stepped together: every
    stage of the step is one launch over all instances and one step of the
    batch is one CUDA graph (mixed precision: f32 faces, FP32 multigrid inside
    FP64 flexible CG). Each instance's results are the same bits as in a batch
    of its own."""

    def __init__(self, grids: Sequence[GridGeometry], config: Optional[CarrierConfig] = None):
        config = config or CarrierConfig.mixed()
        if config.storage != "f32" or config.implementation != PressureImplementation.MG_MIXED:
            raise SimulationError(N.UNSUPPORTED, detail="batched carriers use the mixed method (f32 faces)")
        if config.with_tracer or config.warm_start:
            raise SimulationError(N.UNSUPPORTED, detail="batched carriers carry no tracer and no warm start")
        self.grids = list(grids)
        self.config = config
        arr = (N.Grid * len(self.grids))(*[g.c() for g in self.grids])
        c = N.BatchConfig(config.density, config.pressure.c(), config.actual_divergence_limit, config.max_courant,
                          config.device, 1 if config.fp32_advection else 0)
        h = C.c_void_p()
        st = lib().rb200_batch_create(arr, len(self.grids), C.byref(c), C.byref(h))
        if st != N.OK:
            raise SimulationError(st, detail="batch construction")
        self._handle = h

    def __len__(self):
        return len(self.grids)

    def close(self):
        if getattr(self, "_handle", None) is not None:
            lib().rb200_batch_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def allocated_bytes(self) -> int:
        return int(lib().rb200_batch_allocated_bytes(self._handle))

    def stream(self) -> int:
        return int(lib().rb200_batch_stream(self._handle) or 0)

    def upload(self, index: int, faces: Sequence[np.ndarray]):
        fs = [np.ascontiguousarray(f, dtype=np.float32) for f in faces]
        for d in range(3):
            if fs[d].size != self.grids[index].face_len(d):
                raise SimulationError(N.LENGTH_MISMATCH)
        st = lib().rb200_batch_upload(self._handle, index, *[f.ctypes.data_as(C.c_void_p) for f in fs])
        if st != N.OK:
            raise SimulationError(st)

    def upload_ptrs(self, index: int, u: int, v: int, w: int):
        """Upload from host or device pointers (e.g. pinned buffers)."""
        st = lib().rb200_batch_upload(self._handle, index, u, v, w)
        if st != N.OK:
            raise SimulationError(st)

    def download(self, index: int):
        fs = [np.empty(self.grids[index].face_len(d), np.float32) for d in range(3)]
        st = lib().rb200_batch_download(self._handle, index, *[f.ctypes.data_as(C.c_void_p) for f in fs])
        if st != N.OK:
            raise SimulationError(st)
        return fs

    def download_ptrs(self, index: int, u: int, v: int, w: int):
        st = lib().rb200_batch_download(self._handle, index, u, v, w)
        if st != N.OK:
            raise SimulationError(st)

    def pressure(self, index: int) -> np.ndarray:
        out = np.empty(self.grids[index].cell_len(), np.float64)
        st = lib().rb200_batch_pressure(self._handle, index, out.ctypes.data_as(C.c_void_p), out.size)
        if st != N.OK:
            raise SimulationError(st)
        return out

    def _params(self, params):
        if isinstance(params, StepParams):
            params = [params] * len(self.grids)
        return (N.StepParams * len(self.grids))(*[CarrierSimulation._params(p) for p in params])

    def step(self, params) -> list:
        """One step of every instance (one CUDA graph); returns
        [(status, StepReport)] per instance. `params` is one StepParams for
        all instances or one per instance."""
        self.step_async(params)
        return self.step_wait()

    def step_async(self, params) -> None:
        st = lib().rb200_batch_step_async(self._handle, self._params(params))
        if st != N.OK:
            raise SimulationError(st, detail=(lib().rb200_batch_last_error(self._handle) or b"").decode())

    def step_done(self) -> bool:
        return bool(lib().rb200_batch_step_poll(self._handle))

    def profile_step(self, params) -> dict:
        """A profiling aid: one step issued eagerly with an event after every
        launch (the state advances as in step()); returns {"statuses",
        "reports", "kernels": {name: (ms, launches)}}."""
        n = len(self.grids)
        kinds = int(lib().rb200_batch_profile_kinds())
        reps = (N.StepReport * n)()
        sts = (C.c_int * n)()
        ms = (C.c_double * kinds)()
        cnt = (C.c_int * kinds)()
        names = (C.c_char_p * kinds)()
        st = lib().rb200_batch_profile_step(self._handle, self._params(params), reps, sts, ms, cnt, names, kinds)
        if st != N.OK:
            raise SimulationError(st, detail=(lib().rb200_batch_last_error(self._handle) or b"").decode())
        return {"statuses": [int(x) for x in sts],
                "reports": [CarrierSimulation._report(reps[i]) for i in range(n)],
                "kernels": {names[k].decode(): (ms[k], int(cnt[k])) for k in range(kinds) if cnt[k]}}

    def step_wait(self) -> list:
        n = len(self.grids)
        reps = (N.StepReport * n)()
        sts = (C.c_int * n)()
        st = lib().rb200_batch_step_wait(self._handle, reps, sts)
        if st != N.OK:
            raise SimulationError(st)
        return [(int(sts[i]), CarrierSimulation._report(reps[i])) for i in range(n)]
