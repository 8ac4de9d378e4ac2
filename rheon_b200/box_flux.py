"""Prescribed box flux on the device (src/box_flux.rs).

BoxFluxWorkspace mirrors the reference's type of the same name: it owns a
pressure workspace for one grid and density, and project() imposes uniform
outward speeds on the six sides of the fixed box on a provisional f32 face
field, rejects a boundary whose net flux exceeds its rounding budget, solves
the sealed pressure system for the imposed field on the device, corrects the
interior faces into the caller's output, gates the stored field's divergence
and reports the interior energy ledger. Face arrays are either all CUDA
tensors (the device path) or all numpy arrays (copied through the library).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from typing import Callable, Optional, Sequence

import numpy as np

from . import _native as N
from ._native import lib

__all__ = ["BoxFluxError", "BoxFluxStamp", "PrescribedBoxFlux", "BoxFluxSettings", "BoxFluxStage", "BoxFluxWork",
           "BoxFluxReport", "BoxFluxWorkspace"]


class BoxFluxStage:
    """BoxFluxStage (src/box_flux.rs:53-59)."""
    BEFORE_SOLVE = "BeforeSolve"
    PRESSURE_ITERATION = "PressureIteration"
    CORRECTION_SLICE = "CorrectionSlice"
    BEFORE_ACCEPTANCE = "BeforeAcceptance"


class BoxFluxError(RuntimeError):
    """BoxFluxError (src/box_flux.rs:60-72). kind is the variant: "Operator"
    and "Pressure" wrap the inner error named by `inner`; the others are the
    box-flux variants with their payloads (stage, net/rounding_budget,
    actual/limit, required/limit)."""

    def __init__(self, kind: str, inner: Optional[str] = None, status: int = 0, **payload):
        self.kind = kind
        self.inner = inner
        self.status = status
        self.stage = payload.get("stage")
        self.net = payload.get("net")
        self.rounding_budget = payload.get("rounding_budget")
        self.actual = payload.get("actual")
        self.limit = payload.get("limit")
        self.required = payload.get("required")
        self.iterations = payload.get("iterations")
        super().__init__(f"box flux projection rejected operation: {kind}" + (f"({inner})" if inner else "")
                         + (f" {payload}" if payload else ""))


_PRESSURE = {N.CANCELLED: "Cancelled", N.ITERATION_LIMIT: "IterationLimit", N.BREAKDOWN: "Breakdown",
             N.OUT_OF_MEMORY: "BufferLimit", N.INCOMPATIBLE_RHS: "IncompatibleRhs"}
_OPERATOR = {N.NONFINITE_INPUT: "NonFiniteInput", N.LENGTH_MISMATCH: "LengthMismatch",
             N.ARITHMETIC_FAILURE: "ArithmeticFailure"}


def _error(status: int, r: N.BoxFluxReport, invalid_argument: str = "InvalidTimeStep") -> BoxFluxError:
    if status == N.BOX_FLUX_REJECTED:
        kind = N.BOX_FLUX_ERRORS.get(r.error, f"Error{r.error}")
        payload = {}
        if kind == "Cancelled":
            payload["stage"] = N.BOX_FLUX_STAGES[r.stage]
        elif kind == "IncompatibleFlux":
            payload.update(net=r.error_actual, rounding_budget=r.error_limit)
        elif kind == "DivergenceLimit":
            payload.update(actual=r.error_actual, limit=r.error_limit)
        elif kind == "BufferLimit":
            payload.update(required=int(r.required), limit=int(r.limit))
        return BoxFluxError(kind, status=status, **payload)
    if status in _PRESSURE:
        return BoxFluxError("Pressure", _PRESSURE[status], status, iterations=int(r.pressure.iterations))
    if status in _OPERATOR:
        return BoxFluxError("Operator", _OPERATOR[status], status)
    if status == N.INVALID_ARGUMENT:
        if invalid_argument == "InvalidSettings":
            return BoxFluxError("Pressure", "InvalidSettings", status)
        return BoxFluxError("Operator", invalid_argument, status)
    return BoxFluxError(N.STATUS_NAMES.get(status, f"Status{status}"), status=status)


@dataclass(frozen=True)
class BoxFluxStamp:
    id: int
    version: int


class PrescribedBoxFlux:
    """PrescribedBoxFlux (src/box_flux.rs:15-46): outward[d] = (lower, upper)
    outward-normal speed of axis d's sides in m/s, stored as f32."""

    def __init__(self, stamp: BoxFluxStamp, outward: Sequence[Sequence[float]]):
        speeds = np.asarray(outward, dtype=np.float32).reshape(3, 2)
        if not np.all(np.isfinite(speeds)):
            raise BoxFluxError("InvalidBoundary")
        self._stamp = stamp
        self._outward = speeds

    def stamp(self) -> BoxFluxStamp:
        return self._stamp

    def outward_speeds(self):
        return [(float(a), float(b)) for a, b in self._outward]

    def c(self) -> N.BoxFluxBoundary:
        b = N.BoxFluxBoundary()
        b.id, b.version = int(self._stamp.id), int(self._stamp.version)
        for i, x in enumerate(self._outward.reshape(6)):
            b.outward[i] = float(x)
        return b


@dataclass
class BoxFluxSettings:
    """BoxFluxSettings (src/box_flux.rs:47-52)."""
    pressure: object  # PressureSettings
    actual_divergence_limit: float


@dataclass
class BoxFluxWork:
    """BoxFluxWork (src/box_flux.rs:89-107)."""
    kinetic_before: float
    kinetic_after: float
    correction_energy: float
    boundary_pressure_work: float
    divergence_residual_work: float
    correction_residual_work: float
    budget_error: float


@dataclass
class BoxFluxReport:
    """BoxFluxReport (src/box_flux.rs:108-116)."""
    boundary: BoxFluxStamp
    pressure: object  # PressureReport
    actual_divergence_max: float
    net_outward_flux: float
    flux_rounding_budget: float
    work: BoxFluxWork

    @classmethod
    def from_c(cls, r: N.BoxFluxReport) -> "BoxFluxReport":
        from . import PressureReport

        return cls(BoxFluxStamp(int(r.boundary_id), int(r.boundary_version)), PressureReport.from_c(r.pressure),
                   r.actual_divergence_max, r.net_outward_flux, r.flux_rounding_budget,
                   BoxFluxWork(r.kinetic_before, r.kinetic_after, r.correction_energy, r.boundary_pressure_work,
                               r.divergence_residual_work, r.correction_residual_work, r.budget_error))


def _faces(arrays, writable: bool):
    """(pointer array, length array, device?, keep-alive) of three face arrays."""
    ptrs, lens, keep = (C.c_void_p * 3)(), (C.c_size_t * 3)(), []
    device = [hasattr(a, "data_ptr") for a in arrays]
    if any(device) and not all(device):
        raise ValueError("face arrays must be all CUDA tensors or all numpy arrays")
    for i, a in enumerate(arrays):
        if device[i]:
            if a.dtype.itemsize != 4 or not a.is_floating_point() or not a.is_contiguous():
                raise ValueError("contiguous f32 tensors required")
            ptrs[i], lens[i] = a.data_ptr(), a.numel()
        else:
            if not isinstance(a, np.ndarray) or a.dtype != np.float32 or not a.flags.c_contiguous:
                raise ValueError("contiguous f32 numpy arrays required")
            if writable and not a.flags.writeable:
                raise ValueError("writable output required")
            ptrs[i], lens[i] = a.ctypes.data, a.size
            keep.append(a)
    return ptrs, lens, all(device), keep


class BoxFluxWorkspace:
    """BoxFluxWorkspace (src/box_flux.rs:117-198): a pressure workspace plus
    the projection's device passes, for one grid and density."""

    def __init__(self, grid, density: float, limit: int, implementation=0, device: int = 0):
        self.grid = grid
        self.density = float(density)
        self._implementation = implementation
        h = C.c_void_p()
        r = N.BoxFluxReport()
        st = lib().rb200_box_flux_create(C.byref(grid.c()), self.density, int(limit), int(implementation), device,
                                         C.byref(h), C.byref(r))
        if st != N.OK:
            inv = "InvalidDensity" if not (math.isfinite(self.density) and self.density > 0) else "InvalidGrid"
            raise _error(st, r, inv)
        self._h = h
        self.device = device

    def close(self):
        if getattr(self, "_h", None):
            lib().rb200_box_flux_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def allocated_bytes(self) -> int:
        return int(lib().rb200_box_flux_allocated_bytes(self._h))

    def implementation(self):
        return self._implementation

    def stream(self) -> int:
        return int(lib().rb200_box_flux_stream(self._h) or 0)

    def pressure(self) -> np.ndarray:
        """The last pressure (gauge cell zero); meaningful after a successful projection."""
        out = np.empty(self.grid.cell_len(), np.float64)
        st = lib().rb200_box_flux_pressure(self._h, out.ctypes.data, out.size)
        if st != N.OK:
            raise _error(st, N.BoxFluxReport())
        return out

    def pressure_device_ptr(self) -> int:
        return int(lib().rb200_box_flux_pressure_device(self._h) or 0)

    @staticmethod
    def _sync_producers(arrays):
        for a in arrays:
            if hasattr(a, "device"):
                import torch

                torch.cuda.current_stream(a.device).synchronize()
                return

    def divergence(self, velocity: Sequence, out) -> None:
        """The measured divergence of a full face field (CUDA tensors), outer samples included."""
        ptrs, lens, dev, _ = _faces(velocity, False)
        if not dev or not hasattr(out, "data_ptr"):
            raise ValueError("divergence runs on CUDA tensors")
        self._sync_producers(velocity)
        st = lib().rb200_box_flux_divergence_device(self._h, ptrs, lens, out.data_ptr(), out.numel())
        if st == N.BOX_FLUX_REJECTED:
            r = N.BoxFluxReport()
            r.error = 8
            raise _error(st, r)
        if st != N.OK:
            raise _error(st, N.BoxFluxReport())

    def project(self, old: Sequence, dt: float, boundary: PrescribedBoxFlux, settings: BoxFluxSettings,
                output: Sequence, cancelled: Optional[Callable[[str], bool]] = None) -> BoxFluxReport:
        """project (src/box_flux.rs:213-397). `cancelled(stage)` is asked at
        each stage; a failure after the correction began may leave `output`
        partial."""
        iptr, ilen, idev, keep_in = _faces(old, False)
        optr, olen, odev, keep_out = _faces(output, True)
        if idev != odev:
            raise ValueError("old and output must both be CUDA tensors or both numpy arrays")
        if idev:
            self._sync_producers(list(old) + list(output))
        r = N.BoxFluxReport()
        if cancelled is None:
            cb = C.cast(None, N.BOX_FLUX_CANCEL_FN)
        else:
            cb = N.BOX_FLUX_CANCEL_FN(lambda _ctx, stage: 1 if cancelled(N.BOX_FLUX_STAGES[stage]) else 0)
        fn = lib().rb200_box_flux_project_device if idev else lib().rb200_box_flux_project
        st = fn(self._h, iptr, ilen, float(dt), C.byref(boundary.c()), C.byref(settings.pressure.c()),
                float(settings.actual_divergence_limit), optr, olen, C.byref(r), cb, None)
        if st != N.OK:
            inv = "InvalidTimeStep" if not (math.isfinite(dt) and dt > 0) else "InvalidSettings"
            raise _error(st, r, inv)
        return BoxFluxReport.from_c(r)

    def last_pass_ms(self):
        """(RHS pass, correction pass) device milliseconds inside the last projection (-1: not run)."""
        a, b = C.c_double(), C.c_double()
        st = lib().rb200_box_flux_last_pass_ms(self._h, C.byref(a), C.byref(b))
        if st != N.OK:
            raise _error(st, N.BoxFluxReport())
        return a.value, b.value

    def profile(self, which: int, launches: int = 20) -> float:
        """Average device milliseconds of the last projection's RHS (0) or correction (1) pass."""
        ms = C.c_double()
        st = lib().rb200_box_flux_profile(self._h, which, launches, C.byref(ms))
        if st != N.OK:
            raise _error(st, N.BoxFluxReport())
        return ms.value
