"""Liquid-volume transport on the device (src/liquid_volume.rs).

LiquidVolumeState mirrors the reference's type of the same name for an inlet
boundary and the all-cells divergence domain: the represented liquid fraction
(f64 per cell) is moved through f32 face velocities by first-order
shared-face donor transfer, with the reference's checked arithmetic, volume
ledger and error order. The state lives in device memory; advance() runs one
interval and commits it only when it is accepted.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from . import _native as N
from ._native import lib

__all__ = ["LiquidVolumeError", "LiquidVolumeSettings", "LiquidInlet", "LiquidVolumeReport", "LiquidVolumeState",
           "LiquidOccupancy", "LiquidStepReport", "LiquidTransportSimulation"]


class LiquidVolumeError(RuntimeError):
    """LiquidVolumeError (src/liquid_volume.rs:27-72): kind names the variant;
    cell, actual and limit carry its payload where it has one."""

    def __init__(self, kind: str, cell: int = 0, actual: float = 0.0, limit: float = 0.0, status: int = 0):
        self.kind = kind
        self.cell = cell
        self.actual = actual
        self.limit = limit
        self.status = status
        super().__init__(f"liquid volume transport rejected operation: {kind}"
                         + (f" (cell {cell}, {actual}, {limit})" if kind in ("CourantLimit", "FractionBounds")
                            else ""))

    @classmethod
    def from_report(cls, status: int, r: N.LiquidReport) -> "LiquidVolumeError":
        if status != N.LIQUID_REJECTED:
            return cls(N.STATUS_NAMES.get(status, f"Status{status}"), status=status)
        err = cls(N.LIQUID_ERRORS.get(r.error, f"Error{r.error}"), int(r.error_cell), r.error_actual,
                  r.error_limit, status)
        # Cancelled { stage } (src/liquid_volume.rs:60-62)
        err.stage = N.VOLUME_STAGES[int(r.error_cell)] if err.kind == "Cancelled" else None
        return err


@dataclass
class LiquidVolumeSettings:
    """LiquidVolumeSettings (src/liquid_volume.rs:192-199)."""
    max_outward_courant: float
    actual_divergence_limit: float


@dataclass
class LiquidInlet:
    """LiquidInlet (src/liquid_volume.rs:76-96): fraction[d] = (lower, upper)
    outside fraction of axis d, used on inflow only."""
    stamp: tuple
    fraction: Sequence[Sequence[float]]


class LiquidOccupancy:
    DRY, MIXED, FULL = "Dry", "Mixed", "Full"


@dataclass
class LiquidVolumeReport:
    """LiquidVolumeReport (src/liquid_volume.rs:200-229)."""
    stamp: tuple
    flow: tuple
    inlet: tuple
    source: Optional[tuple]
    dt: float
    time: float
    liquid_volume_before: float
    liquid_volume_after: float
    inward_boundary_volume: float
    outward_boundary_volume: float
    source_volume: float
    volume_balance_error: float
    volume_rounding_budget: float
    liquid_mass_before: float
    liquid_mass_after: float
    max_outward_courant: float
    actual_divergence_max: float
    fraction_min: float
    fraction_max: float
    dry_cells: int
    mixed_cells: int
    full_cells: int
    periodic: bool = False

    @classmethod
    def from_c(cls, r: N.LiquidReport) -> "LiquidVolumeReport":
        st = lambda s: (int(s.id), int(s.version))  # noqa: E731
        return cls(st(r.stamp), st(r.flow), st(r.inlet), st(r.source) if r.has_source else None, r.dt, r.time,
                   r.liquid_volume_before, r.liquid_volume_after, r.inward_boundary_volume,
                   r.outward_boundary_volume, r.source_volume, r.volume_balance_error, r.volume_rounding_budget,
                   r.liquid_mass_before, r.liquid_mass_after, r.max_outward_courant, r.actual_divergence_max,
                   r.fraction_min, r.fraction_max, int(r.dry_cells), int(r.mixed_cells), int(r.full_cells),
                   bool(r.periodic))


def _ptr(x):
    """Device pointer of a CUDA tensor, or a host numpy array kept alive by the caller."""
    if hasattr(x, "data_ptr"):
        if not x.is_contiguous():
            raise ValueError("contiguous tensor required")
        return x.data_ptr()
    return x.ctypes.data_as(C.c_void_p).value


class LiquidVolumeState:
    """The accepted liquid fraction of one box on the device."""

    def __init__(self, grid, density: float, stamp, fraction, limit: int = 1 << 62, device: int = 0):
        self.grid = grid
        self.density = float(density)
        if not hasattr(fraction, "data_ptr"):
            fraction = np.ascontiguousarray(fraction, dtype=np.float64)
            if fraction.size != grid.cell_len():
                raise LiquidVolumeError("LengthMismatch")
        elif fraction.numel() != grid.cell_len():
            raise LiquidVolumeError("LengthMismatch")
        h = C.c_void_p()
        err = N.LiquidReport()
        st = lib().rb200_liquid_create(C.byref(grid.c()), self.density, N.LiquidStamp(*stamp), _ptr(fraction),
                                       int(limit), device, C.byref(h), C.byref(err))
        if st != N.OK:
            raise LiquidVolumeError.from_report(st, err)
        self._h = h
        self.device = device

    def close(self):
        if getattr(self, "_h", None):
            lib().rb200_liquid_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def allocated_bytes(self) -> int:
        return int(lib().rb200_liquid_allocated_bytes(self._h))

    def _state(self):
        p = C.c_void_p()
        s = N.LiquidStamp()
        t = C.c_double()
        lib().rb200_liquid_state(self._h, C.byref(p), C.byref(s), C.byref(t))
        return p.value or 0, (int(s.id), int(s.version)), t.value

    @property
    def stamp(self):
        return self._state()[1]

    @property
    def time(self) -> float:
        return self._state()[2]

    def fraction_device_ptr(self) -> int:
        """Device pointer of the accepted fraction (valid until the next advance)."""
        return self._state()[0]

    def fraction(self) -> np.ndarray:
        out = np.empty(self.grid.cell_len(), np.float64)
        st = lib().rb200_liquid_download(self._h, out.ctypes.data_as(C.c_void_p), out.size)
        if st != N.OK:
            raise LiquidVolumeError(N.STATUS_NAMES.get(st, f"Status{st}"), status=st)
        return out

    def occupancy(self, cell: int) -> Optional[str]:
        f = self.fraction()
        if not 0 <= cell < f.size:
            return None
        return LiquidOccupancy.DRY if f[cell] == 0.0 else (LiquidOccupancy.FULL if f[cell] == 1.0
                                                           else LiquidOccupancy.MIXED)

    def _flow(self, velocity, start, dt, flow_stamp):
        ptrs = [v if isinstance(v, int) else _ptr(v) for v in velocity]
        return N.LiquidFlow(N.LiquidStamp(*flow_stamp), ptrs[0], ptrs[1], ptrs[2], float(start), float(dt))

    @staticmethod
    def _source(source, source_stamp):
        if source is None:
            return None
        return N.LiquidSource(N.LiquidStamp(*source_stamp), source if isinstance(source, int) else _ptr(source))

    @staticmethod
    def _settings(settings):
        return N.LiquidSettings(settings.max_outward_courant, settings.actual_divergence_limit)

    @staticmethod
    def _cancel(cancel):
        """The C callback for `cancel(stage_name) -> bool` (None: never)."""
        if cancel is None:
            return N.STEP_CANCEL_FN()
        return N.STEP_CANCEL_FN(lambda ctx, stage: 1 if cancel(N.VOLUME_STAGES[stage]) else 0)

    def advance(self, velocity, start: float, dt: float, flow_stamp, inlet: LiquidInlet,
                settings: LiquidVolumeSettings, source=None, source_stamp=(0, 0), stream: int = 0,
                cancel=None) -> LiquidVolumeReport:
        """One interval through the f32 face velocities `velocity` (three CUDA
        tensors, or device pointers) over [start, start + dt]; source: an f64
        CUDA tensor of m^3/s per cell or None. `cancel(stage)` is asked at the
        reference's VolumeStage points ("BeforeFlux", "FaceFluxSlice",
        "CellUpdateSlice", "BeforeCommit"); True cancels with the state
        unchanged (LiquidVolumeError kind "Cancelled", .stage)."""
        inl = N.LiquidInlet(N.LiquidStamp(*inlet.stamp),
                            (C.c_double * 6)(*[float(x) for pair in inlet.fraction for x in pair]))
        src = self._source(source, source_stamp)
        rep = N.LiquidReport()
        cb = self._cancel(cancel)
        st = lib().rb200_liquid_advance_cancellable(self._h, C.byref(self._flow(velocity, start, dt, flow_stamp)),
                                                    C.byref(inl), C.byref(src) if src else None,
                                                    C.byref(self._settings(settings)), cb, None, C.byref(rep),
                                                    stream or None)
        if st != N.OK:
            raise LiquidVolumeError.from_report(st, rep)
        return LiquidVolumeReport.from_c(rep)

    def advance_periodic(self, velocity, start: float, dt: float, flow_stamp, boundary_stamp,
                         settings: LiquidVolumeSettings, source=None, source_stamp=(0, 0), stream: int = 0,
                         cancel=None) -> LiquidVolumeReport:
        """advance_periodic (src/liquid_volume.rs:389-406): the box wraps
        around on every axis; seams must carry equal velocities. `cancel` as
        for advance."""
        src = self._source(source, source_stamp)
        rep = N.LiquidReport()
        cb = self._cancel(cancel)
        st = lib().rb200_liquid_advance_periodic_cancellable(
            self._h, C.byref(self._flow(velocity, start, dt, flow_stamp)), N.LiquidStamp(*boundary_stamp),
            C.byref(src) if src else None, C.byref(self._settings(settings)), cb, None, C.byref(rep),
            stream or None)
        if st != N.OK:
            raise LiquidVolumeError.from_report(st, rep)
        return LiquidVolumeReport.from_c(rep)


@dataclass
class LiquidStepReport:
    """LiquidStepReport's carrier and liquid parts (src/liquid_step.rs)."""
    carrier: object
    liquid: LiquidVolumeReport


class LiquidTransportSimulation:
    """LiquidTransportSimulation (src/liquid_step.rs:828-900) on a resident
    carrier: the carrier owns a liquid-volume state, and each step advances it
    through the step's corrected faces before the step commits. A rejected
    transport rejects the whole step; neither state changes."""

    def __init__(self, carrier, density: float, stamp, fraction, flow_id: int = 0, limit: int = 1 << 62):
        self.carrier = carrier
        grid = carrier.grid
        if not hasattr(fraction, "data_ptr"):
            fraction = np.ascontiguousarray(fraction, dtype=np.float64)
            if fraction.size != grid.cell_len():
                raise LiquidVolumeError("LengthMismatch")
        err = N.LiquidReport()
        st = lib().rb200_carrier_attach_liquid(carrier._handle, float(density), N.LiquidStamp(*stamp), int(flow_id),
                                               _ptr(fraction), int(limit), C.byref(err))
        if st != N.OK:
            raise LiquidVolumeError.from_report(st, err)
        self._keep = []

    def step(self, params, inlet: LiquidInlet, settings: LiquidVolumeSettings, source=None,
             source_stamp=(0, 0)) -> LiquidStepReport:
        """One liquid step; raises LiquidVolumeError when the transport
        rejects it, the carrier's SimulationError when the carrier does."""
        inl = N.LiquidInlet(N.LiquidStamp(*inlet.stamp),
                            (C.c_double * 6)(*[float(x) for pair in inlet.fraction for x in pair]))
        src = None
        if source is not None:
            src = N.LiquidSource(N.LiquidStamp(*source_stamp), _ptr(source))
            self._keep = [source]
        st = lib().rb200_carrier_liquid_inputs(self.carrier._handle, C.byref(inl), C.byref(src) if src else None,
                                               C.byref(N.LiquidSettings(settings.max_outward_courant,
                                                                        settings.actual_divergence_limit)))
        if st != N.OK:
            raise LiquidVolumeError(N.STATUS_NAMES.get(st, f"Status{st}"), status=st)
        from . import SimulationError

        try:
            rep = self.carrier.step(params)
        except SimulationError as e:
            if e.status == N.LIQUID_REJECTED:
                lr = N.LiquidReport()
                lib().rb200_carrier_liquid_report(self.carrier._handle, C.byref(lr))
                raise LiquidVolumeError.from_report(N.LIQUID_REJECTED, lr) from None
            raise
        lr = N.LiquidReport()
        lib().rb200_carrier_liquid_report(self.carrier._handle, C.byref(lr))
        return LiquidStepReport(rep, LiquidVolumeReport.from_c(lr))

    def _inputs(self, inlet, settings, source, source_stamp):
        inl = N.LiquidInlet(N.LiquidStamp(*inlet.stamp),
                            (C.c_double * 6)(*[float(x) for pair in inlet.fraction for x in pair]))
        src = None
        if source is not None:
            src = N.LiquidSource(N.LiquidStamp(*source_stamp), _ptr(source))
            self._keep = [source]
        st = lib().rb200_carrier_liquid_inputs(self.carrier._handle, C.byref(inl), C.byref(src) if src else None,
                                               C.byref(N.LiquidSettings(settings.max_outward_courant,
                                                                        settings.actual_divergence_limit)))
        if st != N.OK:
            raise LiquidVolumeError(N.STATUS_NAMES.get(st, f"Status{st}"), status=st)

    def step_with_box_flux(self, requested_dt: float, inlet: LiquidInlet, settings: LiquidVolumeSettings, workspace,
                           boundary, smoke_source=None, forces=(), source=None, source_stamp=(0, 0), cancel=None):
        """LiquidTransportSimulation::step_with_box_flux (src/liquid_step.rs:548-567):
        the carrier's box-flux step (rheon_b200.simulation.step_with_box_flux)
        with the transport through its candidate faces, one transaction.
        Returns (BoxFluxStepReport, LiquidVolumeReport); raises
        LiquidVolumeError when the transport rejects the step, StepError when
        the carrier does."""
        from . import simulation as S

        self._inputs(inlet, settings, source, source_stamp)
        try:
            rep = S.step_with_box_flux(self.carrier, requested_dt, smoke_source, forces, workspace, boundary, cancel)
        except S.StepError as e:
            if e.status == N.LIQUID_REJECTED:
                lr = N.LiquidReport()
                lib().rb200_carrier_liquid_report(self.carrier._handle, C.byref(lr))
                raise LiquidVolumeError.from_report(N.LIQUID_REJECTED, lr) from None
            raise
        lr = N.LiquidReport()
        lib().rb200_carrier_liquid_report(self.carrier._handle, C.byref(lr))
        return rep, LiquidVolumeReport.from_c(lr)

    def _state(self):
        p = C.c_void_p()
        s = N.LiquidStamp()
        t = C.c_double()
        st = lib().rb200_carrier_liquid_state(self.carrier._handle, C.byref(p), C.byref(s), C.byref(t))
        if st != N.OK:
            raise LiquidVolumeError(N.STATUS_NAMES.get(st, f"Status{st}"), status=st)
        return p.value or 0, (int(s.id), int(s.version)), t.value

    @property
    def stamp(self):
        return self._state()[1]

    @property
    def time(self) -> float:
        return self._state()[2]

    def fraction(self) -> np.ndarray:
        out = np.empty(self.carrier.grid.cell_len(), np.float64)
        st = lib().rb200_carrier_liquid_download(self.carrier._handle, out.ctypes.data_as(C.c_void_p), out.size)
        if st != N.OK:
            raise LiquidVolumeError(N.STATUS_NAMES.get(st, f"Status{st}"), status=st)
        return out
