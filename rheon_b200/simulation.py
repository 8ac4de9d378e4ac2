"""The step owner's forcing and boundary domains on the resident carrier
(src/simulation.rs:393-581, src/forces.rs, src/box_flux_step.rs).

step / step_with_forces / step_with_box_flux run the reference's
prepare_impl stage sequence on an f32 carrier with a tracer: the smoke
source, the caller's body forces and (for step_with_box_flux) the prescribed
box flux, with the reference's dt policy, gates, cancellation stages and work
ledger. A failed or cancelled step leaves the accepted state untouched.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Callable, Optional, Sequence

from . import _native as N
from ._native import lib
from .box_flux import BoxFluxReport, BoxFluxWorkspace, PrescribedBoxFlux

__all__ = ["SmokeSource", "ForceUnits", "ForceRegion", "BodyForce", "StepStage", "ForceReport", "ForcedStepReport",
           "BoxFluxTracerPolicy", "BoxFluxStepBoundary", "BoxFluxStepWork", "BoxFluxStepReport",
           "BoxFluxStepWorkspace", "StepError", "step", "step_with_forces", "step_with_box_flux"]


@dataclass(frozen=True)
class SmokeSource:
    """SmokeSource (src/simulation.rs:19-27)."""
    lower: Sequence[float]
    upper: Sequence[float]
    tracer_rate: float
    vertical_acceleration: float

    def c(self) -> N.SmokeSourceC:
        return N.SmokeSourceC((C.c_double * 3)(*self.lower), (C.c_double * 3)(*self.upper), self.tracer_rate,
                              self.vertical_acceleration)


class ForceUnits:
    ACCELERATION = 0
    FORCE_DENSITY = 1


@dataclass(frozen=True)
class ForceRegion:
    lower: Sequence[float]
    upper: Sequence[float]


@dataclass(frozen=True)
class BodyForce:
    """BodyForce (src/forces.rs:28-45)."""
    value: Sequence[float]
    units: int = ForceUnits.ACCELERATION
    region: Optional[ForceRegion] = None


class StepStage:
    """StepStage (src/simulation.rs:28-42), by name."""
    BEFORE_ADVECTION, VELOCITY_SLICE, BEFORE_FORCES, FORCE_SLICE, VISCOSITY, BEFORE_PRESSURE, PRESSURE_ITERATION, \
        PROJECTION_SLICE, BEFORE_PROJECTION_ACCEPTANCE, BEFORE_TRACER, TRACER_SLICE, BEFORE_COMMIT, \
        LIQUID_BEFORE_COMMIT = N.STEP_STAGES


class BoxFluxTracerPolicy:
    CLAMPED_APPEARANCE = 0


@dataclass(frozen=True)
class BoxFluxStepBoundary:
    """BoxFluxStepBoundary (src/box_flux_step.rs:13-20)."""
    flux: PrescribedBoxFlux
    tracer: int = BoxFluxTracerPolicy.CLAMPED_APPEARANCE


@dataclass
class ForceReport:
    """ForceReport (src/forces.rs:47-55)."""
    kinetic_energy_before: float
    kinetic_energy_after: float
    applied_work: float


@dataclass
class ForcedStepReport:
    """ForcedStepReport (src/forces.rs:56-61): the StepReport fields and the force stage's report."""
    dt: float
    time: float
    generation: int
    pressure: object
    actual_divergence_max: float
    courant: float
    tracer_integral: float
    kinetic_energy: float
    forces: Optional[ForceReport]


@dataclass
class BoxFluxStepWork:
    """BoxFluxStepWork (src/box_flux_step.rs:22-42)."""
    kinetic_old: float
    kinetic_after_advection: float
    kinetic_after_smoke_force: float
    kinetic_before_projection: float
    kinetic_accepted: float
    advection_change: float
    smoke_force_work: float
    external_force_work: float
    budget_error: float
    boundary_volume_imbalance: float
    tracer_old_integral: float
    tracer_transport_change: float
    tracer_source_change: float


@dataclass
class BoxFluxStepReport:
    """BoxFluxStepReport (src/box_flux_step.rs:43-52)."""
    step: ForcedStepReport
    projection: BoxFluxReport
    work: BoxFluxStepWork
    tracer_policy: int
    simulation_array_bytes: int
    boundary_workspace_array_bytes: int


class StepError(RuntimeError):
    """SimulationError (src/simulation.rs:55-83). kind is the variant
    ("InvalidSource", "Cancelled", "DivergenceLimit", "Pressure", "BoxFlux",
    "Operator", ...); inner names a wrapped error; stage, actual and limit
    carry the payloads."""

    def __init__(self, status: int, r: N.ForcedStepReport, invalid_time_step: bool = False):
        self.status = status
        self.stage = None
        self.actual = None
        self.limit = None
        self.inner = None
        if status == N.SIMULATION_REJECTED:
            self.kind = N.SIMULATION_ERRORS.get(r.error, f"Error{r.error}")
            if self.kind == "Cancelled":
                self.stage = N.STEP_STAGES[r.stage]
        elif status in (N.DIVERGENCE_LIMIT, N.COURANT_LIMIT):
            self.kind = "DivergenceLimit" if status == N.DIVERGENCE_LIMIT else "CourantLimit"
            self.actual, self.limit = r.error_actual, r.error_limit
        elif status == N.ARITHMETIC_FAILURE:
            self.kind = "ArithmeticFailure"
        elif status == N.LIQUID_REJECTED:
            self.kind = "LiquidVolume"  # the transport's report: rb200_carrier_liquid_report
        elif status == N.BOX_FLUX_REJECTED:
            self.kind = "BoxFlux"
            self.inner = N.BOX_FLUX_ERRORS.get(r.projection.error, str(r.projection.error))
        elif status in (N.CANCELLED, N.ITERATION_LIMIT, N.BREAKDOWN, N.INCOMPATIBLE_RHS, N.OUT_OF_MEMORY):
            self.kind = "Pressure"
            self.inner = N.STATUS_NAMES[status]
        elif status in (N.NONFINITE_INPUT, N.NONZERO_WALL_VELOCITY, N.LENGTH_MISMATCH):
            self.kind = "Operator"
            self.inner = N.STATUS_NAMES[status]
        elif status == N.INVALID_ARGUMENT and invalid_time_step:
            self.kind = "InvalidTimeStep"
        else:
            self.kind = N.STATUS_NAMES.get(status, f"Status{status}")
        super().__init__(f"simulation rejected operation: {self.kind}" + (f"({self.inner})" if self.inner else "")
                         + (f" at {self.stage}" if self.stage else ""))


class BoxFluxStepWorkspace:
    """BoxFluxStepWorkspace (src/box_flux_step.rs:58-117): the boundary's
    projection workspace. The provisional faces of the step are the carrier's
    own candidate buffers; the accounting keeps the reference's
    56 bytes per cell plus 4 per face."""

    def __init__(self, grid, density: float, limit: int, implementation=0, device: int = 0):
        faces = sum(grid.face_len(a) for a in range(3))
        required = 56 * grid.cell_len() + 4 * faces
        if required > limit:
            from .box_flux import BoxFluxError

            raise BoxFluxError("BufferLimit", required=required, limit=int(limit))
        self.projection = BoxFluxWorkspace(grid, density, limit - 4 * faces, implementation, device)
        self.grid = grid
        self._faces = faces

    def allocated_bytes(self) -> int:
        return self.projection.allocated_bytes() + 4 * self._faces

    def close(self):
        self.projection.close()


def _run(carrier, requested_dt, source, forces, workspace, boundary, cancel):
    fa = (N.BodyForceC * max(1, len(forces)))()
    for i, f in enumerate(forces):
        fa[i].value = (C.c_double * 3)(*f.value)
        fa[i].units = int(f.units)
        fa[i].has_region = 1 if f.region is not None else 0
        if f.region is not None:
            fa[i].lower = (C.c_double * 3)(*f.region.lower)
            fa[i].upper = (C.c_double * 3)(*f.region.upper)
    src = source.c() if source is not None else None
    bc = boundary.flux.c() if boundary is not None else None
    prm = N.ForcedStepParams(float(requested_dt), C.pointer(src) if src is not None else None,
                             C.cast(fa, C.POINTER(N.BodyForceC)), len(forces),
                             workspace.projection._h if workspace is not None else None,
                             C.pointer(bc) if bc is not None else None,
                             int(boundary.tracer) if boundary is not None else 0)
    rep = N.ForcedStepReport()
    cb = N.STEP_CANCEL_FN(lambda _ctx, stage: 1 if cancel(N.STEP_STAGES[stage]) else 0) if cancel else \
        C.cast(None, N.STEP_CANCEL_FN)
    st = lib().rb200_carrier_step_forced(carrier._handle, C.byref(prm), C.byref(rep), cb, None)
    if st != N.OK:
        import math

        raise StepError(st, rep, not (math.isfinite(requested_dt) and requested_dt > 0))
    return rep


def _forced(rep: N.ForcedStepReport) -> ForcedStepReport:
    from . import PressureReport

    forces = ForceReport(rep.force_kinetic_before, rep.force_kinetic_after, rep.force_applied_work) \
        if rep.has_forces else None
    return ForcedStepReport(rep.dt, rep.time, int(rep.generation), PressureReport.from_c(rep.pressure),
                            rep.actual_divergence_max, rep.courant, rep.tracer_integral, rep.kinetic_energy, forces)


def step(carrier, requested_dt: float, source: Optional[SmokeSource] = None,
         cancel: Optional[Callable[[str], bool]] = None) -> ForcedStepReport:
    """Simulation::step (src/simulation.rs:393-416)."""
    return _forced(_run(carrier, requested_dt, source, (), None, None, cancel))


def step_with_forces(carrier, requested_dt: float, source: Optional[SmokeSource], forces: Sequence[BodyForce],
                     cancel: Optional[Callable[[str], bool]] = None) -> ForcedStepReport:
    """Simulation::step_with_forces (src/simulation.rs:417-429)."""
    return _forced(_run(carrier, requested_dt, source, tuple(forces), None, None, cancel))


def step_with_box_flux(carrier, requested_dt: float, source: Optional[SmokeSource], forces: Sequence[BodyForce],
                       workspace: BoxFluxStepWorkspace, boundary: BoxFluxStepBoundary,
                       cancel: Optional[Callable[[str], bool]] = None) -> BoxFluxStepReport:
    """Simulation::step_with_box_flux (src/simulation.rs:551-579)."""
    rep = _run(carrier, requested_dt, source, tuple(forces), workspace, boundary, cancel)
    work = BoxFluxStepWork(*[getattr(rep, n) for n in N.FORCED_WORK])
    return BoxFluxStepReport(_forced(rep), BoxFluxReport.from_c(rep.projection), work, rep.tracer_policy,
                             int(rep.simulation_array_bytes), int(rep.boundary_workspace_array_bytes))
