"""The forced step on the resident carrier (smoke source, body forces, box-flux
boundary) against the reference's contract cases and the oracle.

Cases restate tests/simulation_contract.rs, tests/forces_contract.rs and
tests/box_flux_step_contract.rs; their exact assertions (hand energies and
works, dt, Courant, tracer values) are kept exact. Against the oracle
(orc_sim_step) on random states: stored faces within one f32 ulp (the device
pressure is within 1e-12 of the oracle's, a rare face rounds the other way),
tracer within 1e-6, energies and works within 1e-9 relative of their
magnitudes.
"""
import math

import numpy as np
import pytest

import oracle as O
import rheon_b200 as R
from rheon_b200 import simulation as S
from rheon_b200.box_flux import BoxFluxStamp, PrescribedBoxFlux

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

V1 = [R.PressureImplementation.JACOBI_PCG_V1, R.PressureImplementation.SGS_PCG_V1]
ORACLE_METHOD = {R.PressureImplementation.JACOBI_PCG_V1: O.JACOBI_PCG_V1,
                 R.PressureImplementation.SGS_PCG_V1: O.SGS_PCG_V1}
MAXF = 1.7976931348623157e308


@pytest.fixture(scope="module", autouse=True)
def _device():
    if not torch.cuda.is_available() or R.device_count() == 0:
        pytest.skip("no B200")
    yield


def near(a, b, tol=2e-10):
    assert abs(a - b) < tol * max(abs(a), abs(b), 1.0), (a, b)


def carrier(counts, spacing=(1.0, 1.0, 1.0), density=2.0, method=R.PressureImplementation.JACOBI_PCG_V1,
            pressure=(1e-12, 1e-12, 1e-9, 1000), limit=1e-5, courant=1.0, faces=None, tracer=None):
    g = R.GridGeometry(counts, spacing)
    cfg = R.CarrierConfig(density=density, pressure=R.PressureSettings(*pressure), actual_divergence_limit=limit,
                          max_courant=courant, storage="f32", implementation=method, with_tracer=True)
    sim = R.CarrierSimulation(g, cfg)
    faces = faces if faces is not None else [np.zeros(g.face_len(d), np.float32) for d in range(3)]
    tracer = tracer if tracer is not None else np.zeros(g.cell_len(), np.float32)
    sim.upload(faces, tracer)
    return sim


def workspace(sim, limit=1 << 30):
    c = sim.config
    return S.BoxFluxStepWorkspace(sim.grid, c.density, limit, c.implementation)


def snapshot(sim):
    fs, tr = sim.download(with_tracer=True)
    return tuple(np.concatenate([f.view(np.uint32) for f in fs] + [tr.view(np.uint32)]))


def state(sim):
    fs, tr = sim.download(with_tracer=True)
    return fs, tr


def boundary(axis, speed, version=0):
    outward = [[0.0, 0.0] for _ in range(3)]
    outward[axis] = [-speed, speed]
    return S.BoxFluxStepBoundary(PrescribedBoxFlux(BoxFluxStamp(73, version), outward))


def divergence_f32(grid, fs):
    """The test's own divergence (simulation_contract.rs:60-80):
    (dx/h0 + dy/h1) + dz/h2 per cell."""
    n, h = grid.counts, grid.spacing
    x = fs[0].reshape(n[2], n[1], n[0] + 1).astype(np.float64)
    y = fs[1].reshape(n[2], n[1] + 1, n[0]).astype(np.float64)
    z = fs[2].reshape(n[2] + 1, n[1], n[0]).astype(np.float64)
    return (x[:, :, 1:] - x[:, :, :-1]) / h[0] + (y[:, 1:, :] - y[:, :-1, :]) / h[1] + \
        (z[1:, :, :] - z[:-1, :, :]) / h[2]


# ------------------------------------------------------------------ box_flux_step_contract.rs
@pytest.mark.parametrize("method", V1 + [R.PressureImplementation.RBSGS_PCG], ids=lambda m: m.name)
@pytest.mark.parametrize("axis", [0, 1, 2])
@pytest.mark.parametrize("speed", [-0.25, 0.25])
def test_signed_end_boundary_hand_flow_and_work(method, axis, speed):
    """box_flux_step_contract.rs:76-126"""
    counts = [1, 1, 1]
    counts[axis] = 3
    sim = carrier(counts, method=method)
    w = workspace(sim)
    b = boundary(axis, speed, 4)
    for step in (1, 2, 3):
        r = S.step_with_box_flux(sim, 0.5, None, [], w, b)
        assert r.projection.boundary == BoxFluxStamp(73, 4)
        assert r.step.generation == step and r.step.time == 0.5 * step
        fs, _ = state(sim)
        for d in range(3):
            assert np.all(fs[d] == (np.float32(speed) if d == axis else 0.0))
        assert r.step.actual_divergence_max == 0.0
        near(r.work.kinetic_accepted, 0.125)
        near(r.step.kinetic_energy, 0.125)
        near(r.work.budget_error, 0.0)
        assert r.work.boundary_volume_imbalance == 0.0
        if step == 1:
            near(r.work.kinetic_old, 0.0)
            near(r.projection.work.boundary_pressure_work, 0.25)
            near(r.projection.work.correction_energy, 0.125)
        else:
            near(r.work.kinetic_old, 0.125)
            near(r.work.advection_change, 0.0)
            near(r.projection.work.boundary_pressure_work, 0.0)
        assert r.simulation_array_bytes == sim.allocated_bytes()
        assert r.boundary_workspace_array_bytes == w.allocated_bytes()


@pytest.mark.parametrize("method", V1, ids=lambda m: m.name)
def test_boundary_speed_controls_dt_and_courant(method):
    """box_flux_step_contract.rs:127-141"""
    sim = carrier((3, 1, 1), (0.5, 1.0, 1.0), method=method)
    r = S.step_with_box_flux(sim, 20.0, None, [], workspace(sim), boundary(0, 2.0))
    assert r.step.dt == 0.125 and r.step.courant == 0.5 and r.step.time == 0.125


@pytest.mark.parametrize("method", V1, ids=lambda m: m.name)
def test_changing_boundary_versions_publish_only_on_success(method):
    """box_flux_step_contract.rs:142-166"""
    sim = carrier((3, 1, 1), method=method)
    w = workspace(sim)
    S.step_with_box_flux(sim, 0.5, None, [], w, boundary(0, 0.25, 8))
    before = snapshot(sim)
    with pytest.raises(S.StepError) as e:
        S.step_with_box_flux(sim, 0.5, None, [], w, boundary(0, -0.25, 9), lambda s: s == S.StepStage.BEFORE_COMMIT)
    assert e.value.kind == "Cancelled" and e.value.stage == "BeforeCommit"
    assert snapshot(sim) == before
    r = S.step_with_box_flux(sim, 0.5, None, [], w, boundary(0, -0.25, 9))
    assert r.projection.boundary == BoxFluxStamp(73, 9)
    assert np.all(state(sim)[0][0] == -0.25)
    near(r.work.kinetic_old, 0.125)
    near(r.work.budget_error, 0.0)


@pytest.mark.parametrize("method", V1, ids=lambda m: m.name)
def test_external_and_smoke_terms_join_the_ledger(method):
    """box_flux_step_contract.rs:167-212"""
    sim = carrier((2, 2, 1), method=method)
    src = S.SmokeSource((0, 0, 0), (2.0, 2.0, 1.0), 0.5, 0.5)
    f = S.BodyForce((1.0, -0.25, 0.0))
    r = S.step_with_box_flux(sim, 0.25, src, [f], workspace(sim), boundary(0, 0.25))
    near(r.work.smoke_force_work, 0.03125)
    near(r.work.external_force_work, 0.1015625)
    near(r.work.kinetic_before_projection, 0.1328125)
    near(r.work.kinetic_accepted, 0.125)
    near(r.step.forces.applied_work, r.work.external_force_work)
    near(r.work.tracer_source_change, 0.5)
    near(r.work.tracer_transport_change, 0.0)
    near(r.work.budget_error, 0.0)
    fs, _ = state(sim)
    assert r.step.actual_divergence_max == np.max(np.abs(divergence_f32(sim.grid, fs)))


@pytest.mark.parametrize("method", V1, ids=lambda m: m.name)
def test_clamped_appearance_transport_and_saturated_source(method):
    """box_flux_step_contract.rs:213-240"""
    sim = carrier((3, 1, 1), method=method)
    w = workspace(sim)
    S.step_with_box_flux(sim, 0.5, S.SmokeSource((0, 0, 0), (1.0, 1.0, 1.0), 10.0, 0.0), [], w, boundary(0, 0.0))
    assert list(state(sim)[1]) == [1.0, 0.0, 0.0]
    r = S.step_with_box_flux(sim, 0.5, None, [], w, boundary(0, 0.25, 1))
    assert list(state(sim)[1]) == [1.0, 0.125, 0.0]
    near(r.work.tracer_old_integral, 1.0)
    near(r.work.tracer_transport_change, 0.125)
    near(r.work.tracer_source_change, 0.0)
    assert r.work.boundary_volume_imbalance == 0.0 and r.tracer_policy == 0


@pytest.mark.parametrize("method", V1, ids=lambda m: m.name)
@pytest.mark.parametrize("stage", list(S.StepStage.__dict__[k] for k in (
    "BEFORE_ADVECTION", "VELOCITY_SLICE", "BEFORE_FORCES", "FORCE_SLICE", "BEFORE_PRESSURE", "PRESSURE_ITERATION",
    "PROJECTION_SLICE", "BEFORE_PROJECTION_ACCEPTANCE", "BEFORE_TRACER", "TRACER_SLICE", "BEFORE_COMMIT")))
def test_box_flux_cancellation_preserves_state_and_retry_matches_fresh(method, stage):
    """box_flux_step_contract.rs:241-318"""
    src = S.SmokeSource((0, 0, 0), (1.0, 2.0, 2.0), 0.5, 0.125)
    f = S.BodyForce((0.125, -0.25, 0.125), region=S.ForceRegion((0, 0, 0), (2.0, 2.0, 2.0)))
    b = boundary(0, 0.25)
    sim = carrier((3, 2, 2), method=method)
    w = workspace(sim)
    S.step_with_box_flux(sim, 0.125, src, [f], w, b)
    before = snapshot(sim)
    calls = [0]

    def cancel(at):
        if at == stage:
            calls[0] += 1
            slice_stage = stage in ("VelocitySlice", "ForceSlice", "ProjectionSlice", "TracerSlice")
            return calls[0] == (2 if slice_stage else 1)
        return False

    with pytest.raises(S.StepError):
        S.step_with_box_flux(sim, 0.125, src, [f], w, b, cancel)
    assert calls[0] > 0
    assert snapshot(sim) == before
    retry = S.step_with_box_flux(sim, 0.125, src, [f], w, b)
    fresh = carrier((3, 2, 2), method=method)
    fw = workspace(fresh)
    S.step_with_box_flux(fresh, 0.125, src, [f], fw, b)
    expected = S.step_with_box_flux(fresh, 0.125, src, [f], fw, b)
    assert snapshot(sim) == snapshot(fresh)
    assert retry.work.budget_error == expected.work.budget_error


@pytest.mark.parametrize("method", V1, ids=lambda m: m.name)
def test_incompatible_flux_late_overflow_and_exhaustion_never_publish(method):
    """box_flux_step_contract.rs:319-374"""
    sim = carrier((3, 1, 1), method=method)
    w = workspace(sim)
    before = snapshot(sim)
    bad = S.BoxFluxStepBoundary(PrescribedBoxFlux(BoxFluxStamp(73, 0), [[0.0, 0.25], [0.0, 0.0], [0.0, 0.0]]))
    with pytest.raises(S.StepError) as e:
        S.step_with_box_flux(sim, 0.5, None, [], w, bad)
    assert (e.value.kind, e.value.inner) == ("BoxFlux", "IncompatibleFlux") and snapshot(sim) == before
    src = S.SmokeSource((0, 0, 0), (3.0, 1.0, 1.0), MAXF, 0.0)
    with pytest.raises(S.StepError) as e:
        S.step_with_box_flux(sim, 4.0, src, [], w, boundary(0, 0.0))
    assert e.value.kind == "ArithmeticFailure" and snapshot(sim) == before
    S.step_with_box_flux(sim, 0.5, None, [], w, boundary(0, 0.25))
    ex = carrier((3, 1, 1), method=method, pressure=(1e-12, 1e-12, 1e-9, 0))
    before = snapshot(ex)
    with pytest.raises(S.StepError) as e:
        S.step_with_box_flux(ex, 0.5, None, [], w, boundary(0, 0.25))
    assert e.value.kind == "Pressure" and snapshot(ex) == before
    S.step_with_box_flux(ex, 0.5, None, [], w, boundary(0, 0.0, 1))


def test_workspace_must_match_before_any_callback():
    """box_flux_step_contract.rs:375-411"""
    sim = carrier((3, 1, 1))
    before = snapshot(sim)
    c = sim.config
    for grid, density, method in [(R.GridGeometry([3, 1, 1], [1.0] * 3, [1.0, 0.0, 0.0]), c.density, 0),
                                  (sim.grid, 1.0, 0), (sim.grid, c.density, 1)]:
        w = S.BoxFluxStepWorkspace(grid, density, 1 << 20, method)
        calls = []
        with pytest.raises(S.StepError) as e:
            S.step_with_box_flux(sim, 0.5, None, [], w, boundary(0, 0.25), lambda s: calls.append(s) or False)
        assert e.value.kind == "BoundaryWorkspaceMismatch" and calls == []
        assert snapshot(sim) == before


def test_workspace_accounting_and_limit():
    """box_flux_step_contract.rs:412-455"""
    from rheon_b200.box_flux import BoxFluxError

    g = R.GridGeometry([1, 1, 1])
    with pytest.raises(BoxFluxError) as e:
        S.BoxFluxStepWorkspace(g, 2.0, 79)
    assert (e.value.required, e.value.limit) == (80, 79)
    sim = carrier((1, 1, 1))
    w = S.BoxFluxStepWorkspace(g, 2.0, 80)
    assert w.allocated_bytes() == 80
    r = S.step_with_box_flux(sim, 0.5, None, [], w, boundary(0, 0.25))
    assert r.step.kinetic_energy == 0.0 and r.projection.pressure.iterations == 0
    assert r.step.actual_divergence_max == 0.0


@pytest.mark.parametrize("method", V1, ids=lambda m: m.name)
def test_zero_boundary_agrees_with_the_sealed_forced_step(method):
    """box_flux_step_contract.rs:456-503"""
    counts, spacing = (3, 2, 2), (0.5, 1.0, 2.0)
    closed, zero = carrier(counts, spacing, method=method), carrier(counts, spacing, method=method)
    w = workspace(zero)
    src = S.SmokeSource((0, 0, 0), (1.5, 2.0, 4.0), 0.25, 0.5)
    f = S.BodyForce((0.5, -0.125, 0.25), region=S.ForceRegion((0, 0, 0), (1.0, 1.0, 2.0)))
    for _ in range(3):
        stages = []
        a = S.step_with_forces(closed, 0.125, src, [f], lambda s: stages.append(s) or False)
        b = S.step_with_box_flux(zero, 0.125, src, [f], w, boundary(0, 0.0))
        assert snapshot(closed) == snapshot(zero)
        assert a.pressure.iterations == b.step.pressure.iterations
        assert a.actual_divergence_max == b.step.actual_divergence_max
        assert "ProjectionSlice" not in stages and "BeforeProjectionAcceptance" not in stages
        near(b.work.budget_error, 0.0)


@pytest.mark.parametrize("method", V1, ids=lambda m: m.name)
def test_stored_divergence_rejection_after_projection(method):
    """box_flux_step_contract.rs:514-549"""
    sim = carrier((3, 2, 2), (0.5, 1.0, 2.0), method=method, limit=0.0)
    w = workspace(sim)
    before = snapshot(sim)
    f = S.BodyForce((0.1, -0.13, 0.2), region=S.ForceRegion((0, 0, 0), (1.0, 1.0, 2.0)))
    with pytest.raises(S.StepError) as e:
        S.step_with_box_flux(sim, 0.125, None, [f], w, boundary(0, 0.375))
    assert e.value.kind == "DivergenceLimit" and e.value.actual > e.value.limit == 0.0
    assert snapshot(sim) == before
    S.step_with_box_flux(sim, 0.125, None, [], w, boundary(0, 0.0, 1))


@pytest.mark.parametrize("method", V1, ids=lambda m: m.name)
def test_balanced_volume_flux_does_not_certify_tracer_mass(method):
    """box_flux_step_contract.rs:551-593"""
    sim = carrier((3, 2, 1), method=method)
    w = workspace(sim)
    S.step_with_box_flux(sim, 0.5, S.SmokeSource((0, 0, 0), (1.0, 2.0, 1.0), 1.0, 0.0), [], w, boundary(0, 0.0))
    f = S.BodyForce((0.0, 0.5, 0.0), region=S.ForceRegion((0, 0, 0), (1.0, 2.0, 1.0)))
    r = S.step_with_box_flux(sim, 0.25, None, [f], w, boundary(0, 0.25, 1))
    assert r.work.boundary_volume_imbalance == 0.0 and r.work.tracer_source_change == 0.0
    tr = state(sim)[1]
    assert np.all((tr >= 0.0) & (tr <= 0.5))
    assert abs(r.work.tracer_transport_change - 0.0625) > 1e-6
    near(r.work.budget_error, 0.0)


# ------------------------------------------------------------------ forces_contract.rs
def cycle_force():
    return S.BodyForce((2.0, 0.0, 0.0), region=S.ForceRegion((0.0, 0.0, 0.0), (2.0, 1.0, 1.0)))


def cycle(method, density):
    return carrier((2, 2, 1), density=density, method=method, pressure=(1e-11, 1e-12, 1e-9, 1000), limit=1e-6)


@pytest.mark.parametrize("method", V1, ids=lambda m: m.name)
def test_signed_uniform_forces_hand_work_and_hydrostatic_rest(method):
    """forces_contract.rs:59-86"""
    for d, a in enumerate([0.25, -0.5, 1.5]):
        counts, spacing = (3, 4, 2), (0.5, 0.25, 1.0)
        g = R.GridGeometry(counts, spacing, (-1.0, 2.0, -2.0))
        cfg = R.CarrierConfig(density=2.0, pressure=R.PressureSettings(1e-11, 1e-12, 1e-9, 1000),
                              actual_divergence_limit=1e-6, max_courant=1.0, storage="f32", implementation=method,
                              with_tracer=True)
        sim = R.CarrierSimulation(g, cfg)
        sim.upload([np.zeros(g.face_len(q), np.float32) for q in range(3)], np.zeros(g.cell_len(), np.float32))
        faces = (counts[d] - 1) * counts[(d + 1) % 3] * counts[(d + 2) % 3]
        expected = 0.5 * 2.0 * g.cell_volume() * faces * (0.125 * a) ** 2
        value = [0.0, 0.0, 0.0]
        value[d] = a
        r = S.step_with_forces(sim, 0.125, None, [S.BodyForce(tuple(value))])
        assert r.dt == 0.125 and r.forces.kinetic_energy_before == 0.0
        assert r.forces.kinetic_energy_after == expected and r.forces.applied_work == expected
        assert r.actual_divergence_max < 1e-6 and r.kinetic_energy < 1e-16


@pytest.mark.parametrize("method", V1, ids=lambda m: m.name)
def test_localized_force_projects_to_the_four_edge_cycle(method):
    """forces_contract.rs:87-117"""
    sim = cycle(method, 1.0)
    r = S.step_with_forces(sim, 0.25, None, [cycle_force()])
    fs, tr = state(sim)
    x = fs[0].reshape(1, 2, 3)
    y = fs[1].reshape(1, 3, 2)
    for value, expected in [(x[0, 0, 1], 0.125), (x[0, 1, 1], -0.125), (y[0, 1, 0], -0.125), (y[0, 1, 1], 0.125)]:
        assert abs(float(value) - expected) < 1e-8
    assert r.forces.applied_work == 0.125 and abs(r.kinetic_energy - 0.03125) < 1e-8
    assert np.all(tr == 0.0) and np.all(fs[2] == 0.0)


@pytest.mark.parametrize("method", V1, ids=lambda m: m.name)
def test_smoke_force_precedes_the_external_stage(method):
    """forces_contract.rs:118-141"""
    sim = cycle(method, 1.0)
    r = S.step_with_forces(sim, 0.25, S.SmokeSource((0, 0, 0), (1.0, 2.0, 1.0), 0.0, 2.0), [cycle_force()])
    f = r.forces
    assert (f.kinetic_energy_before, f.kinetic_energy_after, f.applied_work) == (0.125, 0.25, 0.125)
    assert r.kinetic_energy < 1e-16 and np.all(state(sim)[1] == 0.0)


@pytest.mark.parametrize("method", V1, ids=lambda m: m.name)
def test_force_density_matches_acceleration_bits(method):
    """forces_contract.rs:142-164"""
    for density in (0.5, 2.0, 8.0):
        a, f = cycle(method, density), cycle(method, density)
        fd = S.BodyForce((2.0 * density, 0.0, 0.0), S.ForceUnits.FORCE_DENSITY, cycle_force().region)
        for _ in range(3):
            ra = S.step_with_forces(a, 0.125, None, [cycle_force()])
            rf = S.step_with_forces(f, 0.125, None, [fd])
            assert ra.forces == rf.forces
            assert snapshot(a) == snapshot(f)


def test_support_excludes_upper_planes_and_walls():
    """forces_contract.rs:165-198"""
    sim = cycle(R.PressureImplementation.JACOBI_PCG_V1, 1.0)
    f = S.BodyForce((2.0, 0.0, 0.0), region=S.ForceRegion((0.0, 0.0, 0.0), (1.0, 1.0, 1.0)))
    r = S.step_with_forces(sim, 0.25, None, [f])
    assert r.forces.applied_work == 0.0 and r.kinetic_energy == 0.0


@pytest.mark.parametrize("method", V1, ids=lambda m: m.name)
def test_overlapping_forces_add_and_the_budget_covers_each_axis(method):
    """forces_contract.rs:199-223"""
    sim = cycle(method, 2.0)
    opposite = S.BodyForce((-2.0, 0.0, 0.0), region=cycle_force().region)
    r = S.step_with_forces(sim, 0.125, None, [cycle_force(), opposite])
    assert r.kinetic_energy == 0.0 and r.forces.applied_work == 0.0
    r = S.step_with_forces(sim, 1.0, None, [S.BodyForce((16.0, -16.0, 16.0), S.ForceUnits.FORCE_DENSITY)])
    assert r.dt == math.sqrt(0.5 / 24.0) and r.courant <= 1.0


@pytest.mark.parametrize("method", V1, ids=lambda m: m.name)
def test_force_cancellation_and_exhaustion_preserve_state(method):
    """forces_contract.rs:224-271"""
    ref = cycle(method, 1.0)
    S.step_with_forces(ref, 0.125, None, [cycle_force()])
    S.step_with_forces(ref, 0.125, None, [cycle_force()])
    for stage in ("BeforeForces", "ForceSlice", "BeforePressure", "PressureIteration", "BeforeCommit"):
        sim = cycle(method, 1.0)
        S.step_with_forces(sim, 0.125, None, [cycle_force()])
        before = snapshot(sim)
        slices = [0]

        def cancel(s):
            if s == "ForceSlice":
                slices[0] += 1
            return s == stage and (stage != "ForceSlice" or slices[0] == 2)

        with pytest.raises(S.StepError) as e:
            S.step_with_forces(sim, 0.125, None, [cycle_force()], cancel)
        if stage in ("BeforeForces", "ForceSlice"):
            assert (e.value.kind, e.value.stage) == ("Cancelled", stage)
        assert snapshot(sim) == before
        S.step_with_forces(sim, 0.125, None, [cycle_force()])
        assert snapshot(sim) == snapshot(ref)
    ex = carrier((2, 2, 1), density=1.0, method=method, pressure=(1e-11, 1e-12, 1e-9, 0), limit=1e-6)
    before = snapshot(ex)
    with pytest.raises(S.StepError):
        S.step_with_forces(ex, 0.125, None, [cycle_force()])
    assert snapshot(ex) == before


def test_invalid_or_unrepresentable_forces():
    """forces_contract.rs:273-333"""
    sim = cycle(R.PressureImplementation.JACOBI_PCG_V1, 0.5)
    S.step_with_forces(sim, 0.125, None, [cycle_force()])
    before = snapshot(sim)
    region = cycle_force().region
    for bad in [S.BodyForce((float("nan"), 0, 0)), S.BodyForce((0, float("inf"), 0)),
                S.BodyForce((2.0, 0, 0), region=S.ForceRegion((0, 0, 0), (3.0, 3.0, 3.0))),
                S.BodyForce((2.0, 0, 0), region=S.ForceRegion((0, 0, 0), (0.0, 0.0, 0.0)))]:
        with pytest.raises(S.StepError) as e:
            S.step_with_forces(sim, 0.125, None, [bad])
        assert e.value.kind == "InvalidForce" and snapshot(sim) == before
    with pytest.raises(S.StepError) as e:
        S.step_with_forces(sim, 0.125, None, [S.BodyForce((MAXF, 0, 0))])
    assert e.value.kind == "TimeResolution" and snapshot(sim) == before
    with pytest.raises(S.StepError) as e:
        S.step_with_forces(sim, 0.125, None, [S.BodyForce((MAXF, 0, 0), S.ForceUnits.FORCE_DENSITY)])
    assert e.value.kind == "ArithmeticFailure" and snapshot(sim) == before
    fresh = cycle(R.PressureImplementation.JACOBI_PCG_V1, 0.5)
    before = snapshot(fresh)
    with pytest.raises(S.StepError) as e:
        S.step_with_forces(fresh, 0.125, None, [S.BodyForce((MAXF, 0, 0))])
    assert e.value.kind == "ArithmeticFailure" and snapshot(fresh) == before
    del region


# ------------------------------------------------------------------ simulation_contract.rs
def eight(**kw):
    kw.setdefault("pressure", (1e-10, 1e-12, 1e-8, 1000))
    return carrier((8, 8, 8), (0.125,) * 3, density=1.0, **kw)


SMOKE = S.SmokeSource((0.25, 0.125, 0.25), (0.75, 0.375, 0.75), 1.0, 0.5)


def test_localized_smoke_is_nontrivial_and_divergence_checked():
    """simulation_contract.rs:54-86"""
    sim = eight()
    for _ in range(6):
        r = S.step(sim, 0.02, SMOKE)
        assert r.tracer_integral > 0.0 and r.kinetic_energy > 0.0
        fs, tr = state(sim)
        maximum = np.max(np.abs(divergence_f32(sim.grid, fs)))
        assert r.actual_divergence_max == maximum <= 1e-5
        assert np.all(np.isfinite(tr)) and np.all((tr >= 0) & (tr <= 1))


@pytest.mark.parametrize("stage", ["BeforeAdvection", "VelocitySlice", "BeforePressure", "PressureIteration",
                                   "BeforeTracer", "TracerSlice", "BeforeCommit"])
def test_cancellation_at_every_stage_preserves_the_state(stage):
    """simulation_contract.rs:87-112"""
    sim = eight()
    S.step(sim, 0.02, SMOKE)
    before = snapshot(sim)
    with pytest.raises(S.StepError):
        S.step(sim, 0.02, SMOKE, lambda s: s == stage)
    assert snapshot(sim) == before
    S.step(sim, 0.02, SMOKE)
    ref = eight()
    S.step(ref, 0.02, SMOKE)
    S.step(ref, 0.02, SMOKE)
    assert snapshot(sim) == snapshot(ref)


def test_exhaustion_invalid_source_single_cell_dt_policy_and_divergence_rejection():
    """simulation_contract.rs:113-128, 154-177, 200-211"""
    sim = eight(pressure=(1e-10, 1e-12, 1e-8, 0))
    before = snapshot(sim)
    with pytest.raises(S.StepError):
        S.step(sim, 0.02, SMOKE)
    assert snapshot(sim) == before
    with pytest.raises(S.StepError) as e:
        S.step(sim, 0.02, S.SmokeSource(SMOKE.lower, SMOKE.upper, float("nan"), 0.5))
    assert e.value.kind == "InvalidSource" and snapshot(sim) == before
    one = carrier((1, 1, 1), density=1.0)
    r = S.step(one, 0.25, S.SmokeSource((0, 0, 0), (1, 1, 1), 10.0, 0.0))
    assert r.actual_divergence_max == 0.0 and list(state(one)[1]) == [1.0] and r.pressure.iterations == 0
    r = S.step(eight(), 1.0, S.SmokeSource(SMOKE.lower, SMOKE.upper, 1.0, 8.0))
    assert r.dt < 1.0 and r.courant <= 1.0
    strict = eight(limit=0.0)
    S.step(strict, 0.02)
    before = snapshot(strict)
    with pytest.raises(S.StepError) as e:
        S.step(strict, 0.02, SMOKE)
    assert e.value.kind == "DivergenceLimit" and snapshot(strict) == before


# ------------------------------------------------------------------ parity with the oracle
def random_state(counts, seed):
    g = O.grid(counts)
    rng = np.random.default_rng(seed)
    faces = []
    for d in range(3):
        fc = O.face_counts(g, d)
        f = rng.uniform(-0.5, 0.5, fc[0] * fc[1] * fc[2]).reshape(fc[2], fc[1], fc[0])
        sl = [slice(None)] * 3
        sl[2 - d] = 0
        f[tuple(sl)] = 0.0
        sl[2 - d] = counts[d]
        f[tuple(sl)] = 0.0
        faces.append(f.reshape(-1).astype(np.float32))
    tracer = rng.uniform(0.0, 1.0, int(np.prod(counts))).astype(np.float32)
    return faces, tracer


@pytest.mark.parametrize("method", V1, ids=lambda m: m.name)
@pytest.mark.parametrize("with_boundary", [False, True])
def test_forced_steps_match_the_oracle(method, with_boundary):
    counts, spacing, density = (16, 12, 8), (0.25, 0.25, 0.5), 1.5
    faces, tracer = random_state(counts, 17)
    pressure = (1e-10, 1e-12, 1e-8, 5000)
    sim = carrier(counts, spacing, density, method, pressure, limit=1e-3, courant=1.0, faces=faces, tracer=tracer)
    orc = O.Simulation(O.grid(counts, spacing), density, ORACLE_METHOD[method], O.settings(*pressure), 1e-3, 1.0,
                       faces, tracer)
    src = S.SmokeSource((1.0, 0.5, 1.0), (3.0, 2.0, 3.0), 0.5, 0.25)
    forces = [S.BodyForce((0.25, -0.5, 0.125)),
              S.BodyForce((3.0, 0.0, -1.5), S.ForceUnits.FORCE_DENSITY, S.ForceRegion((0.0, 0.0, 0.0), (2.0, 3.0, 4.0)))]
    oforces = [dict(value=f.value, units=f.units,
                    region=None if f.region is None else (f.region.lower, f.region.upper)) for f in forces]
    outward = [[-0.25, 0.25], [0.375, -0.375], [0.0, 0.0]]
    w = workspace(sim) if with_boundary else None
    for step in range(4):
        if with_boundary:
            rb = S.step_with_box_flux(sim, 0.05, src, forces, w,
                                      S.BoxFluxStepBoundary(PrescribedBoxFlux(BoxFluxStamp(1, step), outward)))
            r = rb.step
        else:
            r = S.step_with_forces(sim, 0.05, src, forces)
        src_d = dict(lower=src.lower, upper=src.upper, tracer_rate=src.tracer_rate,
                     vertical_acceleration=src.vertical_acceleration)
        st, orep = orc.step(0.05, src_d, oforces, outward if with_boundary else None)
        assert st == 0
        near(r.dt, orep.dt, 1e-6)
        assert r.generation == orep.generation
        assert r.pressure.iterations == orep.pressure.iterations
        fs, tr = state(sim)
        for d in range(3):
            ulps = np.abs(fs[d].view(np.int32).astype(np.int64) - orc.faces[d].view(np.int32).astype(np.int64))
            assert ulps.max() <= 1, (step, d, ulps.max())
        assert np.max(np.abs(tr - orc.tracer)) <= 1e-6
        near(r.forces.applied_work, orep.force_applied_work, 1e-9)
        near(r.forces.kinetic_energy_after, orep.force_kinetic_after, 1e-9)
        near(r.kinetic_energy, orep.kinetic_energy, 1e-9)
        near(r.tracer_integral, orep.tracer_integral, 1e-9)
        near(r.courant, orep.courant, 1e-6)
        if with_boundary:
            for name in ("kinetic_old", "kinetic_after_advection", "kinetic_after_smoke_force", "kinetic_accepted",
                         "tracer_old_integral"):
                near(getattr(rb.work, name), getattr(orep, name), 1e-9)
            scale = rb.work.kinetic_accepted + rb.work.kinetic_old + 1e-300
            assert abs(rb.work.budget_error) <= 1e-6 * scale


# ------------------------------------------------------------------ the liquid step with a box-flux boundary
def pilot(flow_id=11):
    """The dense3D pilot channel (tests/dense3d_controls_contract.rs:27-75): 3 x 1 x 1
    cells of 1/3 m, carrier density 1000, represented liquid 800 at [0.5, 0, 0],
    a 0.25 m/s x through-flow."""
    from rheon_b200 import liquid as L

    sim = carrier((3, 1, 1), (1.0 / 3.0, 1.0, 1.0), density=1000.0)
    lts = L.LiquidTransportSimulation(sim, 800.0, (2 ** 64 - 1, 0), [0.5, 0.0, 0.0], flow_id=flow_id)
    return sim, lts


def test_liquid_step_with_box_flux_matches_the_oracle():
    from rheon_b200 import liquid as L

    sim, lts = pilot()
    w = workspace(sim)
    inlet = L.LiquidInlet((53, 0), [[0.0, 0.0]] * 3)
    settings = L.LiquidVolumeSettings(1.0, 1e-5)
    og = O.grid((3, 1, 1), (1.0 / 3.0, 1.0, 1.0))
    orc = O.Simulation(og, 1000.0, O.JACOBI_PCG_V1, O.settings(1e-12, 1e-12, 1e-9, 1000), 1e-5, 1.0)
    fraction = np.array([0.5, 0.0, 0.0])
    outward = [[-0.25, 0.25], [0.0, 0.0], [0.0, 0.0]]
    for step in range(1, 6):
        b = S.BoxFluxStepBoundary(PrescribedBoxFlux(BoxFluxStamp(47, step), outward))
        rep, lrep = lts.step_with_box_flux(0.0625, inlet, settings, w, b)
        start = orc.time
        st, orep = orc.step(0.0625, outward=outward)
        assert st == 0 and rep.step.dt == orep.dt == 0.0625
        err, cand, odict = O.liquid_advance(og, 800.0, fraction, orc.faces, start, orep.dt, [[0.0, 0.0]] * 3,
                                            max_outward_courant=1.0, actual_divergence_limit=1e-5, version=step - 1)
        assert err == "Ok"
        fraction = cand
        assert np.array_equal(lts.fraction(), fraction)
        assert lrep.flow == (11, step) and lrep.stamp == (2 ** 64 - 1, step)
        assert lts.time == rep.step.time == orc.time
        fs, _ = state(sim)
        for d in range(3):
            assert np.array_equal(fs[d], orc.faces[d])
        assert lrep.liquid_volume_after == odict["liquid_volume_after"]
        assert lrep.outward_boundary_volume == odict["outward_boundary_volume"]


def test_a_rejected_transport_rejects_the_box_flux_step():
    from rheon_b200 import liquid as L

    sim, lts = pilot()
    w = workspace(sim)
    inlet = L.LiquidInlet((53, 0), [[0.0, 0.0]] * 3)
    b = S.BoxFluxStepBoundary(PrescribedBoxFlux(BoxFluxStamp(47, 0), [[-0.25, 0.25], [0.0, 0.0], [0.0, 0.0]]))
    lts.step_with_box_flux(0.0625, inlet, L.LiquidVolumeSettings(1.0, 1e-5), w, b)
    before, frac, stamp = snapshot(sim), lts.fraction(), lts.stamp
    with pytest.raises(L.LiquidVolumeError) as e:
        lts.step_with_box_flux(0.0625, inlet, L.LiquidVolumeSettings(1e-9, 1e-5), w, b)
    assert e.value.kind == "CourantLimit"
    assert snapshot(sim) == before and np.array_equal(lts.fraction(), frac) and lts.stamp == stamp
    with pytest.raises(S.StepError) as e:
        lts.step_with_box_flux(0.0625, inlet, L.LiquidVolumeSettings(1.0, 1e-5), w, b,
                               cancel=lambda s: s == S.StepStage.LIQUID_BEFORE_COMMIT)
    assert (e.value.kind, e.value.stage) == ("Cancelled", "LiquidBeforeCommit")
    assert snapshot(sim) == before and np.array_equal(lts.fraction(), frac) and lts.stamp == stamp
    rep, lrep = lts.step_with_box_flux(0.0625, inlet, L.LiquidVolumeSettings(1.0, 1e-5), w, b)
    assert rep.step.generation == 2 and lrep.stamp[1] == 2


# ------------------------------------------------------------------ the forced step beside the graph step
def test_forced_steps_publish_their_pressure_and_hand_over_to_the_graph_step():
    """A forced sealed step, then a box-flux step, then (sealed state again) a
    graph step: the carrier's accepted pressure is each step's own, and the
    graph step after a forced step matches the oracle's carrier step."""
    from rheon_b200 import dense3d as D

    counts = (12, 10, 8)
    faces, tracer = random_state(counts, 5)
    pressure = (1e-10, 0.0, MAXF, 5000)
    sim = carrier(counts, density=1.0, pressure=pressure, limit=MAXF, faces=faces, tracer=tracer)
    S.step_with_forces(sim, 0.05, None, [S.BodyForce((0.0, -0.5, 0.0))])
    # the sealed forced step's pressure is the carrier solver's
    assert D.Dense3dFields.from_carrier(sim).pressure != 0
    p_forced = sim.pressure()
    assert p_forced[0] == 0.0 and np.any(p_forced != 0.0)
    w = workspace(sim)
    r = S.step_with_box_flux(sim, 0.05, None, [], w, boundary(0, 0.25))
    assert np.array_equal(sim.pressure(), w.projection.pressure())
    assert r.step.pressure.iterations > 0
    # back to a sealed state: a zero-flux box-flux step stores zero outer faces
    S.step_with_box_flux(sim, 0.05, None, [], w, boundary(0, 0.0, 1))
    fs = state(sim)[0]
    rep = sim.step(R.StepParams(0.05, cfl=0.0))
    prm = O.StepParams(rep.dt, 1.0, O.JACOBI_PCG_V1, O.settings(*pressure), 0.0, 0, 1)
    st, ref, _, orep = O.carrier_step(O.grid(counts), fs, prm)
    assert st == O.OK and rep.pressure.iterations == orep.pressure.iterations
    got = sim.download()
    for d in range(3):
        ulps = np.abs(got[d].view(np.int32).astype(np.int64) - np.asarray(ref[d], np.float32).view(np.int32)
                      .astype(np.int64))
        assert ulps.max() <= 1


def test_a_rejected_forced_step_invalidates_the_exported_pressure():
    from rheon_b200 import dense3d as D

    sim = carrier((6, 5, 4), density=1.0, limit=0.0)
    S.step_with_forces(sim, 0.05, None, [S.BodyForce((0.0, 0.0, 0.0))])  # divergence 0: accepted
    D.Dense3dFields.from_carrier(sim)
    with pytest.raises(S.StepError):
        S.step_with_forces(sim, 0.05, None, [S.BodyForce((0.3, -0.2, 0.1),
                                                        region=S.ForceRegion((0, 0, 0), (3.0, 2.0, 2.0)))])
    with pytest.raises(Exception) as e:
        D.Dense3dFields.from_carrier(sim)
    assert "InvalidState" in str(e.value) or getattr(e.value, "kind", "") == "InvalidState"
