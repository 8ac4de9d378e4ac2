"""The oracle's step owner with the smoke source, body forces and box-flux
boundary, against the reference's known answers.

Restates tests/simulation_contract.rs, tests/forces_contract.rs and
tests/box_flux_step_contract.rs on orc_sim_step (Simulation::prepare_impl,
src/simulation.rs:812-1403). The device step is compared with it in
test_gpu_sim_step.py.
"""
import math

import numpy as np
import pytest

import oracle as O

METHODS = [O.JACOBI_PCG_V1, O.SGS_PCG_V1]
INVALID_SOURCE, INVALID_FORCE, TIME_RESOLUTION = 1, 2, 3
MAXF = 1.7976931348623157e308


def near(a, b, tol=2e-10):
    assert abs(a - b) < tol * max(abs(a), abs(b), 1.0), (a, b)


def snapshot(s):
    return (tuple(np.concatenate([f.view(np.uint32) for f in s.faces] + [s.tracer.view(np.uint32)])), s.time,
            s.generation)


# ------------------------------------------------------------------ simulation_contract.rs
def sim_config():
    return dict(pressure=O.settings(1e-10, 1e-12, 1e-8, 1000), actual_divergence_limit=1e-5, max_courant=1.0)


def smoke():
    return dict(lower=(0.25, 0.125, 0.25), upper=(0.75, 0.375, 0.75), tracer_rate=1.0, vertical_acceleration=0.5)


def eight(method=O.JACOBI_PCG_V1, **kw):
    c = dict(sim_config(), **kw)
    return O.Simulation(O.grid((8, 8, 8), (0.125,) * 3), 1.0, method, c["pressure"], c["actual_divergence_limit"],
                        c["max_courant"])


def test_localized_smoke_is_nontrivial_and_divergence_checked():
    """simulation_contract.rs:54-86"""
    s = eight()
    for _ in range(6):
        st, r = s.step(0.02, smoke())
        assert st == 0 and r.tracer_integral > 0.0 and r.kinetic_energy > 0.0
        div = np.zeros(512)
        assert O.lib().orc_divergence_f32(C_grid(s), *[O._ptr(f) for f in s.faces], O._ptr(div)) == 0
        assert r.actual_divergence_max == np.max(np.abs(div)) <= 1e-5
        assert np.all(np.isfinite(s.tracer)) and np.all((s.tracer >= 0) & (s.tracer <= 1))


def C_grid(s):
    import ctypes
    return ctypes.byref(s.g)


def test_exhaustion_and_invalid_source_are_transactional():
    """simulation_contract.rs:113-128"""
    s = eight(pressure=O.settings(1e-10, 1e-12, 1e-8, 0))
    before = snapshot(s)
    st, _ = s.step(0.02, smoke())
    assert st == O.ITERATION_LIMIT and snapshot(s) == before
    bad = dict(smoke(), tracer_rate=float("nan"))
    st, r = s.step(0.02, bad)
    assert (st, r.error) == (29, INVALID_SOURCE) and snapshot(s) == before


def test_single_cell_saturating_source():
    """simulation_contract.rs:154-168"""
    c = sim_config()
    s = O.Simulation(O.grid((1, 1, 1)), 1.0, O.JACOBI_PCG_V1, c["pressure"], 1e-5, 1.0)
    st, r = s.step(0.25, dict(lower=(0, 0, 0), upper=(1, 1, 1), tracer_rate=10.0, vertical_acceleration=0.0))
    assert st == 0 and r.actual_divergence_max == 0.0 and list(s.tracer) == [1.0] and r.pressure.iterations == 0


def test_time_step_policy_for_large_forcing():
    """simulation_contract.rs:169-177"""
    s = eight()
    st, r = s.step(1.0, dict(smoke(), vertical_acceleration=8.0))
    assert st == 0 and r.dt < 1.0 and r.courant <= 1.0


def test_stored_divergence_rejection_preserves_state():
    """simulation_contract.rs:200-211"""
    s = eight(actual_divergence_limit=0.0)
    st, _ = s.step(0.02)
    assert st == 0
    before = snapshot(s)
    st, r = s.step(0.02, smoke())
    assert st == O.DIVERGENCE_LIMIT and r.error_actual > 0.0 and snapshot(s) == before


# ------------------------------------------------------------------ forces_contract.rs
def force(value, units=0, region=None):
    return dict(value=value, units=units, region=region)


def cycle_force():
    return force((2.0, 0.0, 0.0), region=((0.0, 0.0, 0.0), (2.0, 1.0, 1.0)))


def cycle_sim(method, density):
    return O.Simulation(O.grid((2, 2, 1)), density, method, O.settings(1e-11, 1e-12, 1e-9, 1000), 1e-6, 1.0)


def face_value(s, axis, p):
    fc = O.face_counts(s.g, axis)
    return float(s.faces[axis][p[0] + fc[0] * (p[1] + fc[1] * p[2])])


@pytest.mark.parametrize("method", METHODS)
def test_signed_uniform_forces_hand_work_and_hydrostatic_rest(method):
    """forces_contract.rs:59-86"""
    for d, a in enumerate([0.25, -0.5, 1.5]):
        counts, spacing = (3, 4, 2), (0.5, 0.25, 1.0)
        g = O.grid(counts, spacing, (-1.0, 2.0, -2.0))
        faces = (counts[d] - 1) * counts[(d + 1) % 3] * counts[(d + 2) % 3]
        volume = 0.5 * 0.25 * 1.0
        expected = 0.5 * 2.0 * volume * faces * (0.125 * a) ** 2
        value = [0.0, 0.0, 0.0]
        value[d] = a
        s = O.Simulation(g, 2.0, method, O.settings(1e-11, 1e-12, 1e-9, 1000), 1e-6, 1.0)
        st, r = s.step(0.125, forces=[force(value)])
        assert st == 0 and r.dt == 0.125 and r.has_forces
        assert r.force_kinetic_before == 0.0
        assert r.force_kinetic_after == expected and r.force_applied_work == expected
        assert r.actual_divergence_max < 1e-6 and r.kinetic_energy < 1e-16


@pytest.mark.parametrize("method", METHODS)
def test_localized_force_projects_to_the_four_edge_cycle(method):
    """forces_contract.rs:87-117"""
    s = cycle_sim(method, 1.0)
    st, r = s.step(0.25, forces=[cycle_force()])
    assert st == 0
    for axis, p, expected in [(0, (1, 0, 0), 0.125), (0, (1, 1, 0), -0.125), (1, (0, 1, 0), -0.125),
                              (1, (1, 1, 0), 0.125)]:
        assert abs(face_value(s, axis, p) - expected) < 1e-8
    assert r.force_applied_work == 0.125 and abs(r.kinetic_energy - 0.03125) < 1e-8
    assert np.all(s.tracer == 0.0) and np.all(s.faces[2] == 0.0)


@pytest.mark.parametrize("method", METHODS)
def test_smoke_force_precedes_the_external_stage(method):
    """forces_contract.rs:118-141"""
    s = cycle_sim(method, 1.0)
    src = dict(lower=(0, 0, 0), upper=(1.0, 2.0, 1.0), tracer_rate=0.0, vertical_acceleration=2.0)
    st, r = s.step(0.25, src, [cycle_force()])
    assert st == 0
    assert (r.force_kinetic_before, r.force_kinetic_after, r.force_applied_work) == (0.125, 0.25, 0.125)
    assert r.kinetic_energy < 1e-16 and np.all(s.tracer == 0.0)


@pytest.mark.parametrize("method", METHODS)
def test_force_density_matches_acceleration_bits(method):
    """forces_contract.rs:142-164"""
    for density in (0.5, 2.0, 8.0):
        a, f = cycle_sim(method, density), cycle_sim(method, density)
        fd = dict(cycle_force(), units=1, value=(2.0 * density, 0.0, 0.0))
        for _ in range(3):
            sa, ra = a.step(0.125, forces=[cycle_force()])
            sf, rf = f.step(0.125, forces=[fd])
            assert sa == sf == 0
            assert (ra.force_kinetic_before, ra.force_kinetic_after, ra.force_applied_work) == \
                (rf.force_kinetic_before, rf.force_kinetic_after, rf.force_applied_work)
            assert snapshot(a) == snapshot(f)


def test_support_excludes_upper_planes_and_walls():
    """forces_contract.rs:165-198"""
    s = cycle_sim(O.JACOBI_PCG_V1, 1.0)
    f = dict(cycle_force(), region=((0.0, 0.0, 0.0), (1.0, 1.0, 1.0)))
    st, r = s.step(0.25, forces=[f])
    assert st == 0 and r.force_applied_work == 0.0 and r.kinetic_energy == 0.0


@pytest.mark.parametrize("method", METHODS)
def test_overlapping_forces_add_and_the_budget_covers_each_axis(method):
    """forces_contract.rs:199-223"""
    s = cycle_sim(method, 2.0)
    st, r = s.step(0.125, forces=[cycle_force(), dict(cycle_force(), value=(-2.0, 0.0, 0.0))])
    assert st == 0 and r.kinetic_energy == 0.0 and r.force_applied_work == 0.0
    st, r = s.step(1.0, forces=[force((16.0, -16.0, 16.0), units=1)])
    assert st == 0 and r.dt == math.sqrt(0.5 / 24.0) and r.courant <= 1.0


def test_invalid_or_unrepresentable_forces():
    """forces_contract.rs:273-333"""
    s = cycle_sim(O.JACOBI_PCG_V1, 0.5)
    assert s.step(0.125, forces=[cycle_force()])[0] == 0
    before = snapshot(s)
    for bad in [force((float("nan"), 0, 0)), force((0, float("inf"), 0)),
                dict(cycle_force(), region=((0, 0, 0), (3.0, 3.0, 3.0))),
                dict(cycle_force(), region=((0, 0, 0), (0.0, 0.0, 0.0)))]:
        st, r = s.step(0.125, forces=[bad])
        assert (st, r.error) == (29, INVALID_FORCE) and snapshot(s) == before
    st, r = s.step(0.125, forces=[force((MAXF, 0, 0))])
    assert (st, r.error) == (29, TIME_RESOLUTION) and snapshot(s) == before
    st, r = s.step(0.125, forces=[force((MAXF, 0, 0), units=1)])
    assert st == O.ARITHMETIC_FAILURE and snapshot(s) == before
    fresh = cycle_sim(O.JACOBI_PCG_V1, 0.5)
    before = snapshot(fresh)
    st, _ = fresh.step(0.125, forces=[force((MAXF, 0, 0))])
    assert st == O.ARITHMETIC_FAILURE and snapshot(fresh) == before


# ------------------------------------------------------------------ box_flux_step_contract.rs
def step_config():
    return dict(density=2.0, pressure=O.settings(1e-12, 1e-12, 1e-9, 1000), limit=1e-5, courant=1.0)


def box_sim(counts, spacing=(1.0, 1.0, 1.0), method=O.JACOBI_PCG_V1, **kw):
    c = dict(step_config(), **kw)
    return O.Simulation(O.grid(counts, spacing), c["density"], method, c["pressure"], c["limit"], c["courant"])


def through(axis, speed):
    bc = [[0.0, 0.0] for _ in range(3)]
    bc[axis] = [-speed, speed]
    return bc


@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("axis", [0, 1, 2])
@pytest.mark.parametrize("speed", [-0.25, 0.25])
def test_signed_end_boundary_hand_flow_and_work(method, axis, speed):
    """box_flux_step_contract.rs:76-126"""
    counts = [1, 1, 1]
    counts[axis] = 3
    s = box_sim(counts, method=method)
    for step in (1, 2, 3):
        st, r = s.step(0.5, outward=through(axis, speed))
        assert st == 0 and r.generation == step and r.time == 0.5 * step
        for d in range(3):
            assert np.all(s.faces[d] == (np.float32(speed) if d == axis else 0.0))
        assert r.actual_divergence_max == 0.0
        near(r.kinetic_accepted, 0.125)
        near(r.kinetic_energy, 0.125)
        near(r.budget_error, 0.0)
        assert r.boundary_volume_imbalance == 0.0
        if step == 1:
            near(r.kinetic_old, 0.0)
            near(r.projection.boundary_pressure_work, 0.25)
            near(r.projection.correction_energy, 0.125)
        else:
            near(r.kinetic_old, 0.125)
            near(r.advection_change, 0.0)
            near(r.projection.boundary_pressure_work, 0.0)


@pytest.mark.parametrize("method", METHODS)
def test_boundary_speed_controls_dt_and_courant(method):
    """box_flux_step_contract.rs:127-141"""
    s = box_sim((3, 1, 1), (0.5, 1.0, 1.0), method)
    st, r = s.step(20.0, outward=through(0, 2.0))
    assert st == 0 and r.dt == 0.125 and r.courant == 0.5 and s.time == 0.125


@pytest.mark.parametrize("method", METHODS)
def test_changing_boundary_versions(method):
    """box_flux_step_contract.rs:142-166"""
    s = box_sim((3, 1, 1), method=method)
    assert s.step(0.5, outward=through(0, 0.25))[0] == 0
    st, r = s.step(0.5, outward=through(0, -0.25))
    assert st == 0 and np.all(s.faces[0] == -0.25)
    near(r.kinetic_old, 0.125)
    near(r.budget_error, 0.0)


@pytest.mark.parametrize("method", METHODS)
def test_external_and_smoke_terms_join_the_ledger(method):
    """box_flux_step_contract.rs:167-212"""
    s = box_sim((2, 2, 1), method=method)
    src = dict(lower=(0, 0, 0), upper=(2.0, 2.0, 1.0), tracer_rate=0.5, vertical_acceleration=0.5)
    f = force((1.0, -0.25, 0.0))
    st, r = s.step(0.25, src, [f], through(0, 0.25))
    assert st == 0
    near(r.smoke_force_work, 0.03125)
    near(r.external_force_work, 0.1015625)
    near(r.kinetic_before_projection, 0.1328125)
    near(r.kinetic_accepted, 0.125)
    near(r.force_applied_work, r.external_force_work)
    near(r.tracer_source_change, 0.5)
    near(r.tracer_transport_change, 0.0)
    near(r.budget_error, 0.0)
    p = r.projection
    near(r.kinetic_accepted - r.kinetic_old + p.correction_energy,
         r.advection_change + r.smoke_force_work + r.external_force_work + p.boundary_pressure_work
         + p.divergence_residual_work + p.correction_residual_work)


@pytest.mark.parametrize("method", METHODS)
def test_clamped_appearance_transport_and_saturated_source(method):
    """box_flux_step_contract.rs:213-240"""
    s = box_sim((3, 1, 1), method=method)
    src = dict(lower=(0, 0, 0), upper=(1.0, 1.0, 1.0), tracer_rate=10.0, vertical_acceleration=0.0)
    assert s.step(0.5, src, outward=through(0, 0.0))[0] == 0
    assert list(s.tracer) == [1.0, 0.0, 0.0]
    st, r = s.step(0.5, outward=through(0, 0.25))
    assert st == 0 and list(s.tracer) == [1.0, 0.125, 0.0]
    near(r.tracer_old_integral, 1.0)
    near(r.tracer_transport_change, 0.125)
    near(r.tracer_source_change, 0.0)
    assert r.boundary_volume_imbalance == 0.0


@pytest.mark.parametrize("method", METHODS)
def test_incompatible_flux_late_overflow_and_exhaustion_never_publish(method):
    """box_flux_step_contract.rs:319-374"""
    s = box_sim((3, 1, 1), method=method)
    before = snapshot(s)
    st, _ = s.step(0.5, outward=[[0.0, 0.25], [0.0, 0.0], [0.0, 0.0]])
    assert st == 28 and snapshot(s) == before
    src = dict(lower=(0, 0, 0), upper=(3.0, 1.0, 1.0), tracer_rate=MAXF, vertical_acceleration=0.0)
    st, _ = s.step(4.0, src, outward=through(0, 0.0))
    assert st == O.ARITHMETIC_FAILURE and snapshot(s) == before
    assert s.step(0.5, outward=through(0, 0.25))[0] == 0
    ex = box_sim((3, 1, 1), method=method, pressure=O.settings(1e-12, 1e-12, 1e-9, 0))
    before = snapshot(ex)
    st, _ = ex.step(0.5, outward=through(0, 0.25))
    assert st == O.ITERATION_LIMIT and snapshot(ex) == before
    assert ex.step(0.5, outward=through(0, 0.0))[0] == 0


@pytest.mark.parametrize("method", METHODS)
def test_zero_boundary_agrees_with_the_sealed_forced_step(method):
    """box_flux_step_contract.rs:456-503"""
    counts, spacing = (3, 2, 2), (0.5, 1.0, 2.0)
    closed, zero = box_sim(counts, spacing, method), box_sim(counts, spacing, method)
    src = dict(lower=(0, 0, 0), upper=(1.5, 2.0, 4.0), tracer_rate=0.25, vertical_acceleration=0.5)
    f = force((0.5, -0.125, 0.25), region=((0, 0, 0), (1.0, 1.0, 2.0)))
    for _ in range(3):
        sa, a = closed.step(0.125, src, [f])
        sb, b = zero.step(0.125, src, [f], through(0, 0.0))
        assert sa == sb == 0
        assert snapshot(closed) == snapshot(zero)
        assert a.pressure.iterations == b.pressure.iterations
        assert a.actual_divergence_max == b.actual_divergence_max
        near(b.budget_error, 0.0)


@pytest.mark.parametrize("method", METHODS)
def test_stored_divergence_rejection_after_projection(method):
    """box_flux_step_contract.rs:514-549"""
    s = box_sim((3, 2, 2), (0.5, 1.0, 2.0), method, limit=0.0)
    before = snapshot(s)
    f = force((0.1, -0.13, 0.2), region=((0, 0, 0), (1.0, 1.0, 2.0)))
    st, r = s.step(0.125, forces=[f], outward=through(0, 0.375))
    assert st == O.DIVERGENCE_LIMIT and r.error_actual > r.error_limit == 0.0
    assert snapshot(s) == before
    assert s.step(0.125, outward=through(0, 0.0))[0] == 0


@pytest.mark.parametrize("method", METHODS)
def test_balanced_volume_flux_does_not_certify_tracer_mass(method):
    """box_flux_step_contract.rs:551-593"""
    s = box_sim((3, 2, 1), method=method)
    seed = dict(lower=(0, 0, 0), upper=(1.0, 2.0, 1.0), tracer_rate=1.0, vertical_acceleration=0.0)
    assert s.step(0.5, seed, outward=through(0, 0.0))[0] == 0
    f = force((0.0, 0.5, 0.0), region=((0, 0, 0), (1.0, 2.0, 1.0)))
    st, r = s.step(0.25, forces=[f], outward=through(0, 0.25))
    assert st == 0 and r.boundary_volume_imbalance == 0.0 and r.tracer_source_change == 0.0
    assert np.all((s.tracer >= 0.0) & (s.tracer <= 0.5))
    assert abs(r.tracer_transport_change - 0.0625) > 1e-6
    near(r.budget_error, 0.0)
