"""The liquid-volume transport oracle against the reference's known answers.

Each case restates a test of tests/liquid_volume_contract.rs (file:line in the
test name's docstring) with its values; the oracle restates
LiquidVolumeState::advance (src/liquid_volume.rs:520-776). The device
transport is compared with the oracle in test_gpu_liquid.py.
"""
import math

import numpy as np
import pytest

import oracle as O


def fields(g):
    return [np.zeros(O.face_len(g, a), np.float32) for a in range(3)]


def fidx(g, axis, p):
    fc = O.face_counts(g, axis)
    return p[0] + fc[0] * (p[1] + fc[1] * p[2])


def cidx(counts, p):
    return p[0] + counts[0] * (p[1] + counts[1] * p[2])


def test_signed_zero_is_empty_liquid():
    """liquid_volume_contract.rs:40-51"""
    g = O.grid((1, 1, 1))
    v = [np.array([-0.0, 0.0], np.float32) for _ in range(3)]
    err, f, r = O.liquid_advance(g, 1000.0, [-0.0], v, 0.0, 0.5, [[-0.0, 0.0]] * 3)
    assert err == "Ok" and r["liquid_volume_after"] == 0.0 and f[0] == 0.0


@pytest.mark.parametrize("axis", [0, 1, 2])
@pytest.mark.parametrize("speed", [-0.5, 0.5])
def test_upwind_inlet_outlet_hand_volumes(axis, speed):
    """liquid_volume_contract.rs:53-100"""
    counts = [1, 1, 1]
    counts[axis] = 4
    g = O.grid(counts, (1.0, 1.0, 1.0), (2.0, 3.0, 4.0))
    v = fields(g)
    v[axis][:] = speed
    alpha = [[0.0, 0.0] for _ in range(3)]
    alpha[axis] = [0.5, 0.125]
    err, f, r = O.liquid_advance(g, 1000.0, [0.0, 0.25, 0.75, 1.0], v, 0.0, 1.0, alpha)
    assert err == "Ok"
    expected = [0.25, 0.125, 0.5, 0.875] if speed > 0 else [0.125, 0.5, 0.875, 0.5625]
    assert list(f) == expected
    assert r["time"] == 1.0 and r["volume_balance_error"] == 0.0 and r["actual_divergence_max"] == 0.0
    assert r["max_outward_courant"] == 0.5
    if speed > 0:
        assert (r["inward_boundary_volume"], r["outward_boundary_volume"], r["liquid_volume_after"]) == (0.25, 0.5, 1.75)
    else:
        assert (r["inward_boundary_volume"], r["outward_boundary_volume"], r["liquid_volume_after"]) == (0.0625, 0.0,
                                                                                                        2.0625)
    assert r["liquid_mass_after"] == 1000.0 * r["liquid_volume_after"]
    assert (r["dry_cells"], r["mixed_cells"], r["full_cells"]) == (0, 4, 0)


@pytest.mark.parametrize("density", [1.0, 1000.0])
def test_signed_sources_scale_mass_only(density):
    """liquid_volume_contract.rs:101-125"""
    g = O.grid((2, 1, 1))
    err, f, r = O.liquid_advance(g, density, [0.25, 0.75], fields(g), 0.0, 0.5, [[0.0, 0.0]] * 3,
                                 source=[0.25, -0.125])
    assert err == "Ok" and list(f) == [0.375, 0.6875]
    assert r["source_volume"] == 0.0625 and r["liquid_volume_before"] == 1.0 and r["liquid_volume_after"] == 1.0625
    assert r["volume_balance_error"] == 0.0 and r["liquid_mass_after"] == density * 1.0625


def test_closed_anisotropic_circulation():
    """liquid_volume_contract.rs:126-151"""
    g = O.grid((2, 2, 2), (0.5, 1.0, 2.0))
    v = fields(g)
    for z in range(2):
        v[0][fidx(g, 0, (1, 0, z))] = 0.25
        v[0][fidx(g, 0, (1, 1, z))] = -0.25
        v[1][fidx(g, 1, (0, 1, z))] = -0.5
        v[1][fidx(g, 1, (1, 1, z))] = 0.5
    err, f, r = O.liquid_advance(g, 1000.0, [1.0, 0.0, 0.0, 0.0, 0.0, 0.5, 0.0, 0.25], v, 0.0, 0.5, [[1.0, 1.0]] * 3)
    assert err == "Ok"
    assert list(f) == [0.75, 0.25, 0.0, 0.0, 0.0, 0.375, 0.0625, 0.3125]
    assert r["liquid_volume_before"] == 1.75 and r["liquid_volume_after"] == 1.75
    assert r["inward_boundary_volume"] == 0.0 and r["outward_boundary_volume"] == 0.0
    assert r["actual_divergence_max"] == 0.0 and r["volume_balance_error"] == 0.0


def test_oblique_constant_fraction():
    """liquid_volume_contract.rs:152-171"""
    g = O.grid((4, 4, 4), (0.25, 0.5, 1.0))
    v = fields(g)
    for a, speed in enumerate([0.125, 0.25, 0.5]):
        v[a][:] = speed
    err, f, r = O.liquid_advance(g, 1000.0, [0.375] * 64, v, 0.0, 0.5, [[0.375, 0.375]] * 3)
    assert err == "Ok" and np.all(f == 0.375)
    assert r["liquid_volume_before"] == 3.0 and r["liquid_volume_after"] == 3.0
    assert r["inward_boundary_volume"] == 0.5625 and r["outward_boundary_volume"] == 0.5625
    assert r["max_outward_courant"] == 0.75 and r["volume_balance_error"] == 0.0


def test_unsplit_diffusion_of_a_cube():
    """liquid_volume_contract.rs:172-210"""
    g = O.grid((3, 3, 3))
    init = np.zeros(27)
    init[cidx((3, 3, 3), (1, 1, 1))] = 1.0
    v = fields(g)
    for a in range(3):
        v[a][:] = 0.25
    err, f, r = O.liquid_advance(g, 1000.0, init, v, 0.0, 1.0, [[0.0, 0.0]] * 3)
    expected = np.zeros(27)
    for p in [(1, 1, 1), (2, 1, 1), (1, 2, 1), (1, 1, 2)]:
        expected[cidx((3, 3, 3), p)] = 0.25
    assert err == "Ok" and np.array_equal(f, expected)
    assert r["liquid_volume_after"] == 1.0 and r["volume_balance_error"] == 0.0
    error = 0.0
    for z in range(3):
        for y in range(3):
            for x in range(3):
                exact = 1.0
                for i in (x, y, z):
                    exact *= max(min(i + 1.0, 2.25) - max(float(i), 1.25), 0.0)
                error += abs(f[cidx((3, 3, 3), (x, y, z))] - exact)
    assert abs(error - 0.65625) <= 2e-12
    assert (r["full_cells"], r["mixed_cells"]) == (0, 4)


@pytest.mark.parametrize("n,courant", [(16, 0.5), (32, 0.5), (64, 0.5), (64, 0.25)])
def test_translated_slab_matches_the_binomial(n, courant):
    """liquid_volume_contract.rs:219-270"""
    h = 1.0 / n
    g = O.grid((n, 1, 1), (h, 1.0, 1.0))
    init = np.array([1.0 if n // 4 <= i < n // 2 else 0.0 for i in range(n)])
    v = fields(g)
    v[0][:] = 0.25
    dt = courant * h / 0.25
    steps = int(0.5 / dt)
    f, t, max_balance = init.copy(), 0.0, 0.0
    for _ in range(steps):
        err, f, r = O.liquid_advance(g, 1000.0, f, v, t, dt, [[0.0, 0.0]] * 3)
        assert err == "Ok"
        t = r["time"]
        max_balance = max(max_balance, abs(r["volume_balance_error"]))
    for i, value in enumerate(f):
        binomial = sum(math.comb(steps, k) * courant ** k * (1 - courant) ** (steps - k) * init[i - k]
                       for k in range(0, min(steps, i) + 1))
        assert abs(value - binomial) <= 2e-12 * max(abs(value), abs(binomial), 1.0)
    assert max_balance < 1e-14


def test_thin_fractions_are_not_erased():
    """liquid_volume_contract.rs:271-292"""
    g = O.grid((8, 1, 1))
    f = np.zeros(8)
    f[2] = f[4] = 1e-12
    v = fields(g)
    v[0][:] = 0.5
    t = 0.0
    for _ in range(2):
        err, f, r = O.liquid_advance(g, 1000.0, f, v, t, 0.25, [[0.0, 0.0]] * 3)
        assert err == "Ok"
        t = r["time"]
        assert abs(r["liquid_volume_after"] - 2e-12) < 1e-25
        assert abs(r["volume_balance_error"]) <= r["volume_rounding_budget"]
    assert np.all(f[2:7] > 0.0) and abs(f[4] - 0.78125e-12) < 1e-26


def test_courant_divergence_and_bounds_failures():
    """liquid_volume_contract.rs:293-345"""
    g = O.grid((1, 1, 1))
    v = fields(g)
    v[0][:] = 2.0
    err, f, r = O.liquid_advance(g, 1000.0, [0.25], v, 0.0, 1.0, [[0.25, 0.25]] * 3)
    assert err == "CourantLimit" and r["error_actual"] == 2.0 and f is None
    for rate in (1.0, -1.0):
        err, _, _ = O.liquid_advance(g, 1000.0, [0.25], fields(g), 0.0, 1.0, [[0.0, 0.0]] * 3, source=[rate])
        assert err == "FractionBounds"
    assert O.liquid_advance(g, 1000.0, [0.25], fields(g), 0.0, 1.0, [[0.0, 0.0]] * 3)[0] == "Ok"
    g2 = O.grid((2, 1, 1))
    v = fields(g2)
    v[0][1] = 0.25
    err, _, r = O.liquid_advance(g2, 1000.0, [0.25, 0.5], v, 0.0, 1.0, [[0.0, 0.0]] * 3)
    assert err == "DivergenceLimit" and r["error_actual"] == 0.25
    err, f, r = O.liquid_advance(g2, 1000.0, [0.25, 0.5], v, 0.0, 1.0, [[0.0, 0.0]] * 3,
                                 actual_divergence_limit=0.25)
    assert err == "Ok" and r["liquid_volume_after"] == 0.75
    err, _, r = O.liquid_advance(g2, 1000.0, [1.0, 1.0], v, 0.0, 1.0, [[1.0, 1.0]] * 3, actual_divergence_limit=0.25)
    assert err == "FractionBounds" and r["error_actual"] == 1.25


def test_interval_inlet_source_and_settings_validation():
    """src/liquid_volume.rs:84-96, :123-150, :185-190, :485-529"""
    g = O.grid((2, 1, 1))
    v = fields(g)
    ok = [[0.0, 0.0]] * 3
    assert O.liquid_advance(g, 1.0, [0.5, 0.5], v, 0.0, 0.0, ok)[0] == "InvalidTimeStep"
    assert O.liquid_advance(g, 1.0, [0.5, 0.5], v, -1.0, 0.5, ok)[0] == "InvalidTimeStep"
    assert O.liquid_advance(g, 1.0, [0.5, 0.5], v, 1e300, 1e-300, ok)[0] == "TimeResolution"
    bad = [a.copy() for a in v]
    bad[2][0] = np.inf
    assert O.liquid_advance(g, 1.0, [0.5, 0.5], bad, 0.0, 0.5, ok)[0] == "NonFiniteVelocity"
    assert O.liquid_advance(g, 1.0, [0.5, 0.5], v, 0.0, 0.5, [[0.0, 1.5], [0, 0], [0, 0]])[0] == "InvalidInlet"
    assert O.liquid_advance(g, 1.0, [0.5, 0.5], v, 0.0, 0.5, ok, source=[np.nan, 0.0])[0] == "InvalidSource"
    assert O.liquid_advance(g, 1.0, [0.5, 0.5], v, 0.0, 0.5, ok, max_outward_courant=0.0)[0] == "InvalidSettings"
    assert O.liquid_advance(g, 1.0, [0.5, 0.5], v, 0.5, 0.5, ok, state_time=0.0)[0] == "TimeMismatch"
    assert O.liquid_validate_state(g, 0.0, [0.5, 0.5])[0] == "InvalidDensity"
    assert O.liquid_validate_state(g, 1.0, [0.5, 1.5]) == ("InvalidFraction", 1)


# ---- periodic boundary: tests/liquid_volume_periodic_contract.rs

def uniform_fields(g, u):
    return [np.full(O.face_len(g, d), u[d], np.float32) for d in range(3)]


def test_periodic_matches_independent_multiaxis_upwind():
    """liquid_volume_periodic_contract.rs:17-52"""
    g = O.grid((2, 2, 2), (0.5, 0.5, 0.5))
    init = [0.0, 0.25, 0.5, 1.0, 0.75, 0.125, 0.625, 0.875]
    speeds = [0.25, -0.125, 0.0625]
    err, f, r = O.liquid_advance(g, 998.2, init, uniform_fields(g, speeds), 0.0, 0.25, [[0.0, 0.0]] * 3,
                                 actual_divergence_limit=0.0, periodic=True)
    assert err == "Ok"
    for k in range(2):
        for j in range(2):
            for i in range(2):
                p = [i, j, k]
                idx = i + 2 * j + 4 * k
                exact = init[idx]
                for d in range(3):
                    donor = list(p)
                    donor[d] = 1 - p[d]
                    q = donor[0] + 2 * donor[1] + 4 * donor[2]
                    exact += 0.25 * abs(float(np.float32(speeds[d]))) / 0.5 * (init[q] - init[idx])
                assert abs(f[idx] - exact) < 1e-14
    assert r["inward_boundary_volume"] == 0.0 and r["outward_boundary_volume"] == 0.0
    assert abs(r["volume_balance_error"]) < 1e-14


def test_one_cell_periodic_seams_cancel():
    """liquid_volume_periodic_contract.rs:53-68"""
    g = O.grid((1, 1, 1))
    err, f, r = O.liquid_advance(g, 2.0, [0.25], uniform_fields(g, [-0.5, 0.25, -0.125]), 0.0, 0.25,
                                 [[0.0, 0.0]] * 3, source=[0.5], actual_divergence_limit=0.0, periodic=True)
    assert err == "Ok" and list(f) == [0.375]
    assert r["source_volume"] == 0.125 and r["volume_balance_error"] == 0.0
    assert r["inward_boundary_volume"] + r["outward_boundary_volume"] == 0.0


def test_periodic_seam_mismatch_and_courant():
    """liquid_volume_periodic_contract.rs:69-104"""
    g = O.grid((2, 2, 2), (0.5, 0.5, 0.5))
    u = uniform_fields(g, [0.25, 0.0, 0.0])
    u[0][2] = 0.125  # face (2, 0, 0): the upper face of the seam at (0, 0, 0)
    err, _, r = O.liquid_advance(g, 998.2, [0.5] * 8, u, 0.0, 0.25, [[0.0, 0.0]] * 3, actual_divergence_limit=0.0,
                                 periodic=True)
    assert err == "PeriodicVelocityMismatch" and r["error_actual"] == 0.0 and r["error_cell"] == 0
    u[0][:] = 0.25
    err, _, _ = O.liquid_advance(g, 998.2, [0.5] * 8, u, 0.0, 10.0, [[0.0, 0.0]] * 3, actual_divergence_limit=0.0,
                                 periodic=True)
    assert err == "CourantLimit"


def test_box_policy_stays_non_periodic():
    """liquid_volume_periodic_contract.rs:105-121"""
    g = O.grid((1, 1, 1))
    err, f, r = O.liquid_advance(g, 1.0, [0.0], uniform_fields(g, [0.5, 0.0, 0.0]), 0.0, 0.25,
                                 [[1.0, 0.0], [0.0, 0.0], [0.0, 0.0]], actual_divergence_limit=0.0)
    assert err == "Ok" and r["inward_boundary_volume"] == 0.125 and list(f) == [0.125]


@pytest.mark.parametrize("d", [0, 1, 2])
@pytest.mark.parametrize("sign", [-1.0, 1.0])
def test_three_cell_impulse_periodic_donors(d, sign):
    """liquid_volume_periodic_contract.rs:122-156"""
    counts = [1, 1, 1]
    counts[d] = 3
    spacing = [1.0, 1.0, 1.0]
    spacing[d] = 1.0 / 3.0
    g = O.grid(counts, spacing)
    speed = [0.0, 0.0, 0.0]
    speed[d] = sign
    err, f, _ = O.liquid_advance(g, 1.0, [1.0, 0.0, 0.0], uniform_fields(g, speed), 0.0, spacing[d] * 0.5,
                                 [[0.0, 0.0]] * 3, actual_divergence_limit=0.0, periodic=True)
    exact = [0.5, 0.5, 0.0] if sign > 0 else [0.5, 0.0, 0.5]
    assert err == "Ok" and all(abs(a - b) < 1e-14 for a, b in zip(f, exact))
