"""Pins the oracle to the reference's own known-answer tests.

Each test restates one hand-derived fixture from the Rheon test suite (cited by
file:line within the Rheon project) and checks the oracle against it. These run
on CPU only; they are what makes the oracle a trustworthy checker for the GPU
parity tests.
"""
import math

import numpy as np
import pytest

import oracle as O


def S(rel=1e-11, abs_=1e-12, div=1e-9, it=1000):
    return O.settings(rel, abs_, div, it)


# ------------------------------------------------------------ operator_contract.rs
def test_three_cell_hand_calculation_and_residual_identity(orc):
    # tests/operator_contract.rs:3-27
    g = O.grid([3, 1, 1])
    x = np.array([0.0, 2.0, -1.0, 0.0], np.float32)
    y = np.zeros(6, np.float32)
    z = np.zeros(6, np.float32)
    st, rhs = O.build_rhs(g, 1.0, [x, y, z], 0.5)
    assert st == O.OK
    assert rhs.tolist() == [-4.0, 6.0, -2.0]
    st, product = O.apply_full(g, 1.0, [0.0, 4.0, 2.0])
    assert st == O.OK and product.tolist() == rhs.tolist()
    st, (ox, oy, oz) = O.correct(g, 1.0, [0.0, 4.0, 2.0], 0.5, [x, y, z])
    assert st == O.OK and ox.tolist() == [0.0] * 4
    st, div = O.divergence(g, [ox, oy, oz])
    assert st == O.OK and div.tolist() == [0.0] * 3


def test_independent_rectangular_dense_operator(orc):
    # tests/operator_contract.rs:29-56
    g = O.grid([3, 2, 1], [0.5, 2.0, 3.0])
    edges = [(0, 1, 6.0), (1, 2, 6.0), (3, 4, 6.0), (4, 5, 6.0), (0, 3, 0.375), (1, 4, 0.375), (2, 5, 0.375)]
    p = [0.7, -0.3, 1.4, 2.0, -1.0, 0.9]
    expected = [0.0] * 6
    for a, b, w in edges:
        v = w * (p[a] - p[b])
        expected[a] += v
        expected[b] -= v
    st, actual = O.apply_full(g, 2.0, p)
    assert st == O.OK
    assert np.max(np.abs(actual - expected)) < 1e-12
    st, const = O.apply_full(g, 2.0, [3.0] * 6)
    assert const.tolist() == [0.0] * 6


def test_integrated_rhs_matches_independent_physical_divergence(orc):
    # tests/operator_contract.rs:58-73
    g = O.grid([2, 1, 1], [0.25, 0.5, 2.0])
    x = np.array([0.0, 0.75, 0.0], np.float32)
    y = np.zeros(4, np.float32)
    z = np.zeros(4, np.float32)
    _, rhs = O.build_rhs(g, 1.0, [x, y, z], 0.1)
    _, div = O.divergence(g, [x, y, z])
    assert div.tolist() == [3.0, -3.0]
    assert rhs.tolist() == [-7.5, 7.5]
    vol = 0.25 * 0.5 * 2.0
    for i in range(2):
        assert abs(div[i] + 0.1 * rhs[i] / vol) < 1e-12


def test_all_six_faces_of_single_cell_are_walls(orc):
    # tests/operator_contract.rs:75-91
    g = O.grid([1, 1, 1])
    zero = np.zeros(2, np.float32)
    st, rhs = O.build_rhs(g, 1.0, [zero, zero, zero], 1.0)
    assert st == O.OK and rhs.tolist() == [0.0]
    st, out = O.apply_full(g, 1.0, [5.0])
    assert out.tolist() == [0.0]
    nonzero = np.array([0.0, 1.0], np.float32)
    st, _ = O.build_rhs(g, 1.0, [nonzero, zero, zero], 1.0)
    assert st == O.NONZERO_WALL_VELOCITY


def test_nonfinite_fields_are_rejected(orc):
    # tests/operator_contract.rs:93-112
    g = O.grid([2, 2, 2])
    st, _ = O.apply_full(g, 1.0, [math.inf] * 8)
    assert st == O.NONFINITE_INPUT
    st, _ = O.apply_full(g, float("nan"), [0.0] * 8)
    assert st == O.INVALID_ARGUMENT


def test_cached_boundary_diagonals_match_original_order_for_every_row(orc):
    # src/operator.rs:898-924: cached 64-entry table equals the ordered sum.
    for counts in ([5, 4, 3], [1, 7, 2], [3, 1, 1], [1, 1, 1]):
        h = [0.13, 0.27, 0.41]
        g = O.grid(counts, h, [-1.0, 2.0, 0.3])
        rho = 1.37
        area = [h[1] * h[2], h[0] * h[2], h[0] * h[1]]
        w = [area[d] * (1.0 / (rho * h[d])) for d in range(3)]
        for zc in range(counts[2]):
            for yc in range(counts[1]):
                for xc in range(counts[0]):
                    p = [xc, yc, zc]
                    original = 0.0
                    for d in range(3):
                        if p[d] > 0:
                            original += w[d]
                        if p[d] + 1 < counts[d]:
                            original += w[d]
                    assert O.diagonal(g, rho, p) == original


# ------------------------------------------------------------ pressure_contract.rs
def test_solves_hand_chain_and_reports_full_residual(orc):
    # tests/pressure_contract.rs:13-25
    g = O.grid([3, 1, 1])
    r = O.solve_rhs(g, 1.0, O.JACOBI_PCG_V1, [-4.0, 6.0, -2.0], 0.5, S())
    assert r.status == O.OK
    assert abs(r.pressure[1] - 4.0) < 1e-10
    assert abs(r.pressure[2] - 2.0) < 1e-10
    assert r.pressure[0] == 0.0
    assert r.report.true_residual_max < 1e-10


def test_single_cell_zero_rhs_returns_without_iteration(orc):
    # tests/pressure_contract.rs:27-37
    r = O.solve_rhs(O.grid([1, 1, 1]), 1.0, O.JACOBI_PCG_V1, [0.0], 1.0, S())
    assert r.status == O.OK
    assert r.report.iterations == 0 and r.report.true_residual_max == 0.0


def test_incompatible_rhs_is_not_mean_shifted(orc):
    # tests/pressure_contract.rs:39-48
    r = O.solve_rhs(O.grid([2, 1, 1]), 1.0, O.JACOBI_PCG_V1, [1.0, 0.0], 1.0, S())
    assert r.status == O.INCOMPATIBLE_RHS


def test_eliminated_gauge_row_participates_in_physical_stopping(orc):
    # tests/pressure_contract.rs:50-72
    r = O.solve_rhs(O.grid([4, 1, 1]), 1.0, O.JACOBI_PCG_V1, [-0.003, 0.001, 0.001, 0.001], 1.0,
                    S(1.0, 1.0, 0.0015, 0))
    assert r.status == O.ITERATION_LIMIT and r.report.iterations == 0


def _manufactured(counts, spacing, rho, fn):
    g = O.grid(counts, spacing)
    n = O.cell_len(g)
    exact = np.array([fn(i) for i in range(n)])
    _, rhs = O.apply_full(g, rho, exact)
    return g, exact, rhs


@pytest.mark.parametrize("method", [O.JACOBI_PCG_V1, O.SGS_PCG_V1])
def test_manufactured_three_dimensional_pressure_recovers_modulo_gauge(orc, method):
    # tests/pressure_contract.rs:74-88
    g, exact, rhs = _manufactured([5, 4, 3], [0.2, 0.25, 0.3], 1.3, lambda i: math.sin(i * 0.7))
    r = O.solve_rhs(g, 1.3, method, rhs, 0.02, S())
    assert r.status == O.OK
    assert np.max(np.abs(r.pressure - (exact - exact[0]))) < 1e-8
    assert r.report.predicted_divergence_max <= 1e-9


def test_tighter_divergence_gate_keeps_conjugate_gradient_progress(orc):
    # tests/pressure_contract.rs:91-157 (independent product restated here)
    counts, spacing, rho = [5, 4, 3], [0.2, 0.25, 0.3], 1.3
    g = O.grid(counts, spacing)
    n = O.cell_len(g)
    exact = np.array([((i * 17) % 31) / 31.0 for i in range(n)])
    vol = spacing[0] * spacing[1] * spacing[2]
    strides = [1, counts[0], counts[0] * counts[1]]

    def product(p):
        out = np.zeros(n)
        for row in range(n):
            c = [row % counts[0], (row // counts[0]) % counts[1], row // strides[2]]
            value = 0.0
            for d in range(3):
                w = vol / (rho * spacing[d] * spacing[d])
                if c[d] > 0:
                    value += w * (p[row] - p[row - strides[d]])
                if c[d] + 1 < counts[d]:
                    value += w * (p[row] - p[row + strides[d]])
            out[row] = value
        return out

    rhs = product(exact)
    lim = S(1e-3, 1e-12, 1e-9, 120)
    r = O.solve_rhs(g, rho, O.JACOBI_PCG_V1, rhs, 0.02, lim)
    assert r.status == O.OK
    res = rhs - product(r.pressure)
    assert np.sqrt(np.sum(res * res)) <= max(1e-12, 1e-3 * np.sqrt(np.sum(rhs * rhs)))
    assert np.max(np.abs(res)) * 0.02 / vol <= 1e-9
    assert r.report.predicted_divergence_max <= 1e-9
    assert r.pressure[0] == 0.0
    assert np.max(np.abs(r.pressure - exact)) < 1e-8


def test_iteration_exhaustion_is_explicit(orc):
    # tests/pressure_contract.rs:159-174
    r = O.solve_rhs(O.grid([3, 1, 1]), 1.0, O.JACOBI_PCG_V1, [-4.0, 6.0, -2.0], 0.5, S(it=1))
    assert r.status == O.ITERATION_LIMIT and r.report.iterations == 1


def lcg_faces(g, seed=0x12345678):
    """Fields of tests/pressure_contract.rs:195-215 (LCG seeded, interior faces)."""
    fields = []
    mask = (1 << 64) - 1
    counts = [int(g.counts[d]) for d in range(3)]
    for d in range(3):
        shape = O.face_counts(g, d)
        f = np.zeros(shape[0] * shape[1] * shape[2], np.float32)
        for k in range(shape[2]):
            for j in range(shape[1]):
                for i in range(shape[0]):
                    c = [i, j, k]
                    if 0 < c[d] < counts[d]:
                        seed = (seed * 6364136223846793005 + 1) & mask
                        value = (seed >> 40) / float(1 << 24) - 0.5
                        f[i + shape[0] * (j + shape[1] * k)] = np.float32(value)
        fields.append(f)
    return fields


def test_random_three_dimensional_projection_checks_actual_f32_divergence(orc):
    # tests/pressure_contract.rs:195-235
    g = O.grid([8, 7, 6], [0.2, 0.3, 0.4])
    faces = lcg_faces(g)
    st, rhs = O.build_rhs(g, 1.0, faces, 0.02)
    assert st == O.OK
    r = O.solve_rhs(g, 1.0, O.JACOBI_PCG_V1, rhs, 0.02, S())
    assert r.status == O.OK and r.report.predicted_divergence_max < 1e-9
    st, out = O.correct(g, 1.0, r.pressure, 0.02, faces)
    assert st == O.OK
    _, div = O.divergence(g, out)
    assert np.max(np.abs(div)) < 1e-5
    before = sum(float(np.sum(f.astype(np.float64) ** 2)) for f in faces)
    after = sum(float(np.sum(f.astype(np.float64) ** 2)) for f in out)
    assert after <= before + 1e-6


def test_a_rectangular_cycle_retains_circulation(orc):
    # tests/pressure_contract.rs:238-262
    g = O.grid([2, 2, 1])
    x = np.array([0, 1, 0, 0, -1, 0], np.float32)
    y = np.array([0, 0, -1, 1, 0, 0], np.float32)
    z = np.zeros(8, np.float32)
    _, rhs = O.build_rhs(g, 1.0, [x, y, z], 0.1)
    r = O.solve_rhs(g, 1.0, O.JACOBI_PCG_V1, rhs, 0.1, S())
    assert r.status == O.OK and r.report.iterations == 0
    _, out = O.correct(g, 1.0, r.pressure, 0.1, [x, y, z])
    assert out[0].tolist() == x.tolist() and out[1].tolist() == y.tolist()


# ------------------------------------------------------------ pressure.rs / sgs.rs inline
def test_sgs_matches_independently_assembled_triangular_system(orc):
    # src/pressure.rs:824-842
    g = O.grid([2, 2, 1])
    st, z, rz = O.precondition(g, 1.0, O.SGS_PCG_V1, [-12.0, 2.0, 4.0, 6.0])
    assert st == O.OK
    assert z.tolist() == [0.0, 3.25, 4.25, 4.5]
    assert rz == 50.5


def test_sgs_triangular_equations_hold(orc):
    # src/sgs.rs:293-361 (serial sweep; the residual check of (D-L)D^-1(D-U)z = r)
    counts, h, rho = [17, 10, 9], [0.5, 0.75, 1.25], 1.3
    g = O.grid(counts, h, [2.0, -1.0, 3.0])
    n = O.cell_len(g)
    residual = np.array([0.0 if i == 0 else ((i * 17) % 113) / 113.0 - 0.5 for i in range(n)])
    st, z, _ = O.precondition(g, rho, O.SGS_PCG_V1, residual)
    assert st == O.OK and z[0] == 0.0 and np.all(np.isfinite(z))
    area = [h[1] * h[2], h[0] * h[2], h[0] * h[1]]
    w = [area[d] * (1.0 / (rho * h[d])) for d in range(3)]
    strides = [1, counts[0], counts[0] * counts[1]]
    yv = np.zeros(n)
    coords = [[row % counts[0], (row // counts[0]) % counts[1], row // strides[2]] for row in range(n)]
    for row in range(1, n):
        p = coords[row]
        upper = sum(w[d] * z[row + strides[d]] for d in range(3) if p[d] + 1 < counts[d])
        yv[row] = z[row] - upper / O.diagonal(g, rho, p)
    for row in range(1, n):
        p = coords[row]
        lower = sum(w[d] * yv[row - strides[d]] for d in range(3) if p[d] > 0)
        assert abs(O.diagonal(g, rho, p) * yv[row] - lower - residual[row]) < 1e-12


# ------------------------------------------------------------ implementation_contract.rs
@pytest.mark.parametrize("method", [O.JACOBI_PCG_V1, O.SGS_PCG_V1])
@pytest.mark.parametrize("counts", [[1, 1, 1], [3, 1, 1], [5, 4, 3]])
def test_all_methods_recover_anisotropic_manufactured_pressure(orc, method, counts):
    # tests/implementation_contract.rs:57-84
    g, exact, rhs = _manufactured(counts, [0.2, 0.35, 0.7], 1.3, lambda i: math.sin(i * 0.7))
    r = O.solve_rhs(g, 1.3, method, rhs, 0.02, S())
    assert r.status == O.OK
    assert r.report.predicted_divergence_max <= 1e-9
    assert np.max(np.abs(r.pressure - exact + exact[0])) < 1e-8
    r = O.solve_rhs(g, 1.3, method, np.ones_like(rhs), 0.02, S())
    if len(rhs) > 0:
        assert r.status == O.INCOMPATIBLE_RHS


# ------------------------------------------------------------ sampling_contract.rs
def _face_field(g, axis, f):
    dims = O.face_counts(g, axis)
    out = []
    h = [g.spacing[d] for d in range(3)]
    o = [g.origin[d] for d in range(3)]
    for zc in range(dims[2]):
        for yc in range(dims[1]):
            for xc in range(dims[0]):
                c = [xc, yc, zc]
                pos = [o[d] + (c[d] + (0.0 if d == axis else 0.5)) * h[d] for d in range(3)]
                out.append(f(pos))
    return np.array(out, np.float32)


def test_component_offsets_reproduce_affine_fields(orc):
    # tests/sampling_contract.rs:14-26
    g = O.grid([4, 5, 6], [0.5, 0.25, 0.125], [-1.0, -0.5, 0.0])
    f = lambda p: p[0] + 2.0 * p[1] - 3.0 * p[2] + 2.0
    for axis in range(3):
        values = _face_field(g, axis, f)
        p = [-0.2, 0.2, 0.4]
        st, s = O.sample(g, axis, values, p)
        assert st == O.OK and abs(s - f(p)) < 1e-12


def test_convex_bounds_and_singleton_axes_hold(orc):
    # tests/sampling_contract.rs:27-38
    g = O.grid([2, 1, 1])
    vals = np.array([-2.0, 8.0], np.float32)
    assert O.sample(g, 3, vals, [1.0, 0.5, 0.5]) == (O.OK, 3.0)
    big = np.finfo(np.float64).max
    assert O.sample(g, 3, vals, [-big] * 3) == (O.OK, -2.0)
    assert O.sample(g, 3, vals, [big] * 3) == (O.OK, 8.0)
    assert O.sample(g, 3, vals, [float("nan")] * 3)[0] == O.NONFINITE_POSITION


def test_midpoint_backtrace_matches_constant_translation(orc):
    # tests/sampling_contract.rs:39-52
    g = O.grid([8, 8, 8])
    u = _face_field(g, 0, lambda p: 1.0)
    v = _face_field(g, 1, lambda p: -2.0)
    w = _face_field(g, 2, lambda p: 0.5)
    assert O.backtrace(g, u, v, w, [4.0] * 3, 0.5) == (O.OK, [3.5, 5.0, 3.75])
    assert O.backtrace(g, u, v, w, [0.1, 7.9, 0.1], 0.5) == (O.OK, [0.0, 8.0, 0.0])
    assert O.backtrace(g, u, v, w, [4.0] * 3, 0.0)[0] == O.INVALID_TIME_STEP


def test_midpoint_rotation_matches_independent_polynomial(orc):
    # tests/sampling_contract.rs:53-64
    g = O.grid([8, 8, 1], origin=[-4.0, -4.0, 0.0])
    u = _face_field(g, 0, lambda p: -p[1])
    v = _face_field(g, 1, lambda p: p[0])
    w = _face_field(g, 2, lambda p: 0.0)
    dt = 0.1
    st, a = O.backtrace(g, u, v, w, [1.0, 0.0, 0.5], dt)
    assert st == O.OK
    assert abs(a[0] - (1.0 - dt * dt / 2.0)) < 1e-14
    assert abs(a[1] + dt) < 1e-14


# ------------------------------------------------------------ advection_contract.rs
def test_constant_translation_advects_an_interior_pulse_one_cell(orc):
    # tests/advection_contract.rs:69-80
    g = O.grid([8, 1, 1])
    u = np.ones(9, np.float32)
    v = np.zeros(16, np.float32)
    w = np.zeros(16, np.float32)
    old = np.array([0, 0, 1, 0, 0, 0, 0, 0], np.float32)
    st, out = O.advect_tracer(g, old, [u, v, w], 1.0)
    assert st == O.OK and out.tolist() == [0, 0, 0, 1, 0, 0, 0, 0]


def test_rest_state_is_preserved_on_degenerate_grid(orc):
    # tests/advection_contract.rs:81-96
    g = O.grid([1, 1, 1], [0.5, 0.25, 0.125])
    old = np.zeros(2, np.float32)
    st, (u, v, w) = O.advect_velocity(g, [old, old, old], 0.1)
    assert st == O.OK and [u.tolist(), v.tolist(), w.tolist()] == [[0.0, 0.0]] * 3
    st, tr = O.advect_tracer(g, np.array([0.37], np.float32), [u, v, w], 0.1)
    assert tr.tolist() == [np.float32(0.37)]


def test_tracer_matches_composed_rk2_samples_bitwise(orc):
    # tests/advection_contract.rs:7-41: every cell equals sample(backtrace(cell)).
    g = O.grid([9, 7, 5], [0.07, 0.11, 0.19], [-2.0, 4.0, 0.3])
    vel = [np.array([0.8 * math.sin(i * 0.017 + d) for i in range(O.face_len(g, d))], np.float32)
           for d in range(3)]
    n = [int(g.counts[d]) for d in range(3)]
    old = np.zeros(O.cell_len(g), np.float32)
    old[n[0] * (3 + n[1] * 2)] = 1.0
    old[n[0] - 1 + n[0] * (4 + n[1] * 3)] = -0.5
    for dt in (0.01, 0.5, 3.0):
        st, out = O.advect_tracer(g, old, vel, dt)
        assert st == O.OK
        for zc in range(n[2]):
            for yc in range(n[1]):
                for xc in range(n[0]):
                    pos = [g.origin[d] + ([xc, yc, zc][d] + 0.5) * g.spacing[d] for d in range(3)]
                    _, dep = O.backtrace(g, *vel, pos, dt)
                    _, s = O.sample(g, 3, old, dep)
                    assert out[xc + n[0] * (yc + n[1] * zc)] == np.float32(s)


# ------------------------------------------------------------ solver_provider_contract.rs
def test_exact_candidate_qualifies_and_bad_ones_are_rejected(orc):
    # tests/solver_provider_contract.rs:64-96 and :97-169
    g = O.grid([4, 3, 2], [0.25, 0.3, 0.4])
    pressure = np.array([math.sin(i * 0.3) for i in range(24)])
    _, rhs = O.apply_full(g, 1.25, pressure)
    s = S(1e-10, 1e-12, 1e-8, 1000)
    gauged = pressure - pressure[0]
    st, rep = O.qualify_pressure(g, 1.25, rhs, 0.01, s, gauged)
    assert st == O.OK
    st, _ = O.qualify_pressure(g, 1.25, rhs, 0.01, s, np.full(24, math.inf))
    assert st == O.NONFINITE_OUTPUT
    st, _ = O.qualify_pressure(g, 1.25, rhs, 0.01, s, pressure + 1.0)
    assert st == O.NONZERO_GAUGE
    st, _ = O.qualify_pressure(g, 1.25, rhs, 0.01, s, np.zeros(24))
    assert st == O.QUALITY_GATE


# ------------------------------------------------------------ pressure_initial_guess.rs
# Seeded solves (solve_rhs_with_initial_pressure, feature
# "accepted-pressure-warm-start"), both methods.
METHODS = (O.JACOBI_PCG_V1, O.SGS_PCG_V1)


@pytest.mark.parametrize("method", METHODS)
def test_exact_and_approximate_guesses_recover_independent_chain(orc, method):
    # tests/pressure_initial_guess.rs:17-52
    g = O.grid([3, 1, 1])
    r = O.solve_rhs(g, 1.0, method, [-4.0, 6.0, -2.0], 0.5, S(), initial=[0.0, 4.0, 2.0])
    assert r.status == O.OK and r.report.iterations == 0 and r.report.true_residual_l2 == 0.0
    r = O.solve_rhs(g, 1.0, method, [-4.0, 6.0, -2.0], 0.125, S(), initial=[0.0, 3.0, -1.0])
    assert r.status == O.OK and r.report.iterations > 0
    assert np.max(np.abs(r.pressure - [0.0, 4.0, 2.0])) < 1e-10


def test_zero_rhs_still_checks_seed_and_current_rhs_threshold(orc):
    # tests/pressure_initial_guess.rs:54-83
    g = O.grid([3, 1, 1])
    r = O.solve_rhs(g, 1.0, O.JACOBI_PCG_V1, [0.0] * 3, 1.0, O.settings(1.0, 0.0, 100.0, 0), initial=[0.0, 4.0, 2.0])
    assert r.status == O.ITERATION_LIMIT and r.report.iterations == 0
    r = O.solve_rhs(g, 1.0, O.JACOBI_PCG_V1, [0.0] * 3, 1.0, S(), initial=[0.0, 4.0, 2.0])
    assert r.status == O.OK and r.report.iterations > 0
    assert np.all(np.abs(r.pressure) < 1e-10)


def test_full_gauge_row_and_compatibility_are_not_hidden_by_guess(orc):
    # tests/pressure_initial_guess.rs:85-118
    g = O.grid([4, 1, 1])
    r = O.solve_rhs(g, 1.0, O.JACOBI_PCG_V1, [-0.003, 0.001, 0.001, 0.001], 1.0, O.settings(1.0, 1.0, 0.0015, 0),
                    initial=[0.0] * 4)
    assert r.status == O.ITERATION_LIMIT
    r = O.solve_rhs(g, 1.0, O.JACOBI_PCG_V1, [1.0, 0.0, 0.0, 0.0], 1.0, S(), initial=[0.0] * 4)
    assert r.status == O.INCOMPATIBLE_RHS


def test_invalid_guesses_are_rejected(orc):
    # tests/pressure_initial_guess.rs:120-172 (the seed validation part)
    g = O.grid([3, 1, 1])
    rhs = [-4.0, 6.0, -2.0]
    assert O.solve_rhs(g, 1.0, 0, rhs, 0.5, S(), initial=[0.0, 1.0]).status == O.LENGTH_MISMATCH
    assert O.solve_rhs(g, 1.0, 0, rhs, 0.5, S(), initial=[0.0, math.nan, 0.0]).status == O.NONFINITE_INPUT
    assert O.solve_rhs(g, 1.0, 0, rhs, 0.5, S(), initial=[0.0, math.inf, 0.0]).status == O.NONFINITE_INPUT
    assert O.solve_rhs(g, 1.0, 0, rhs, 0.5, S(), initial=[1.0, 4.0, 2.0]).status == O.INVALID_INITIAL_PRESSURE
    seeded = O.solve_rhs(g, 1.0, 0, rhs, 0.5, S(), initial=[0.0, 3.0, -1.0])
    again = O.solve_rhs(g, 1.0, 0, rhs, 0.5, S(), initial=[0.0, 3.0, -1.0])
    assert seeded.report.iterations == again.report.iterations
    assert np.array_equal(seeded.pressure, again.pressure)


@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("seeded", [False, True])
def test_neumann_cosine_refines_at_second_order_for_both_initializations(orc, method, seeded):
    # tests/pressure_initial_guess.rs:175-218
    previous = None
    for n in (8, 16, 32, 64):
        h = 1.0 / n
        g = O.grid([n, 1, 1], [h, 1.0, 1.0])
        x = (np.arange(n) + 0.5) * h
        cosine = np.cos(math.pi * x)
        rhs = h * math.pi * math.pi * cosine
        seed = 0.75 * (cosine - cosine[0])
        r = O.solve_rhs(g, 1.0, method, rhs, 0.125, S(), initial=seed if seeded else None)
        assert r.status == O.OK
        eigen = 4.0 * math.sin(math.pi * h / 2.0) ** 2 / (h * h)
        continuum = cosine - cosine[0]
        discrete = math.pi * math.pi / eigen * continuum
        assert np.max(np.abs(r.pressure - discrete)) < 1e-8
        error = np.max(np.abs(r.pressure - continuum))
        if previous is not None:
            assert 3.8 <= previous / error <= 4.2
        previous = error


@pytest.mark.parametrize("method", METHODS)
def test_seeded_chain_retains_full_gauge_acceptance(orc, method):
    # tests/pressure_initial_guess.rs:220-253
    n = 64
    g = O.grid([n, 1, 1])
    seed = np.array([i * (2 * n - 1 - i) * 0.1e-5 for i in range(n)])
    s = O.settings(0.0, 1e-4, 1e-4, 100)
    r = O.solve_rhs(g, 1.0, method, np.zeros(n), 1.0, s, initial=seed)
    assert r.status == O.OK and r.report.iterations > 0
    assert r.report.true_residual_l2 <= 1e-4
    p = r.pressure
    squared = p[1] * p[1]
    for i in range(1, n):
        res = p[i] - p[i - 1] if i == n - 1 else 2.0 * p[i] - p[i - 1] - p[i + 1]
        squared += res * res
    assert math.sqrt(squared) <= 1e-4
