"""The box-flux projection oracle against the reference's known answers.

Each case restates a test of tests/box_flux_contract.rs; the oracle restates
BoxFluxWorkspace::project (src/box_flux.rs:213-397). The device projection is
compared with the oracle in test_gpu_box_flux.py.
"""
import numpy as np
import pytest

import oracle as O
from box_flux_cases import MIXED, dense_pressure, divergence, face_counts, imposed, mixed_old

METHODS = [O.JACOBI_PCG_V1, O.SGS_PCG_V1]


def settings(max_iterations=1000):
    return O.settings(1e-12, 1e-12, 1e-9, max_iterations)


def near(a, b):
    assert abs(a - b) < 2e-11 * max(abs(a), abs(b), 1.0), (a, b)


def mixed():
    c = MIXED
    g = O.grid(c["counts"], c["spacing"], c["origin"])
    return c["counts"], c["spacing"], g, mixed_old(c["counts"]), c["outward"]


@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("axis", [0, 1, 2])
@pytest.mark.parametrize("speed", [-0.25, 0.25])
def test_signed_through_flow_hand_pressure_and_energy(method, axis, speed):
    """box_flux_contract.rs:75-138"""
    counts = [1, 1, 1]
    counts[axis] = 3
    g = O.grid(counts)
    old = [np.zeros(O.face_len(g, d), np.float32) for d in range(3)]
    for d in range(3):  # irrelevant outer provisional values are replaced
        fc = face_counts(counts, d)
        arr = old[d].reshape(fc[2], fc[1], fc[0])
        lo = [slice(None)] * 3
        hi = [slice(None)] * 3
        lo[2 - d] = 0
        hi[2 - d] = counts[d]
        arr[tuple(lo)] = 17.0
        arr[tuple(hi)] = 17.0
    bc = [[0.0, 0.0] for _ in range(3)]
    bc[axis] = [-speed, speed]
    st, out, p, r = O.box_flux_project(g, 2.0, method, old, 0.5, bc, settings(), 1e-5)
    assert st == 0 and r["net_outward_flux"] == 0.0
    for i, pi in enumerate(p):
        near(pi, -4.0 * speed * i)
    for d in range(3):
        assert np.all(out[d] == (np.float32(speed) if d == axis else 0.0))
    assert r["actual_divergence_max"] == 0.0
    near(r["kinetic_before"], 0.0)
    near(r["kinetic_after"], 0.125)
    near(r["correction_energy"], 0.125)
    near(r["boundary_pressure_work"], 0.25)
    near(r["divergence_residual_work"], 0.0)
    near(r["correction_residual_work"], 0.0)
    near(r["budget_error"], 0.0)


@pytest.mark.parametrize("method", METHODS)
def test_unequal_side_areas_match_the_dense_projection(method):
    """box_flux_contract.rs:219-263"""
    counts, spacing, g, old, bc = mixed()
    expected = dense_pressure(counts, spacing, old, bc, 1.5, 0.2)
    st, out, p, r = O.box_flux_project(g, 1.5, method, old, 0.2, bc, settings(), 1e-5)
    assert st == 0
    for a, b in zip(p, expected):
        near(a, b)
    imp = imposed(counts, old, bc)
    for d in range(3):
        fc = face_counts(counts, d)
        for k in range(fc[2]):
            for j in range(fc[1]):
                for i in range(fc[0]):
                    q = [i, j, k]
                    idx = i + fc[0] * (j + fc[1] * k)
                    if q[d] == 0 or q[d] == counts[d]:
                        assert out[d][idx] == imp[d][idx]
                    else:
                        left = list(q)
                        left[d] -= 1
                        c = q[0] + counts[0] * (q[1] + counts[1] * q[2])
                        cl = left[0] + counts[0] * (left[1] + counts[1] * left[2])
                        val = float(old[d][idx]) - 0.2 / (1.5 * spacing[d]) * (expected[c] - expected[cl])
                        assert abs(float(out[d][idx]) - val) < 1e-6
    assert np.max(np.abs(divergence(counts, spacing, out))) == r["actual_divergence_max"]
    near(r["budget_error"], 0.0)


@pytest.mark.parametrize("method", METHODS)
def test_known_net_flux_rejects(method):
    """box_flux_contract.rs:314-329"""
    g = O.grid((3, 1, 1))
    old = [np.full(O.face_len(g, d), 1e20, np.float32) for d in range(3)]
    out0 = [np.full(O.face_len(g, d), -777.0, np.float32) for d in range(3)]
    st, out, _, r = O.box_flux_project(g, 1.0, method, old, 0.1, [[-1.0, 0.0], [0.0, 0.0], [0.0, 0.0]], settings(),
                                       1e-5, out=out0)
    assert st == 28 and r["net_outward_flux"] == -1.0
    assert all(np.array_equal(a, b) for a, b in zip(out, out0))


@pytest.mark.parametrize("method", METHODS)
def test_zero_flux_matches_the_sealed_solve_and_correction(method):
    """box_flux_contract.rs:330-361"""
    counts, spacing, g, old, _ = mixed()
    old = imposed(counts, old, [[0.0, 0.0]] * 3)
    st, rhs = O.build_rhs(g, 1.5, old, 0.2)
    assert st == O.OK
    res = O.solve_rhs(g, 1.5, method, rhs, 0.2, settings())
    assert res.status == O.OK
    st, expected = O.correct(g, 1.5, res.pressure, 0.2, old)
    assert st == O.OK
    st, out, p, r = O.box_flux_project(g, 1.5, method, old, 0.2, [[0.0, 0.0]] * 3, settings(), 1e-5)
    assert st == 0 and np.array_equal(p, res.pressure) and r["iterations"] == res.report.iterations
    for d in range(3):
        assert np.array_equal(out[d].view(np.uint32), np.asarray(expected[d], np.float32).view(np.uint32))
    assert r["kinetic_after"] <= r["kinetic_before"] + 1e-14
    near(r["boundary_pressure_work"], 0.0)
    near(r["budget_error"], 0.0)


def test_divergence_gate_and_iteration_budget():
    """box_flux_contract.rs:418-449"""
    counts, spacing, g, old, bc = mixed()
    out0 = [np.full(O.face_len(g, d), -777.0, np.float32) for d in range(3)]
    st, _, _, r = O.box_flux_project(g, 1.5, O.JACOBI_PCG_V1, old, 0.2, bc, settings(), 0.0, out=out0)
    assert st == 15 and r["actual_divergence_max"] > 0.0
    st, out, _, r = O.box_flux_project(g, 1.5, O.JACOBI_PCG_V1, old, 0.2, bc, settings(max_iterations=0), 1e-5,
                                       out=out0)
    assert st == O.ITERATION_LIMIT and r["iterations"] == 0
    assert all(np.array_equal(a, b) for a, b in zip(out, out0))


@pytest.mark.parametrize("method", METHODS)
def test_singleton_flow(method):
    """box_flux_contract.rs:451-482"""
    g = O.grid((1, 1, 1), (0.5, 1.0, 2.0))
    old = [np.zeros(O.face_len(g, d), np.float32) for d in range(3)]
    st, out, p, r = O.box_flux_project(g, 1.0, method, old, 0.25, [[-0.5, 0.5], [0.0, 0.0], [0.0, 0.0]], settings(),
                                       1e-5)
    assert st == 0 and r["iterations"] == 0 and r["actual_divergence_max"] == 0.0
    assert list(p) == [0.0] and r["kinetic_before"] == 0.0 and r["kinetic_after"] == 0.0
    assert out[0][0] == 0.5 and out[0][1] == 0.5


def test_nonzero_flux_cannot_underflow_out_of_the_gate():
    """box_flux_contract.rs:539-560"""
    g = O.grid((1, 1, 1), (1e100, 1e-150, 1e-150))
    old = [np.zeros(O.face_len(g, d), np.float32) for d in range(3)]
    out0 = [np.full(O.face_len(g, d), -777.0, np.float32) for d in range(3)]
    st, out, _, _ = O.box_flux_project(g, 1e-100, O.JACOBI_PCG_V1, old, 1.0, [[1e-30, 0.0], [0.0, 0.0], [0.0, 0.0]],
                                       settings(), 1e-5, out=out0)
    assert st == 14
    assert all(np.array_equal(a, b) for a, b in zip(out, out0))


def test_shared_numpy_restatement_matches_the_oracle():
    """The numpy correction and divergence used by the device tests reproduce the oracle bit for bit."""
    from box_flux_cases import correct_from_pressure, work_terms
    import math
    counts, spacing = (7, 5, 4), (0.5, 0.25, 0.75)
    g = O.grid(counts, spacing)
    rng = np.random.default_rng(3)
    old = [rng.uniform(-1, 1, O.face_len(g, d)).astype(np.float32) for d in range(3)]
    bc = [[-0.25, 0.25], [0.5, -0.5], [0.0, 0.0]]
    st, out, p, r = O.box_flux_project(g, 1.25, O.JACOBI_PCG_V1, old, 0.1, bc, settings(), 1e-3)
    assert st == 0
    again = correct_from_pressure(counts, spacing, 1.25, old, p, 0.1, bc)
    for d in range(3):
        assert np.array_equal(again[d].view(np.uint32), out[d].view(np.uint32))
    terms, div = work_terms(counts, spacing, 1.25, old, out, p, 0.1, bc)
    assert np.max(np.abs(div)) == r["actual_divergence_max"]
    for name, t in terms.items():
        exact = math.fsum(t)
        scale = math.fsum(np.abs(t)) + 1e-300
        assert abs(r[name] - exact) <= 1e-13 * scale, name
