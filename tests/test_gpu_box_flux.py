"""Box-flux projection on the device against the oracle, through the C ABI.

The oracle restates BoxFluxWorkspace::project (src/box_flux.rs:213-397); the
cases follow tests/box_flux_contract.rs. Tolerances:
- output faces, the divergence maximum and the side components: bit for bit
  against the numpy restatement applied to the device's own pressure (the
  correction rounds every product as the reference does);
- pressure: 1e-12 relative to the oracle's for the two reference methods
  (per-iteration parity of the device solve), the contract's 2e-11 `near` for
  the hand and dense-solve cases;
- energy terms: the device adds the reference's rounded terms (a few per
  thread in double, the partials in double-double), so each is within 1e-13
  of the sum of the terms' magnitudes of the exactly rounded sum (math.fsum). Against the oracle's serial sums:
  1e-9 of that magnitude for the energies and the boundary work, 1e-2 for the
  two residual works, whose terms sit at the f32 rounding level.
"""
import math

import numpy as np
import pytest

import oracle as O
import rheon_b200 as R
from box_flux_cases import (MIXED, balanced_outward, component, correct_from_pressure, dense_pressure, divergence,
                            face_counts, imposed, mixed_old, work_terms)
from rheon_b200.box_flux import (BoxFluxError, BoxFluxSettings, BoxFluxStage, BoxFluxStamp, BoxFluxWorkspace,
                                 PrescribedBoxFlux)

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

V1 = [R.PressureImplementation.JACOBI_PCG_V1, R.PressureImplementation.SGS_PCG_V1]
ALL = V1 + [R.PressureImplementation.RBSGS_PCG, R.PressureImplementation.MG_MIXED]
ORACLE_METHOD = {R.PressureImplementation.JACOBI_PCG_V1: O.JACOBI_PCG_V1,
                 R.PressureImplementation.SGS_PCG_V1: O.SGS_PCG_V1}
WORK = ("kinetic_before", "kinetic_after", "correction_energy", "boundary_pressure_work", "divergence_residual_work",
        "correction_residual_work")


@pytest.fixture(scope="module", autouse=True)
def _device():
    if not torch.cuda.is_available() or R.device_count() == 0:
        pytest.skip("no B200")
    yield
    torch.cuda.synchronize()


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def settings(max_iterations=1000, rel=1e-12, limit=1e-5, div=1e-9):
    return BoxFluxSettings(R.PressureSettings(rel, 1e-12, div, max_iterations), limit)


def flux(outward):
    return PrescribedBoxFlux(BoxFluxStamp(37, 8), outward)


def near(a, b):
    assert abs(a - b) < 2e-11 * max(abs(a), abs(b), 1.0), (a, b)


def fields(g, value):
    return [torch.full((g.face_len(d),), value, dtype=torch.float32, device="cuda") for d in range(3)]


def project(w, old, dt, outward, s, out=None, cancelled=None):
    g = w.grid
    out = fields(g, -777.0) if out is None else out
    r = w.project([dev(o) for o in old], dt, flux(outward), s, out, cancelled)
    return r, [host(o) for o in out]


def check_against_restatement(g, density, old, dt, outward, r, out, p):
    """Output bits, divergence maximum and work terms from the device's own pressure."""
    counts, spacing = tuple(g.counts), tuple(g.spacing)
    again = correct_from_pressure(counts, spacing, density, old, p, dt, outward)
    for d in range(3):
        assert np.array_equal(out[d].view(np.uint32), again[d].view(np.uint32)), d
    terms, div = work_terms(counts, spacing, density, old, out, p, dt, outward)
    assert r.actual_divergence_max == np.max(np.abs(div))
    for name in WORK:
        t = terms[name]
        exact = math.fsum(t)
        scale = math.fsum(np.abs(t)) + 1e-300
        assert abs(getattr(r.work, name) - exact) <= 1e-13 * scale, (name, getattr(r.work, name), exact)
    w = r.work
    be = w.kinetic_after - w.kinetic_before + w.correction_energy - (
        w.boundary_pressure_work + w.divergence_residual_work + w.correction_residual_work)
    assert w.budget_error == be


# ------------------------------------------------------------------ hand and dense cases
@pytest.mark.parametrize("method", ALL, ids=lambda m: m.name)
@pytest.mark.parametrize("axis", [0, 1, 2])
@pytest.mark.parametrize("speed", [-0.25, 0.25])
def test_signed_through_flow_hand_pressure_and_energy(method, axis, speed):
    """box_flux_contract.rs:75-138"""
    counts = [1, 1, 1]
    counts[axis] = 3
    g = R.GridGeometry(counts)
    old = [np.zeros(g.face_len(d), np.float32) for d in range(3)]
    for d in range(3):
        fc = face_counts(counts, d)
        arr = old[d].reshape(fc[2], fc[1], fc[0])
        sl = [slice(None)] * 3
        sl[2 - d] = 0
        arr[tuple(sl)] = 17.0
        sl[2 - d] = counts[d]
        arr[tuple(sl)] = 17.0
    bc = [[0.0, 0.0] for _ in range(3)]
    bc[axis] = [-speed, speed]
    w = BoxFluxWorkspace(g, 2.0, 4096, method)
    r, out = project(w, old, 0.5, bc, settings())
    assert r.boundary == BoxFluxStamp(37, 8) and r.net_outward_flux == 0.0
    for i, pi in enumerate(w.pressure()):
        near(pi, -4.0 * speed * i)
    for d in range(3):
        assert np.all(out[d] == (np.float32(speed) if d == axis else 0.0))
    assert r.actual_divergence_max == 0.0
    near(r.work.kinetic_before, 0.0)
    near(r.work.kinetic_after, 0.125)
    near(r.work.correction_energy, 0.125)
    near(r.work.boundary_pressure_work, 0.25)
    near(r.work.divergence_residual_work, 0.0)
    near(r.work.correction_residual_work, 0.0)
    near(r.work.budget_error, 0.0)


@pytest.mark.parametrize("method", ALL, ids=lambda m: m.name)
def test_unequal_side_areas_match_the_dense_projection(method):
    """box_flux_contract.rs:219-263"""
    c = MIXED
    g = R.GridGeometry(c["counts"], c["spacing"], c["origin"])
    old = mixed_old(c["counts"])
    expected = dense_pressure(c["counts"], c["spacing"], old, c["outward"], c["density"], c["dt"])
    w = BoxFluxWorkspace(g, c["density"], 4096, method)
    r, out = project(w, old, c["dt"], c["outward"], settings())
    p = w.pressure()
    for a, b in zip(p, expected):
        near(a, b)
    check_against_restatement(g, c["density"], old, c["dt"], c["outward"], r, out, p)
    near(r.work.budget_error, 0.0)


# ------------------------------------------------------------------ parity with the oracle
CASES = [
    ((3, 2, 1), (0.5, 1.0, 2.0), 1.5, 0.2),
    ((17, 10, 9), (0.5, 0.75, 1.25), 1.0, 0.05),
    ((40, 33, 9), (0.07, 0.11, 0.19), 998.0, 0.01),
    ((64, 40, 24), (0.1, 0.12, 0.15), 1.2, 0.02),  # the persistent Jacobi-PCG kernel
    ((32, 32, 32), (0.25, 0.25, 0.25), 1.0, 0.1),
]


@pytest.mark.parametrize("method", V1, ids=lambda m: m.name)
@pytest.mark.parametrize("counts, spacing, density, dt", CASES, ids=str)
def test_projection_matches_the_oracle(method, counts, spacing, density, dt):
    g = R.GridGeometry(counts, spacing)
    rng = np.random.default_rng(sum(counts))
    old = [rng.uniform(-1, 1, g.face_len(d)).astype(np.float32) for d in range(3)]
    bc = balanced_outward(counts, spacing)
    s = settings(rel=1e-10, limit=1.0, div=1e-3)
    ps = s.pressure
    st, oout, op, orep = O.box_flux_project(O.grid(counts, spacing), density, ORACLE_METHOD[method], old, dt, bc,
                                            O.settings(ps.relative_residual, ps.absolute_residual,
                                                       ps.divergence_limit, ps.max_iterations), 1.0)
    assert st == 0
    w = BoxFluxWorkspace(g, density, 1 << 34, method)
    r, out = project(w, old, dt, bc, s)
    p = w.pressure()
    assert r.pressure.iterations == orep["iterations"]
    nb = np.linalg.norm(op)
    assert np.linalg.norm(p - op) <= 1e-12 * max(nb, 1.0)
    assert r.net_outward_flux == orep["net_outward_flux"]
    assert r.flux_rounding_budget == orep["flux_rounding_budget"]
    check_against_restatement(g, density, old, dt, bc, r, out, p)
    # against the oracle's own output: the same bits wherever the pressures round alike
    for d in range(3):
        ulps = np.abs(out[d].view(np.int32).astype(np.int64) - oout[d].view(np.int32).astype(np.int64))
        assert ulps.max() <= 1, d
    # The oracle adds serially; its pressure and a rare output bit differ. The
    # energies and the boundary work move by about the pressure's 1e-12; the
    # two residual works are sums of rounding-level terms, where one output
    # bit changes a term by its own size.
    terms, _ = work_terms(counts, spacing, density, old, out, p, dt, bc)
    for name in WORK:
        a, b = getattr(r.work, name), orep[name]
        scale = math.fsum(np.abs(terms[name])) + 1e-300
        tol = 1e-2 if name in ("divergence_residual_work", "correction_residual_work") else 1e-9
        assert abs(a - b) <= tol * scale, (name, a, b)


@pytest.mark.parametrize("method", ALL, ids=lambda m: m.name)
def test_native_methods_and_a_large_box(method):
    """Every device method, 96 x 64 x 48 (RBSGS and multigrid: the device's own
    methods, judged by the stored field's divergence and the restatement)."""
    counts, spacing, density, dt = (96, 64, 48), (1 / 96, 1 / 64, 1 / 48), 1.0, 0.01
    g = R.GridGeometry(counts, spacing)
    rng = np.random.default_rng(7)
    old = [rng.uniform(-1, 1, g.face_len(d)).astype(np.float32) for d in range(3)]
    bc = balanced_outward(counts, spacing)
    w = BoxFluxWorkspace(g, density, 1 << 36, method)
    r, out = project(w, old, dt, bc, settings(5000, rel=1e-10, limit=1e-2, div=1e-3))
    check_against_restatement(g, density, old, dt, bc, r, out, w.pressure())
    assert r.actual_divergence_max < 1e-2
    scale = r.work.kinetic_before + r.work.kinetic_after + r.work.correction_energy
    assert abs(r.work.budget_error) <= 1e-6 * scale


def test_host_arrays_match_the_device_path():
    counts, spacing = (17, 10, 9), (0.5, 0.75, 1.25)
    g = R.GridGeometry(counts, spacing)
    rng = np.random.default_rng(4)
    old = [rng.uniform(-1, 1, g.face_len(d)).astype(np.float32) for d in range(3)]
    bc = balanced_outward(counts, spacing)
    w = BoxFluxWorkspace(g, 1.0, 1 << 30)
    s = settings(rel=1e-10, limit=1.0, div=1e-3)
    r1, out1 = project(w, old, 0.05, bc, s)
    out2 = [np.full(g.face_len(d), -777.0, np.float32) for d in range(3)]
    r2 = w.project(old, 0.05, flux(bc), s, out2)
    for d in range(3):
        assert np.array_equal(out1[d].view(np.uint32), out2[d].view(np.uint32))
    assert r1.work == r2.work and r1.pressure.iterations == r2.pressure.iterations


# ------------------------------------------------------------------ contract cases
@pytest.mark.parametrize("method", V1, ids=lambda m: m.name)
def test_known_net_flux_rejects(method):
    """box_flux_contract.rs:314-329"""
    g = R.GridGeometry([3, 1, 1])
    old = [np.full(g.face_len(d), 1e20, np.float32) for d in range(3)]
    w = BoxFluxWorkspace(g, 1.0, 4096, method)
    out = fields(g, -777.0)
    with pytest.raises(BoxFluxError) as e:
        w.project([dev(o) for o in old], 0.1, flux([[-1.0, 0.0], [0.0, 0.0], [0.0, 0.0]]), settings(), out)
    assert e.value.kind == "IncompatibleFlux" and e.value.net == -1.0
    assert all(bool(torch.all(o == -777.0)) for o in out)


@pytest.mark.parametrize("method", V1, ids=lambda m: m.name)
def test_zero_flux_matches_the_sealed_solve_and_correction(method):
    """box_flux_contract.rs:330-361: the workspace's pressure and the stored bits
    equal a sealed pressure workspace's solve followed by the f32 correction."""
    c = MIXED
    g = R.GridGeometry(c["counts"], c["spacing"], c["origin"])
    old = imposed(c["counts"], mixed_old(c["counts"]), [[0.0, 0.0]] * 3)
    op = R.PressureOperator(g, c["density"])
    faces = [dev(o) for o in old]
    rhs = torch.empty(g.cell_len(), dtype=torch.float64, device="cuda")
    op.build_rhs(faces, c["dt"], rhs)
    ws = R.PressureWorkspace(g, 1 << 20, method, density=c["density"])
    rep = ws.solve_rhs(op, rhs, c["dt"], settings().pressure)
    expected = [f.clone() for f in faces]
    op.correct_candidate_in_place(dev(ws.pressure()), c["dt"], expected)
    w = BoxFluxWorkspace(g, c["density"], 4096, method)
    r, out = project(w, old, c["dt"], [[0.0, 0.0]] * 3, settings())
    assert np.array_equal(w.pressure(), ws.pressure()) and r.pressure.iterations == rep.iterations
    for d in range(3):
        assert np.array_equal(out[d].view(np.uint32), host(expected[d]).view(np.uint32))
    assert r.work.kinetic_after <= r.work.kinetic_before + 1e-14
    near(r.work.boundary_pressure_work, 0.0)
    near(r.work.budget_error, 0.0)


@pytest.mark.parametrize("method", V1, ids=lambda m: m.name)
@pytest.mark.parametrize("stage", [BoxFluxStage.BEFORE_SOLVE, BoxFluxStage.PRESSURE_ITERATION,
                                   BoxFluxStage.CORRECTION_SLICE, BoxFluxStage.BEFORE_ACCEPTANCE])
def test_cancellation_partial_output_and_retry(method, stage):
    """box_flux_contract.rs:362-417"""
    c = MIXED
    g = R.GridGeometry(c["counts"], c["spacing"], c["origin"])
    old = mixed_old(c["counts"])
    saved = [o.copy() for o in old]
    w = BoxFluxWorkspace(g, c["density"], 4096, method)
    slices = [0]

    def cancelled(s):
        if s == BoxFluxStage.CORRECTION_SLICE:
            slices[0] += 1
        return s == stage and (stage != BoxFluxStage.CORRECTION_SLICE or slices[0] == 2)

    out = fields(g, -777.0)
    with pytest.raises(BoxFluxError) as e:
        w.project([dev(o) for o in old], c["dt"], flux(c["outward"]), settings(), out, cancelled)
    if stage == BoxFluxStage.PRESSURE_ITERATION:
        assert (e.value.kind, e.value.inner) == ("Pressure", "Cancelled")
    else:
        assert e.value.kind == "Cancelled" and e.value.stage == stage
    untouched = all(bool(torch.all(o == -777.0)) for o in out)
    assert untouched == (stage in (BoxFluxStage.BEFORE_SOLVE, BoxFluxStage.PRESSURE_ITERATION))
    assert all(np.array_equal(a, b) for a, b in zip(old, saved))
    r = w.project([dev(o) for o in old], c["dt"], flux(c["outward"]), settings(), out)
    fresh = BoxFluxWorkspace(g, c["density"], 4096, method)
    r2, expected = project(fresh, old, c["dt"], c["outward"], settings())
    for d in range(3):
        assert np.array_equal(host(out[d]), expected[d])
    assert np.array_equal(w.pressure(), fresh.pressure())
    assert r.pressure.iterations == r2.pressure.iterations


def test_correction_slices_are_asked_as_often_as_in_the_reference():
    """CorrectionSlice is asked once per face slice: nz + nz + (nz + 1)."""
    counts = (6, 5, 4)
    g = R.GridGeometry(counts)
    old = [np.zeros(g.face_len(d), np.float32) for d in range(3)]
    seen = []
    w = BoxFluxWorkspace(g, 1.0, 1 << 20)
    w.project([dev(o) for o in old], 0.1, flux([[-0.5, 0.5], [0.0, 0.0], [0.0, 0.0]]), settings(),
              fields(g, 0.0), lambda s: seen.append(s) or False)
    assert seen[0] == BoxFluxStage.BEFORE_SOLVE and seen[-1] == BoxFluxStage.BEFORE_ACCEPTANCE
    assert seen.count(BoxFluxStage.CORRECTION_SLICE) == 3 * counts[2] + 1


@pytest.mark.parametrize("method", V1, ids=lambda m: m.name)
def test_divergence_gate_after_solver_acceptance(method):
    """box_flux_contract.rs:418-432"""
    c = MIXED
    g = R.GridGeometry(c["counts"], c["spacing"], c["origin"])
    old = mixed_old(c["counts"])
    w = BoxFluxWorkspace(g, c["density"], 4096, method)
    with pytest.raises(BoxFluxError) as e:
        project(w, old, c["dt"], c["outward"], settings(limit=0.0))
    assert e.value.kind == "DivergenceLimit" and e.value.actual > 0.0 and e.value.limit == 0.0
    project(w, old, c["dt"], c["outward"], settings())


def test_iteration_budget_precedes_any_output_write():
    """box_flux_contract.rs:433-450"""
    c = MIXED
    g = R.GridGeometry(c["counts"], c["spacing"], c["origin"])
    w = BoxFluxWorkspace(g, c["density"], 4096)
    out = fields(g, -777.0)
    with pytest.raises(BoxFluxError) as e:
        w.project([dev(o) for o in mixed_old(c["counts"])], c["dt"], flux(c["outward"]), settings(0), out)
    assert (e.value.kind, e.value.inner, e.value.iterations) == ("Pressure", "IterationLimit", 0)
    assert all(bool(torch.all(o == -777.0)) for o in out)


@pytest.mark.parametrize("method", V1, ids=lambda m: m.name)
def test_singleton_flow_and_exact_capacity(method):
    """box_flux_contract.rs:451-482"""
    g = R.GridGeometry([1, 1, 1], [0.5, 1.0, 2.0])
    w = BoxFluxWorkspace(g, 1.0, 56, method)
    assert w.allocated_bytes() == 56
    r, out = project(w, [np.zeros(g.face_len(d), np.float32) for d in range(3)], 0.25,
                     [[-0.5, 0.5], [0.0, 0.0], [0.0, 0.0]], settings())
    assert r.pressure.iterations == 0 and r.actual_divergence_max == 0.0
    assert list(w.pressure()) == [0.0]
    assert r.work.kinetic_before == 0.0 and r.work.kinetic_after == 0.0
    assert out[0][0] == 0.5 and out[0][1] == 0.5


def test_invalid_inputs_reject_before_output_mutation():
    """box_flux_contract.rs:483-538"""
    g = R.GridGeometry([2, 1, 1])
    w = BoxFluxWorkspace(g, 1.0, 4096)
    old = [np.zeros(g.face_len(d), np.float32) for d in range(3)]
    bc = [[0.0, 0.0]] * 3
    out = fields(g, -777.0)

    def rejects(kind, inner, *args, o=None):
        target = out if o is None else o
        before = [host(t).copy() for t in target]
        with pytest.raises(BoxFluxError) as e:
            w.project(*args, target)
        assert (e.value.kind, e.value.inner) == (kind, inner)
        for a, t in zip(before, target):
            assert np.array_equal(a, host(t))

    rejects("Operator", "InvalidTimeStep", [dev(o) for o in old], 0.0, flux(bc), settings())
    bad = [o.copy() for o in old]
    bad[0][0] = np.nan
    rejects("Operator", "NonFiniteInput", [dev(o) for o in bad], 0.1, flux(bc), settings())
    rejects("InvalidSettings", None, [dev(o) for o in old], 0.1, flux(bc), settings(limit=float("nan")))
    short = fields(g, -777.0)
    short[2] = short[2][:-1].contiguous()
    rejects("Operator", "LengthMismatch", [dev(o) for o in old], 0.1, flux(bc), settings(), o=short)
    # the values of an earlier axis are checked before a later axis' length
    bad2 = [dev(bad[0]), dev(old[1]), dev(old[2][:-1])]
    rejects("Operator", "NonFiniteInput", bad2, 0.1, flux(bc), settings())


def test_nonzero_flux_cannot_underflow_out_of_the_gate():
    """box_flux_contract.rs:539-560"""
    g = R.GridGeometry([1, 1, 1], [1e100, 1e-150, 1e-150])
    w = BoxFluxWorkspace(g, 1e-100, 4096)
    out = fields(g, -777.0)
    with pytest.raises(BoxFluxError) as e:
        w.project([dev(np.zeros(g.face_len(d), np.float32)) for d in range(3)], 1.0,
                  flux([[1e-30, 0.0], [0.0, 0.0], [0.0, 0.0]]), settings(), out)
    assert e.value.kind == "ArithmeticFailure"
    assert all(bool(torch.all(o == -777.0)) for o in out)


def test_measured_divergence_of_a_full_field():
    """BoxFluxWorkspace::divergence (src/box_flux.rs:201-206): outer samples included."""
    counts, spacing = (9, 7, 5), (0.5, 0.25, 2.0)
    g = R.GridGeometry(counts, spacing)
    rng = np.random.default_rng(2)
    faces = [rng.uniform(-1, 1, g.face_len(d)).astype(np.float32) for d in range(3)]
    w = BoxFluxWorkspace(g, 1.0, 1 << 20)
    out = torch.empty(g.cell_len(), dtype=torch.float64, device="cuda")
    w.divergence([dev(f) for f in faces], out)
    assert np.array_equal(host(out), divergence(counts, spacing, faces))
    faces[1][3] = np.inf
    with pytest.raises(BoxFluxError) as e:
        w.divergence([dev(f) for f in faces], out)
    assert (e.value.kind, e.value.inner) == ("Operator", "NonFiniteInput")
