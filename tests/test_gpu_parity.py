"""Parity of the CUDA library with the oracle, through the C ABI.

Tolerances: operator/advection/correction primitives are compared bit for bit
(same per-element operation order, no FMA). Jacobi-PCG is compared per
iteration: trace scalars and iterates within 1e-12 relative (the device's
double-double reductions usually reproduce the serial Neumaier sums exactly).
Red-black SGS is a different preconditioner and is judged at convergence.
"""
import math

import numpy as np
import pytest

import oracle as O
import rheon_b200 as R
from rheon_b200 import workloads as W

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


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


def og(g: R.GridGeometry):
    return O.grid(g.counts, g.spacing, g.origin)


def relerr(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


GRIDS = [
    R.GridGeometry([1, 1, 1]),
    R.GridGeometry([3, 1, 1]),
    R.GridGeometry([2, 2, 1]),
    R.GridGeometry([5, 4, 3], [0.2, 0.25, 0.3]),
    R.GridGeometry([17, 10, 9], [0.5, 0.75, 1.25], [2.0, -1.0, 3.0]),
    R.GridGeometry([40, 33, 9], [0.07, 0.11, 0.19], [-2.0, 4.0, 0.3]),
    R.GridGeometry([32, 32, 32]),
]


def rand_faces(g, seed, dtype, walls=True):
    rng = np.random.default_rng(seed)
    out = []
    for d in range(3):
        f = rng.uniform(-1, 1, g.face_len(d))
        if walls:
            f[W.wall_mask(g.counts, d)] = 0.0
        out.append(f.astype(dtype))
    return out


# ------------------------------------------------------------------ operator primitives
@pytest.mark.parametrize("g", GRIDS, ids=str)
def test_apply_full_is_bitwise(g):
    rho = 1.37
    p = np.random.default_rng(1).uniform(-1, 1, g.cell_len())
    out = torch.empty(g.cell_len(), dtype=torch.float64, device="cuda")
    R.PressureOperator(g, rho).apply_full(dev(p), out)
    st, ref = O.apply_full(og(g), rho, p)
    assert st == O.OK
    assert np.array_equal(host(out), ref)


@pytest.mark.parametrize("density", [1.0, 1.3, 997.0, 1e-3])
def test_jacobi_preconditioner_divides_exactly(density):
    """z = r/D through the reciprocal-and-correction sequence equals IEEE
    division bit for bit (the oracle divides), over residuals whose binary
    exponents span the fast path and both fallbacks, on grids whose
    diagonals take many values; r.z matches the oracle's Neumaier sum."""
    rng = np.random.default_rng(int(density * 1000) + 7)
    for counts, h in (([9, 7, 5], [0.31, 0.17, 0.9]), ([6, 6, 6], [1.0, 1.0, 1.0]), ([5, 3, 8], [3.7, 0.013, 0.6])):
        g = R.GridGeometry(counts, h)
        n = g.cell_len()
        op = R.PressureOperator(g, density)
        for trial in range(40):
            mant = rng.uniform(1.0, 2.0, n) * rng.choice([-1.0, 1.0], n)
            expo = rng.integers(-1000, 1000, n) if trial % 2 else rng.integers(-60, 60, n)
            r = np.ldexp(mant, expo)
            r[rng.random(n) < 0.05] = 0.0
            z = torch.empty(n, dtype=torch.float64, device="cuda")
            rz = op.precondition_jacobi(dev(r), z)
            st, zref, rzref = O.precondition(og(g), density, O.JACOBI_PCG_V1, r)
            assert st == O.OK
            got = host(z)
            assert np.array_equal(got.view(np.uint64), zref.view(np.uint64)), (counts, trial)
            if trial % 2 == 0:
                assert rz == rzref or abs(rz - rzref) <= 1e-15 * abs(rzref), (rz, rzref)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("g", GRIDS, ids=str)
def test_build_rhs_divergence_and_correction_are_bitwise(g, dtype):
    rho, dt = 1.3, 0.02
    faces = rand_faces(g, 2, dtype)
    op = R.PressureOperator(g, rho)
    dfaces = [dev(f) for f in faces]
    rhs = torch.empty(g.cell_len(), dtype=torch.float64, device="cuda")
    op.build_rhs(dfaces, dt, rhs)
    st, ref = O.build_rhs(og(g), rho, faces, dt)
    assert st == O.OK and np.array_equal(host(rhs), ref)
    div = torch.empty_like(rhs)
    op.divergence(dfaces, div)
    st, ref = O.divergence(og(g), faces)
    assert st == O.OK and np.array_equal(host(div), ref)
    p = np.random.default_rng(3).uniform(-1, 1, g.cell_len())
    op.correct_candidate_in_place(dev(p), dt, dfaces)
    st, ref = O.correct(og(g), rho, p, dt, faces)
    assert st == O.OK
    for d in range(3):
        assert np.array_equal(host(dfaces[d]), ref[d])


def test_operator_errors_match_the_reference():
    g = R.GridGeometry([3, 1, 1])
    op = R.PressureOperator(g, 1.0)
    x = dev(np.array([1.0, 2.0, -1.0, 0.0], np.float32))  # nonzero wall face
    y = dev(np.zeros(6, np.float32))
    z = dev(np.zeros(6, np.float32))
    out = torch.empty(3, dtype=torch.float64, device="cuda")
    with pytest.raises(R.OperatorError) as e:
        op.build_rhs([x, y, z], 0.5, out)
    assert e.value.kind == "NonZeroWallVelocity"
    with pytest.raises(R.OperatorError) as e:
        op.apply_full(dev(np.array([0.0, math.inf, 1.0])), out)
    assert e.value.kind == "NonFiniteInput"


def test_three_cell_hand_calculation_on_device():
    # tests/operator_contract.rs:3-27
    g = R.GridGeometry([3, 1, 1])
    op = R.PressureOperator(g, 1.0)
    x = dev(np.array([0.0, 2.0, -1.0, 0.0], np.float32))
    y = dev(np.zeros(6, np.float32))
    z = dev(np.zeros(6, np.float32))
    rhs = torch.empty(3, dtype=torch.float64, device="cuda")
    op.build_rhs([x, y, z], 0.5, rhs)
    assert host(rhs).tolist() == [-4.0, 6.0, -2.0]
    prod = torch.empty_like(rhs)
    op.apply_full(dev(np.array([0.0, 4.0, 2.0])), prod)
    assert host(prod).tolist() == [-4.0, 6.0, -2.0]
    op.correct_candidate_in_place(dev(np.array([0.0, 4.0, 2.0])), 0.5, [x, y, z])
    assert host(x).tolist() == [0.0] * 4


# ------------------------------------------------------------------ advection
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("g", GRIDS[1:], ids=str)
@pytest.mark.parametrize("dt", [0.01, 0.25, 3.0])
def test_advect_velocity_is_bitwise(g, dtype, dt):
    faces = rand_faces(g, 5, dtype, walls=False)  # the sampler does not impose walls
    out = [torch.empty(g.face_len(d), dtype=torch.float32 if dtype == np.float32 else torch.float64,
                       device="cuda") for d in range(3)]
    R.advect_velocity(g, [dev(f) for f in faces], dt, out)
    st, ref = O.advect_velocity(og(g), faces, dt)
    assert st == O.OK
    for d in range(3):
        assert np.array_equal(host(out[d]), ref[d]), d


@pytest.mark.parametrize("g", GRIDS[1:], ids=str)
def test_advect_tracer_is_bitwise(g):
    faces = rand_faces(g, 6, np.float32)
    old = np.random.default_rng(7).uniform(0, 1, g.cell_len()).astype(np.float32)
    out = torch.empty(g.cell_len(), dtype=torch.float32, device="cuda")
    for dt in (0.01, 0.5, 3.0):
        R.advect_tracer(g, dev(old), [dev(f) for f in faces], dt, out)
        st, ref = O.advect_tracer(og(g), old, faces, dt)
        assert st == O.OK and np.array_equal(host(out), ref)


def test_rest_state_and_pulse_shift_on_device():
    # tests/advection_contract.rs:69-96
    g = R.GridGeometry([8, 1, 1])
    u = dev(np.ones(9, np.float32))
    v = dev(np.zeros(16, np.float32))
    w = dev(np.zeros(16, np.float32))
    old = dev(np.array([0, 0, 1, 0, 0, 0, 0, 0], np.float32))
    out = torch.empty(8, dtype=torch.float32, device="cuda")
    R.advect_tracer(g, old, [u, v, w], 1.0, out)
    assert host(out).tolist() == [0, 0, 0, 1, 0, 0, 0, 0]


# ------------------------------------------------------------------ pressure solves
def S(rel=1e-11, abs_=1e-12, div=1e-9, it=1000):
    return R.PressureSettings(rel, abs_, div, it)


METHODS = [R.PressureImplementation.JACOBI_PCG_V1, R.PressureImplementation.SGS_PCG_V1,
           R.PressureImplementation.RBSGS_PCG]
# device method -> oracle method it must reproduce per iteration
EXACT = {R.PressureImplementation.JACOBI_PCG_V1: O.JACOBI_PCG_V1, R.PressureImplementation.SGS_PCG_V1: O.SGS_PCG_V1}


@pytest.mark.parametrize("method", METHODS)
def test_solves_hand_chain_and_reports_full_residual(method):
    # tests/pressure_contract.rs:13-25
    g = R.GridGeometry([3, 1, 1])
    ws = R.PressureWorkspace(g, 3 * 48, method)
    rep = ws.solve_rhs(R.PressureOperator(g, 1.0), [-4.0, 6.0, -2.0], 0.5, S())
    p = ws.pressure()
    assert abs(p[1] - 4.0) < 1e-10 and abs(p[2] - 2.0) < 1e-10 and p[0] == 0.0
    assert rep.true_residual_max < 1e-10


def test_single_cell_incompatible_and_gauge_row_contracts():
    # tests/pressure_contract.rs:27-72
    g1 = R.GridGeometry([1, 1, 1])
    rep = R.PressureWorkspace(g1, 48).solve_rhs(R.PressureOperator(g1, 1.0), [0.0], 1.0, S())
    assert rep.iterations == 0 and rep.true_residual_max == 0.0
    g2 = R.GridGeometry([2, 1, 1])
    with pytest.raises(R.PressureError) as e:
        R.PressureWorkspace(g2, 96).solve_rhs(R.PressureOperator(g2, 1.0), [1.0, 0.0], 1.0, S())
    assert e.value.kind == "IncompatibleRhs"
    g4 = R.GridGeometry([4, 1, 1])
    with pytest.raises(R.PressureError) as e:
        R.PressureWorkspace(g4, 192).solve_rhs(R.PressureOperator(g4, 1.0), [-0.003, 0.001, 0.001, 0.001], 1.0,
                                               S(1.0, 1.0, 0.0015, 0))
    assert e.value.kind == "IterationLimit" and e.value.iterations == 0


def test_nonfinite_rhs_cancellation_and_exhaustion():
    g = R.GridGeometry([3, 1, 1])
    ws = R.PressureWorkspace(g, 144)
    op = R.PressureOperator(g, 1.0)
    with pytest.raises(R.PressureError) as e:
        ws.solve_rhs(op, [-4.0, 6.0, -2.0], 0.5, S(), cancelled=lambda: True)
    assert e.value.kind == "Cancelled"
    with pytest.raises(R.PressureError) as e:
        ws.solve_rhs(op, [-4.0, 6.0, -2.0], 0.5, S(it=1))
    assert e.value.kind == "IterationLimit" and e.value.iterations == 1
    with pytest.raises(R.PressureError) as e:
        ws.solve_rhs(op, [-4.0, math.nan, -2.0], 0.5, S())
    assert e.value.kind == "NonFiniteInput"
    bad = S()
    bad.relative_residual = math.nan
    with pytest.raises(R.PressureError) as e:
        ws.solve_rhs(op, [-4.0, 6.0, -2.0], 0.5, bad)
    assert e.value.kind == "InvalidArgument"


@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("counts", [[1, 1, 1], [3, 1, 1], [5, 4, 3]])
def test_all_methods_recover_anisotropic_manufactured_pressure(method, counts):
    # tests/implementation_contract.rs:57-84
    g = R.GridGeometry(counts, [0.2, 0.35, 0.7])
    exact = np.sin(np.arange(g.cell_len()) * 0.7)
    _, rhs = O.apply_full(og(g), 1.3, exact)
    ws = R.PressureWorkspace(g, 48 * g.cell_len(), method, density=1.3)
    rep = ws.solve_rhs(R.PressureOperator(g, 1.3), rhs, 0.02, S())
    assert rep.predicted_divergence_max <= 1e-9
    assert np.max(np.abs(ws.pressure() - exact + exact[0])) < 1e-8
    with pytest.raises(R.PressureError) as e:
        ws.solve_rhs(R.PressureOperator(g, 1.3), np.ones_like(rhs), 0.02, S())
    assert e.value.kind == "IncompatibleRhs"


def compatible_rhs(g, seed=11, dtype=np.float64):
    faces = W.uniform_faces(g.counts, seed=seed, dtype=dtype)
    st, rhs = O.build_rhs(og(g), 1.0, faces, 0.25)
    assert st == O.OK
    return rhs


# [64, 40, 24] and [96, 16, 12] take the TMA slab path (even nx, at least one
# slab box in every direction); the others take the cp.async path.
@pytest.mark.parametrize("method", list(EXACT))
@pytest.mark.parametrize("counts", [[32, 32, 32], [17, 10, 9], [48, 20, 7], [64, 40, 24], [96, 16, 12],
                                    [72, 41, 57]])
def test_pcg_per_iteration_parity(counts, method):
    """Every iteration's scalars and the iterates track the oracle to 1e-12."""
    g = R.GridGeometry(counts)
    rhs = compatible_rhs(g)
    iters = 200 if method == R.PressureImplementation.JACOBI_PCG_V1 else 60
    s = S(0.0, 0.0, 1.7976931348623157e308, iters)
    ref = O.solve_rhs(og(g), 1.0, EXACT[method], rhs, 0.25, O.settings(0.0, 0.0, 1.7976931348623157e308, iters),
                      trace=True)
    assert ref.status == O.ITERATION_LIMIT
    ws = R.PressureWorkspace(g, 1 << 34, method)
    ws.set_trace(iters)
    with pytest.raises(R.PressureError) as e:
        ws.solve_rhs(R.PressureOperator(g, 1.0), rhs, 0.25, s)
    assert e.value.kind == "IterationLimit" and e.value.iterations == iters
    tr = ws.trace(iters)
    worst = 0.0
    for k in range(iters):
        for name in ("curvature", "alpha", "recursive_l2"):
            a, b = getattr(tr[k], name), getattr(ref.trace[k], name)
            worst = max(worst, abs(a - b) / abs(b))
        if k < iters - 1:
            for name in ("rz", "beta"):
                a, b = getattr(tr[k], name), getattr(ref.trace[k], name)
                worst = max(worst, abs(a - b) / abs(b))
    assert worst <= 1e-12, worst
    assert relerr(ws.pressure(), ref.pressure) <= 1e-12
    # iterates at intermediate counts (IterationLimit leaves the k-th iterate)
    for k in (1, 7, 50):
        refk = O.solve_rhs(og(g), 1.0, EXACT[method], rhs, 0.25, O.settings(0.0, 0.0, 1.7976931348623157e308, k))
        with pytest.raises(R.PressureError):
            ws.solve_rhs(R.PressureOperator(g, 1.0), rhs, 0.25, S(0.0, 0.0, 1.7976931348623157e308, k))
        assert relerr(ws.pressure(), refk.pressure) <= 1e-12


# [64, 40, 24] runs the persistent Jacobi-PCG kernel (true-residual checks
# and restarts inside the kernel); [24, 20, 16] the per-pass kernels.
@pytest.mark.parametrize("counts, rel", [([24, 20, 16], 1e-8), ([64, 40, 24], 1e-8), ([64, 40, 24], 1e-12)])
def test_jacobi_converged_solve_matches_oracle_iterations_and_report(counts, rel):
    g = R.GridGeometry(counts, [0.1, 0.12, 0.15])
    rhs = compatible_rhs(g, seed=5)
    s = S(rel, 0.0, 1.7976931348623157e308, 5000)
    ref = O.solve_rhs(og(g), 1.0, O.JACOBI_PCG_V1, rhs, 0.25, O.settings(rel, 0.0, 1.7976931348623157e308, 5000))
    assert ref.status == O.OK
    ws = R.PressureWorkspace(g, 1 << 34)
    rep = ws.solve_rhs(R.PressureOperator(g, 1.0), rhs, 0.25, s)
    assert rep.iterations == ref.report.iterations
    assert abs(rep.true_residual_l2 - ref.report.true_residual_l2) <= 1e-12 * ref.report.true_residual_l2
    assert relerr(ws.pressure(), ref.pressure) <= 1e-12


def test_sgs_known_answer_first_iteration():
    """src/pressure.rs:824-842: on the 2x2x1 grid r = [-12, 2, 4, 6] (row 0
    eliminated) gives z = [0, 3.25, 4.25, 4.5] and r.z = 50.5. The first
    iteration then sees d = z, q = A z = [2, 4, 1.5] on rows 1..3, d.q = 30.25
    and alpha = 50.5 / 30.25, all exact but the last, which both sides round
    once."""
    g = R.GridGeometry([2, 2, 1])
    ws = R.PressureWorkspace(g, 1 << 20, R.PressureImplementation.SGS_PCG_V1)
    ws.set_trace(1)
    with pytest.raises(R.PressureError) as e:
        ws.solve_rhs(R.PressureOperator(g, 1.0), [-12.0, 2.0, 4.0, 6.0], 1.0, S(0.0, 0.0, 1.7976931348623157e308, 1))
    assert e.value.kind == "IterationLimit" and e.value.iterations == 1
    tr = ws.trace(1)
    assert tr[0].curvature == 30.25 and tr[0].alpha == 50.5 / 30.25
    assert ws.pressure().tolist() == [0.0, 3.25 * (50.5 / 30.25), 4.25 * (50.5 / 30.25), 4.5 * (50.5 / 30.25)]


# Lexicographic SGS: the tile queue's sweeps reproduce the serial sweep, so a
# converged solve takes the oracle's iteration count to the same pressure.
@pytest.mark.parametrize("counts", [[40, 33, 28], [9, 70, 17]])
def test_sgs_converged_solve_matches_oracle_iterations_and_report(counts):
    g = R.GridGeometry(counts, [0.1, 0.12, 0.15])
    rhs = compatible_rhs(g, seed=6)
    s = S(1e-10, 0.0, 1.7976931348623157e308, 5000)
    ref = O.solve_rhs(og(g), 1.0, O.SGS_PCG_V1, rhs, 0.25, O.settings(1e-10, 0.0, 1.7976931348623157e308, 5000))
    assert ref.status == O.OK
    ws = R.PressureWorkspace(g, 1 << 34, R.PressureImplementation.SGS_PCG_V1)
    rep = ws.solve_rhs(R.PressureOperator(g, 1.0), rhs, 0.25, s)
    assert rep.iterations == ref.report.iterations
    assert abs(rep.true_residual_l2 - ref.report.true_residual_l2) <= 1e-12 * ref.report.true_residual_l2
    assert relerr(ws.pressure(), ref.pressure) <= 1e-12
    # a second solve on the same workspace starts from a clean tile queue
    rep2 = ws.solve_rhs(R.PressureOperator(g, 1.0), rhs, 0.25, s)
    assert rep2.iterations == rep.iterations and relerr(ws.pressure(), ref.pressure) <= 1e-12


@pytest.mark.parametrize("counts", [[32, 32, 32], [64, 48, 40]])
def test_rbsgs_converges_to_the_same_pressure(counts):
    g = R.GridGeometry(counts)
    rhs = compatible_rhs(g, seed=9)
    s = S(1e-10, 0.0, 1.7976931348623157e308, 5000)
    ref = O.solve_rhs(og(g), 1.0, O.JACOBI_PCG_V1, rhs, 0.25, O.settings(1e-10, 0.0, 1.7976931348623157e308, 5000))
    ws = R.PressureWorkspace(g, 1 << 34, R.PressureImplementation.RBSGS_PCG)
    rep = ws.solve_rhs(R.PressureOperator(g, 1.0), rhs, 0.25, s)
    assert rep.true_residual_l2 <= 1e-10 * np.linalg.norm(rhs) * (1 + 1e-12)
    assert rep.iterations < ref.report.iterations
    assert relerr(ws.pressure(), ref.pressure) < 1e-7
    # independent check of the reported residual with the oracle operator
    qst, qrep = O.qualify_pressure(og(g), 1.0, rhs, 0.25, O.settings(1e-10, 0.0, 1.7976931348623157e308, 1),
                                   ws.pressure())
    assert qst == O.OK


# ------------------------------------------------------------------ provider drop-in
def test_provider_prediction_qualifies_on_the_host():
    # tests/solver_provider_contract.rs:64-96, with the B200 as the provider.
    g = R.GridGeometry([4, 3, 2], [0.25, 0.3, 0.4])
    pressure = np.sin(np.arange(24) * 0.3)
    _, rhs = O.apply_full(og(g), 1.25, pressure)
    s = S(1e-10, 1e-12, 1e-8, 1000)
    prov = R.B200PressureProvider(g, 1.25, S(1e-12, 0.0, 1e-8, 1000))
    md = prov.metadata()
    assert md.stage == "pressure" and md.input["layout"] == "x-fastest-cell-centered"
    assert md.output["units"] == "Pa" and md.input["shape_xyz"] == [4, 3, 2]
    req = R.PressureRequest(g, 1.25, 0.01, rhs)
    prov.supports(req)
    out = np.full(24, np.nan)
    prov.predict(req, out)
    assert out[0] == 0.0 and np.all(np.isfinite(out))
    st, rep = O.qualify_pressure(og(g), 1.25, rhs, 0.01, O.settings(1e-10, 1e-12, 1e-8, 1000), out)
    assert st == O.OK
    assert np.max(np.abs(out - (pressure - pressure[0]))) < 1e-9
    other = R.PressureRequest(R.GridGeometry([4, 3, 3]), 1.25, 0.01, np.zeros(36))
    with pytest.raises(R.ProviderRejection) as e:
        prov.supports(other)
    assert e.value.kind == "Unsupported"
    with pytest.raises(R.ProviderRejection) as e:
        prov.predict(req, out, cancelled=lambda: True)
    assert e.value.kind == "Cancelled"


# ------------------------------------------------------------------ resident carrier step
def carrier(g, storage, method=R.PressureImplementation.JACOBI_PCG_V1, settings=None, tracer=False):
    cfg = R.CarrierConfig(density=1.0, pressure=settings or S(1e-8, 0.0, 1.7976931348623157e308, 100000),
                          storage=storage, implementation=method, with_tracer=tracer)
    return R.CarrierSimulation(g, cfg)


@pytest.mark.parametrize("storage", ["f64", "f32"])
def test_plain_method_ten_steps_match_the_oracle(storage):
    """32^3, U(-1,1) faces, dt 0.25, exactly 200 Jacobi-PCG iterations per step."""
    n = (32, 32, 32)
    g = R.GridGeometry(n)
    dtype = np.float64 if storage == "f64" else np.float32
    faces = W.uniform_faces(n, dtype=dtype)
    s = S(0.0, 0.0, 1.7976931348623157e308, 200)
    sim = carrier(g, storage, settings=s)
    sim.upload(faces)
    prm = O.StepParams(0.25, 1.0, O.JACOBI_PCG_V1, O.settings(0.0, 0.0, 1.7976931348623157e308, 200), 0.0, 1, 1)
    ref = faces
    for step in range(10):
        rep = sim.step(R.StepParams(0.25, iteration_limit_ok=True))
        assert rep.pressure.iterations == 200
        st, ref, _, orep = O.carrier_step(og(g), ref, prm)
        assert st == O.OK
        got = sim.download()
        for d in range(3):
            e = relerr(got[d].astype(np.float64), ref[d].astype(np.float64))
            assert e <= 1e-10, (step, d, e)
        assert abs(rep.actual_divergence_max - orep.actual_divergence_max) <= 1e-9 * max(
            1e-30, orep.actual_divergence_max) + 1e-14


def test_carrier_rejects_a_gate_failure_without_touching_state():
    n = (16, 16, 16)
    g = R.GridGeometry(n)
    faces = W.uniform_faces(n, dtype=np.float32)
    cfg = R.CarrierConfig(pressure=S(1e-8, 0.0, 1.7976931348623157e308, 10000), storage="f32",
                          actual_divergence_limit=0.0)
    sim = R.CarrierSimulation(g, cfg)
    sim.upload(faces)
    before = sim.download()
    with pytest.raises(R.SimulationError) as e:
        sim.step(R.StepParams(0.1))
    assert e.value.kind == "DivergenceLimit"
    after = sim.download()
    for d in range(3):
        assert np.array_equal(before[d], after[d])


def test_fourier_steps_with_cfl_match_the_oracle():
    n = (48, 48, 48)
    g = R.GridGeometry(n)
    faces = W.fourier_faces(n, dtype=np.float64)
    sim = carrier(g, "f64")
    sim.upload(faces)
    s = O.settings(1e-8, 0.0, 1.7976931348623157e308, 100000)
    ref = faces
    for step in range(3):
        rep = sim.step(R.StepParams(1e30, cfl=0.5))
        _, rate = O.velocity_rate(og(g), ref)
        dt = min(1e30, 0.5 / rate)
        assert rep.dt == dt
        prm = O.StepParams(dt, 1.0, O.JACOBI_PCG_V1, s, 0.0, 0, 1)
        st, ref, _, orep = O.carrier_step(og(g), ref, prm)
        assert st == O.OK
        assert rep.pressure.iterations == orep.pressure.iterations
        got = sim.download()
        for d in range(3):
            assert relerr(got[d], ref[d]) <= 1e-10


def test_buoyant_tracer_step_matches_the_oracle():
    n = (24, 24, 24)
    g = R.GridGeometry(n)
    faces = W.fourier_faces(n, dtype=np.float32)
    blob = W.gaussian_blob(n, sigma=4.0)
    sim = carrier(g, "f32", tracer=True)
    sim.upload(faces, blob)
    s = O.settings(1e-8, 0.0, 1.7976931348623157e308, 100000)
    ref, tr = faces, blob
    for step in range(3):
        rep = sim.step(R.StepParams(0.05, buoyancy=1.0))
        prm = O.StepParams(0.05, 1.0, O.JACOBI_PCG_V1, s, 1.0, 0, 1)
        st, ref, tr, orep = O.carrier_step(og(g), ref, prm, tracer=tr)
        assert st == O.OK
        got, gtr = sim.download(with_tracer=True)
        for d in range(3):
            assert relerr(got[d].astype(np.float64), ref[d].astype(np.float64)) <= 1e-6
        assert relerr(gtr.astype(np.float64), tr.astype(np.float64)) <= 1e-6


# ------------------------------------------------------------------ mixed-precision multigrid
MG = R.PressureImplementation.MG_MIXED


@pytest.mark.parametrize("counts", [[1, 1, 1], [3, 1, 1], [5, 4, 3]])
def test_multigrid_recovers_manufactured_pressure_on_small_grids(counts):
    # tests/implementation_contract.rs:57-84, with the multigrid method.
    g = R.GridGeometry(counts, [0.2, 0.35, 0.7])
    exact = np.sin(np.arange(g.cell_len()) * 0.7)
    _, rhs = O.apply_full(og(g), 1.3, exact)
    ws = R.PressureWorkspace(g, 1 << 30, MG, density=1.3)
    rep = ws.solve_rhs(R.PressureOperator(g, 1.3), rhs, 0.02, S())
    assert rep.predicted_divergence_max <= 1e-9
    assert np.max(np.abs(ws.pressure() - exact + exact[0])) < 1e-8


@pytest.mark.parametrize("counts", [[32, 32, 32], [64, 64, 64], [40, 40, 40], [64, 32, 16], [48, 24, 96],
                                    [9, 9, 9], [17, 9, 33], [72, 40, 24], [100, 52, 20], [13, 1, 70]])
@pytest.mark.parametrize("rel", [1e-8, 1e-10])
def test_multigrid_reaches_the_target_residual_in_few_iterations(counts, rel):
    g = R.GridGeometry(counts)
    rhs = compatible_rhs(g, seed=21)
    ws = R.PressureWorkspace(g, 1 << 34, MG)
    rep = ws.solve_rhs(R.PressureOperator(g, 1.0), rhs, 0.25, S(rel, 0.0, 1.7976931348623157e308, 500))
    # judged at convergence by the FP64 true residual, recomputed by the oracle
    st, q = O.qualify_pressure(og(g), 1.0, rhs, 0.25, O.settings(rel, 0.0, 1.7976931348623157e308, 1),
                               ws.pressure())
    assert st == O.OK, (q.true_residual_l2, rel * np.linalg.norm(rhs))
    assert rep.iterations <= 40, rep.iterations
    ref = O.solve_rhs(og(g), 1.0, O.JACOBI_PCG_V1, rhs, 0.25, O.settings(1e-12, 0.0, 1.7976931348623157e308, 100000))
    assert relerr(ws.pressure(), ref.pressure) < 1e3 * rel


@pytest.mark.parametrize("edge", [8, 24, 56, 104, 136, 200, 248])
def test_multigrid_hierarchy_exists_for_every_serving_edge(edge):
    """Every edge the serving workload draws (multiples of 8 up to 256) gets a
    hierarchy whose coarsest grid is small enough for the dense solve."""
    g = R.GridGeometry((edge, edge, edge))
    sim = R.CarrierSimulation(g, R.CarrierConfig.mixed(pressure=S(1e-8, 0.0, 1.7976931348623157e308, 500)))
    sim.init_fourier(5)
    rep = sim.step(R.StepParams(1e30, cfl=0.5))
    assert rep.pressure.iterations <= 40
    assert rep.actual_divergence_max < 1e-3
    sim.close()


def test_mixed_carrier_tracks_the_fp64_oracle():
    """Mixed precision (FP32 faces, FP32 advection, FP32 V-cycles in FP64 FCG)
    against the FP64-storage oracle step: divergence of the stored faces and
    velocity error per step."""
    n = (64, 64, 64)
    g = R.GridGeometry(n)
    faces64 = W.fourier_faces(n, dtype=np.float64)
    sim = R.CarrierSimulation(g, R.CarrierConfig.mixed(pressure=S(1e-8, 0.0, 1.7976931348623157e308, 500)))
    sim.upload([f.astype(np.float32) for f in faces64])
    s = O.settings(1e-8, 0.0, 1.7976931348623157e308, 100000)
    ref = faces64
    for step in range(3):
        rep = sim.step(R.StepParams(1e30, cfl=0.5))
        prm = O.StepParams(rep.dt, 1.0, O.JACOBI_PCG_V1, s, 0.0, 0, 8)
        st, ref, _, orep = O.carrier_step(og(g), ref, prm)
        assert st == O.OK
        got = sim.download()
        err = max(relerr(got[d].astype(np.float64), ref[d]) for d in range(3))
        assert err < 1e-4, (step, err)
        assert rep.actual_divergence_max < 1e-3, rep.actual_divergence_max
        assert rep.pressure.iterations <= 40


def test_mixed_buoyant_blob_tracks_the_fp64_oracle():
    """The buoyant-blob workload in miniature (40^3, sigma 6 cells, rel
    1e-10): mixed carrier against the FP64-storage oracle step with the same
    tracer and buoyancy, per step."""
    n = (40, 40, 40)
    g = R.GridGeometry(n)
    faces64 = W.fourier_faces(n, seed=3, dtype=np.float64)
    blob = W.gaussian_blob(n, sigma=6.0)
    sim = R.CarrierSimulation(g, R.CarrierConfig.mixed(pressure=S(1e-10, 0.0, 1.7976931348623157e308, 500),
                                                       with_tracer=True))
    sim.upload([f.astype(np.float32) for f in faces64], blob)
    s = O.settings(1e-10, 0.0, 1.7976931348623157e308, 100000)
    ref, tr = faces64, blob
    for step in range(3):
        rep = sim.step(R.StepParams(0.05, buoyancy=1.0))
        prm = O.StepParams(0.05, 1.0, O.JACOBI_PCG_V1, s, 1.0, 0, 8)
        st, ref, tr, _ = O.carrier_step(og(g), ref, prm, tracer=tr)
        assert st == O.OK
        got, gtr = sim.download(with_tracer=True)
        err = max(relerr(got[d].astype(np.float64), ref[d]) for d in range(3))
        assert err < 1e-4, (step, err)
        assert relerr(gtr.astype(np.float64), tr.astype(np.float64)) < 1e-4
        assert rep.actual_divergence_max < 1e-4, rep.actual_divergence_max


def test_carrier_state_round_trips_through_device_memory():
    """upload/download accept device pointers (the copy direction is inferred)."""
    n = (24, 20, 16)
    g = R.GridGeometry(n)
    faces = W.fourier_faces(n, seed=4, dtype=np.float64)
    sim = R.CarrierSimulation(g, R.CarrierConfig(storage="f64"))
    sim.upload(faces)
    bufs = [torch.empty(g.face_len(d), dtype=torch.float64, device="cuda") for d in range(3)]
    sim.download_ptrs(*[b.data_ptr() for b in bufs])
    for d in range(3):
        assert np.array_equal(host(bufs[d]), faces[d])


# ------------------------------------------------------------------ batched instances
def test_batched_instances_match_the_same_instances_stepped_alone():
    """Uneven boxes stepped together (one graph per instance, overlapping on
    the device) give bit-identical states to each box stepped alone."""
    sizes = [(32, 32, 32), (48, 48, 48), (40, 24, 56), (64, 64, 64)]
    cfgs = [R.CarrierConfig.mixed(pressure=S(1e-8, 0.0, 1.7976931348623157e308, 500)),
            R.CarrierConfig(pressure=S(1e-8, 0.0, 1.7976931348623157e308, 100000), storage="f64")]
    for cfg in cfgs:
        dtype = np.float32 if cfg.storage == "f32" else np.float64
        inits = [W.fourier_faces(n, seed=100 + i, dtype=dtype) for i, n in enumerate(sizes)]
        together = [R.CarrierSimulation(R.GridGeometry(n), cfg) for n in sizes]
        for sim, f in zip(together, inits):
            sim.upload(f)
        prm = [R.StepParams(1e30, cfl=0.5)] * len(sizes)
        for _ in range(3):
            out = R.step_all(together, prm)
            assert all(st == 0 for st, _ in out), [R.status_name(st) for st, _ in out]
        for i, n in enumerate(sizes):
            alone = R.CarrierSimulation(R.GridGeometry(n), cfg)
            alone.upload(inits[i])
            for _ in range(3):
                alone.step(R.StepParams(1e30, cfl=0.5))
            a, b = alone.download(), together[i].download()
            for d in range(3):
                assert np.array_equal(a[d], b[d]), (cfg.storage, n, d)
