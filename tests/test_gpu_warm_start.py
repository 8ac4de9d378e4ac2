"""Seeded pressure solves (accepted-pressure warm start) on the device.

The reference's own known answers for solve_rhs_with_initial_pressure
(tests/pressure_initial_guess.rs, feature "accepted-pressure-warm-start") run
through the workspace for every method; Jacobi-PCG and sgs-pcg-v1 are also
compared per iteration with the oracle's seeded solve (1e-12 relative), and
the resident carrier's AcceptedPreviousV1 policy against oracle steps seeded
by the previous step's pressure.
"""
import math

import numpy as np
import pytest

import oracle as O
import rheon_b200 as R
from rheon_b200 import workloads as W

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

MAXF = 1.7976931348623157e308
ALL = [R.PressureImplementation.JACOBI_PCG_V1, R.PressureImplementation.SGS_PCG_V1,
       R.PressureImplementation.RBSGS_PCG, R.PressureImplementation.MG_MIXED]
EXACT = {R.PressureImplementation.JACOBI_PCG_V1: O.JACOBI_PCG_V1, R.PressureImplementation.SGS_PCG_V1: O.SGS_PCG_V1}


@pytest.fixture(scope="module", autouse=True)
def _device():
    if not torch.cuda.is_available() or R.device_count() == 0:
        pytest.skip("no B200")
    yield
    torch.cuda.synchronize()


def S(rel=1e-11, abs_=1e-12, div=1e-9, it=1000):
    return R.PressureSettings(rel, abs_, div, it)


def og(g):
    return O.grid(g.counts, g.spacing, g.origin)


def relerr(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def solve(ws, g, rhs, dt, s, initial):
    return ws.solve_rhs(R.PressureOperator(g, 1.0), np.asarray(rhs, np.float64), dt, s,
                        initial=np.asarray(initial, np.float64))


@pytest.mark.parametrize("method", ALL)
def test_exact_and_approximate_guesses_recover_independent_chain(method):
    # tests/pressure_initial_guess.rs:17-52
    g = R.GridGeometry([3, 1, 1])
    ws = R.PressureWorkspace(g, 1 << 30, method)
    rep = solve(ws, g, [-4.0, 6.0, -2.0], 0.5, S(), [0.0, 4.0, 2.0])
    assert rep.iterations == 0 and rep.true_residual_l2 == 0.0
    rep = solve(ws, g, [-4.0, 6.0, -2.0], 0.125, S(), [0.0, 3.0, -1.0])
    assert rep.iterations > 0
    assert np.max(np.abs(ws.pressure() - [0.0, 4.0, 2.0])) < 1e-10


def test_zero_rhs_still_checks_seed_and_current_rhs_threshold():
    # tests/pressure_initial_guess.rs:54-83
    g = R.GridGeometry([3, 1, 1])
    ws = R.PressureWorkspace(g, 1 << 30)
    with pytest.raises(R.PressureError) as e:
        solve(ws, g, [0.0] * 3, 1.0, S(1.0, 0.0, 100.0, 0), [0.0, 4.0, 2.0])
    assert e.value.kind == "IterationLimit" and e.value.iterations == 0
    rep = solve(ws, g, [0.0] * 3, 1.0, S(), [0.0, 4.0, 2.0])
    assert rep.iterations > 0
    assert np.all(np.abs(ws.pressure()) < 1e-10)


def test_full_gauge_row_and_compatibility_are_not_hidden_by_guess():
    # tests/pressure_initial_guess.rs:85-118
    g = R.GridGeometry([4, 1, 1])
    ws = R.PressureWorkspace(g, 1 << 30)
    with pytest.raises(R.PressureError) as e:
        solve(ws, g, [-0.003, 0.001, 0.001, 0.001], 1.0, S(1.0, 1.0, 0.0015, 0), [0.0] * 4)
    assert e.value.kind == "IterationLimit"
    with pytest.raises(R.PressureError) as e:
        solve(ws, g, [1.0, 0.0, 0.0, 0.0], 1.0, S(), [0.0] * 4)
    assert e.value.kind == "IncompatibleRhs"


def test_invalid_guesses_do_not_poison_a_retry():
    # tests/pressure_initial_guess.rs:120-172
    g = R.GridGeometry([3, 1, 1])
    ws = R.PressureWorkspace(g, 1 << 30)
    rhs = [-4.0, 6.0, -2.0]
    kinds = []
    for seed in ([0.0, 1.0], [0.0, math.nan, 0.0], [0.0, math.inf, 0.0], [1.0, 4.0, 2.0]):
        with pytest.raises(R.PressureError) as e:
            solve(ws, g, rhs, 0.5, S(), seed)
        kinds.append(e.value.kind)
    assert kinds == ["LengthMismatch", "NonFiniteInput", "NonFiniteInput", "InvalidInitialPressure"]
    calls = [0]

    def cancel():
        calls[0] += 1
        return calls[0] == 1

    with pytest.raises(R.PressureError) as e:
        ws.solve_rhs(R.PressureOperator(g, 1.0), np.asarray(rhs), 0.5, S(), cancelled=cancel,
                     initial=np.asarray([0.0, 3.0, -1.0]))
    assert e.value.kind == "Cancelled"
    retry = solve(ws, g, rhs, 0.5, S(), [0.0, 3.0, -1.0])
    clean = R.PressureWorkspace(g, 1 << 30)
    ref = solve(clean, g, rhs, 0.5, S(), [0.0, 3.0, -1.0])
    assert retry.iterations == ref.iterations
    assert retry.true_residual_l2 == ref.true_residual_l2
    assert np.array_equal(ws.pressure(), clean.pressure())
    cold = ws.solve_rhs(R.PressureOperator(g, 1.0), np.asarray(rhs), 0.5, S())
    cold_ref = clean.solve_rhs(R.PressureOperator(g, 1.0), np.asarray(rhs), 0.5, S())
    assert cold.iterations == cold_ref.iterations
    assert np.array_equal(ws.pressure(), clean.pressure())


@pytest.mark.parametrize("method", ALL)
def test_neumann_cosine_refines_at_second_order_when_seeded(method):
    # tests/pressure_initial_guess.rs:175-218
    previous = None
    for n in (8, 16, 32, 64):
        h = 1.0 / n
        g = R.GridGeometry([n, 1, 1], [h, 1.0, 1.0])
        x = (np.arange(n) + 0.5) * h
        cosine = np.cos(math.pi * x)
        rhs = h * math.pi * math.pi * cosine
        ws = R.PressureWorkspace(g, 1 << 30, method)
        solve(ws, g, rhs, 0.125, S(), 0.75 * (cosine - cosine[0]))
        eigen = 4.0 * math.sin(math.pi * h / 2.0) ** 2 / (h * h)
        continuum = cosine - cosine[0]
        p = ws.pressure()
        assert np.max(np.abs(p - math.pi * math.pi / eigen * continuum)) < 1e-8
        error = np.max(np.abs(p - continuum))
        if previous is not None:
            assert 3.8 <= previous / error <= 4.2
        previous = error


@pytest.mark.parametrize("method", ALL)
def test_seeded_chain_retains_full_gauge_acceptance(method):
    # tests/pressure_initial_guess.rs:220-253
    n = 64
    g = R.GridGeometry([n, 1, 1])
    seed = np.array([i * (2 * n - 1 - i) * 0.1e-5 for i in range(n)])
    ws = R.PressureWorkspace(g, 1 << 30, method)
    rep = solve(ws, g, np.zeros(n), 1.0, S(0.0, 1e-4, 1e-4, 100), seed)
    assert rep.iterations > 0 and rep.true_residual_l2 <= 1e-4
    p = ws.pressure()
    squared = p[1] * p[1]
    for i in range(1, n):
        res = p[i] - p[i - 1] if i == n - 1 else 2.0 * p[i] - p[i - 1] - p[i + 1]
        squared += res * res
    assert math.sqrt(squared) <= 1e-4


def compatible_rhs(g, seed=11):
    faces = W.uniform_faces(g.counts, seed=seed, dtype=np.float64)
    st, rhs = O.build_rhs(og(g), 1.0, faces, 0.25)
    assert st == O.OK
    return rhs


def smooth_seed(g, rhs):
    """A partial solution: a few oracle Jacobi-PCG iterations, gauge row 0."""
    r = O.solve_rhs(og(g), 1.0, O.JACOBI_PCG_V1, rhs, 0.25, O.settings(0.0, 0.0, MAXF, 7))
    return r.pressure


# [64, 40, 24] runs the persistent Jacobi-PCG kernel; [17, 10, 9] the per-pass kernels.
@pytest.mark.parametrize("method", list(EXACT))
@pytest.mark.parametrize("counts", [[17, 10, 9], [64, 40, 24]])
def test_seeded_solve_per_iteration_parity(counts, method):
    g = R.GridGeometry(counts)
    rhs = compatible_rhs(g)
    seed = smooth_seed(g, rhs)
    iters = 80
    ref = O.solve_rhs(og(g), 1.0, EXACT[method], rhs, 0.25, O.settings(0.0, 0.0, MAXF, iters), trace=True,
                      initial=seed)
    assert ref.status == O.ITERATION_LIMIT
    ws = R.PressureWorkspace(g, 1 << 34, method)
    ws.set_trace(iters)
    with pytest.raises(R.PressureError) as e:
        solve(ws, g, rhs, 0.25, S(0.0, 0.0, MAXF, iters), seed)
    assert e.value.kind == "IterationLimit" and e.value.iterations == iters
    tr = ws.trace(iters)
    worst = 0.0
    for k in range(iters):
        for name in ("curvature", "alpha", "recursive_l2"):
            a, b = getattr(tr[k], name), getattr(ref.trace[k], name)
            worst = max(worst, abs(a - b) / abs(b))
    assert worst <= 1e-12, worst
    assert relerr(ws.pressure(), ref.pressure) <= 1e-12


@pytest.mark.parametrize("counts", [[17, 10, 9], [64, 40, 24]])
def test_seeded_converged_solve_matches_the_oracle(counts):
    g = R.GridGeometry(counts)
    rhs = compatible_rhs(g, seed=5)
    seed = smooth_seed(g, rhs)
    ref = O.solve_rhs(og(g), 1.0, O.JACOBI_PCG_V1, rhs, 0.25, O.settings(1e-10, 0.0, MAXF, 5000), initial=seed)
    assert ref.status == O.OK
    ws = R.PressureWorkspace(g, 1 << 34)
    rep = solve(ws, g, rhs, 0.25, S(1e-10, 0.0, MAXF, 5000), seed)
    assert rep.iterations == ref.report.iterations
    assert abs(rep.true_residual_l2 - ref.report.true_residual_l2) <= 1e-12 * ref.report.true_residual_l2
    assert relerr(ws.pressure(), ref.pressure) <= 1e-12


def test_carrier_accepted_previous_policy_matches_seeded_oracle_steps():
    """AcceptedPreviousV1: the first step is cold, every later step is seeded
    by the previous accepted pressure; each matches the oracle step seeded the
    same way."""
    n = (48, 48, 48)
    g = R.GridGeometry(n)
    faces = W.fourier_faces(n, dtype=np.float64)
    settings = S(1e-8, 0.0, MAXF, 100000)
    warm = R.CarrierSimulation(g, R.CarrierConfig(pressure=settings, storage="f64", warm_start=True))
    cold = R.CarrierSimulation(g, R.CarrierConfig(pressure=settings, storage="f64"))
    warm.upload(faces)
    cold.upload(faces)
    s = O.settings(1e-8, 0.0, MAXF, 100000)
    ref, prev = faces, None
    for step in range(4):
        rep = warm.step(R.StepParams(0.05))
        crep = cold.step(R.StepParams(0.05))
        assert rep.pressure_initialization == (0 if step == 0 else 1)
        assert crep.pressure_initialization == 0
        prm = O.StepParams(0.05, 1.0, O.JACOBI_PCG_V1, s, 0.0, 0, 8)
        st, ref, _, orep, prev = O.carrier_step(og(g), ref, prm, initial=prev, keep_pressure=True)
        assert st == O.OK
        assert rep.pressure.iterations == orep.pressure.iterations
        got = warm.download()
        for d in range(3):
            assert relerr(got[d], ref[d]) <= 1e-10
    # a new accepted state invalidates the history: the next step is cold
    warm.upload(faces)
    assert warm.step(R.StepParams(0.05)).pressure_initialization == 0


def test_seeding_cuts_iterations_under_steady_forcing():
    """A density blob released from rest: the pressure that balances its
    buoyancy changes little from step to step, so the accepted previous
    pressure is a good start (the case the reference's warm start targets)."""
    n = (32, 32, 32)
    g = R.GridGeometry(n)
    zero = [np.zeros(g.face_len(d)) for d in range(3)]
    blob = W.gaussian_blob(n, sigma=5.0)
    settings = S(1e-8, 0.0, MAXF, 100000)
    sims = {}
    for name, warm in (("warm", True), ("cold", False)):
        sims[name] = R.CarrierSimulation(g, R.CarrierConfig(pressure=settings, storage="f64", with_tracer=True,
                                                            warm_start=warm))
        sims[name].upload(zero, blob)
    its = {"warm": [], "cold": []}
    for _ in range(6):
        for name in ("warm", "cold"):
            its[name].append(sims[name].step(R.StepParams(0.01, buoyancy=1.0)).pressure.iterations)
    assert its["warm"][0] == its["cold"][0]
    # the seed is about 1e-2 off in relative terms, so to a relative residual
    # of 1e-8 it saves about a quarter of the iterations
    assert sum(its["warm"][1:]) < 0.8 * sum(its["cold"][1:]), its
