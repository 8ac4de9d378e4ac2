"""The persistent red-black SGS solver against the per-pass kernels.

Both paths compute the same iteration: the same update, red y = r/D, black
and red passes with the same neighbour order and correctly rounded
quotients; only the order in which r.r and r.z are summed (double-double
partials in both) differs. So the per-iteration scalars agree to 1e-13 and
the iteration counts and final pressures match. RB200_PERSISTENT=0 selects
the per-pass kernels for a workspace made while it is set.
"""
import os

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


def workspace(g, persistent):
    old = os.environ.get("RB200_PERSISTENT")
    try:
        if persistent:
            os.environ.pop("RB200_PERSISTENT", None)
        else:
            os.environ["RB200_PERSISTENT"] = "0"
        return R.PressureWorkspace(g, 1 << 34, R.PressureImplementation.RBSGS_PCG)
    finally:
        if old is None:
            os.environ.pop("RB200_PERSISTENT", None)
        else:
            os.environ["RB200_PERSISTENT"] = old


@pytest.mark.parametrize("counts", [[32, 32, 32], [64, 40, 24], [96, 16, 12]])
def test_persistent_rbsgs_tracks_the_per_pass_solver(counts):
    g = R.GridGeometry(counts, [0.1, 0.12, 0.15])
    faces = W.uniform_faces(counts, seed=3, dtype=np.float64)
    st, rhs = O.build_rhs(O.grid(counts, [0.1, 0.12, 0.15]), 1.0, faces, 0.25)
    assert st == O.OK
    cap = 400
    s = R.PressureSettings(1e-10, 0.0, 1.7976931348623157e308, cap)
    results = []
    for persistent in (False, True):
        ws = workspace(g, persistent)
        ws.set_trace(cap)
        rep = ws.solve_rhs(R.PressureOperator(g, 1.0), rhs, 0.25, s)
        results.append((rep, ws.trace(rep.iterations), ws.pressure()))
    (ra, ta, pa), (rb, tb, pb) = results
    assert ra.iterations == rb.iterations > 10
    worst = 0.0
    for k in range(ra.iterations - 1):
        for name in ("curvature", "alpha", "recursive_l2", "rz", "beta"):
            a, b = getattr(ta[k], name), getattr(tb[k], name)
            worst = max(worst, abs(a - b) / max(abs(a), 1e-300))
    assert worst <= 1e-13, worst
    assert np.linalg.norm(pa - pb) <= 1e-12 * np.linalg.norm(pa)
    assert abs(ra.true_residual_l2 - rb.true_residual_l2) <= 1e-9 * ra.true_residual_l2


def test_persistent_rbsgs_restarts_and_stops_like_the_per_pass_solver():
    """A tight target forces true-residual checks and restarts inside the kernel."""
    counts = [64, 40, 24]
    g = R.GridGeometry(counts)
    faces = W.uniform_faces(counts, seed=8, dtype=np.float64)
    st, rhs = O.build_rhs(O.grid(counts), 1.0, faces, 0.25)
    assert st == O.OK
    s = R.PressureSettings(1e-14, 0.0, 1.7976931348623157e308, 3000)
    out = []
    for persistent in (False, True):
        ws = workspace(g, persistent)
        try:
            rep = ws.solve_rhs(R.PressureOperator(g, 1.0), rhs, 0.25, s)
            out.append(("ok", rep.iterations, ws.pressure()))
        except R.PressureError as e:
            out.append((e.kind, e.iterations, ws.pressure()))
    assert out[0][0] == out[1][0] and out[0][1] == out[1][1]
    assert np.linalg.norm(out[0][2] - out[1][2]) <= 1e-11 * np.linalg.norm(out[0][2])
