"""The allocation-free pressure solve against the workspace solve.

rb200_pressure_solve_static serves callers that cannot allocate device memory
(for example a plug-in inside a host application whose device memory belongs to
its own fixed-budget allocator). It keeps its scratch in one fixed
device array inside the library. This test calls it through the C ABI twice in
a row, with different right-hand sides, and checks each result against the
existing entry point (rb200_workspace_solve_rhs_device, Jacobi-PCG) within the
1e-12 relative tolerance the Jacobi parity tests use. The test buffers are
allocated by the test itself; the entry point allocates nothing.
"""
import ctypes as C

import numpy as np
import pytest

import oracle as O
import rheon_b200 as R
from rheon_b200 import _native as N
from rheon_b200 import workloads as W

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

MAXF = 1.7976931348623157e308


@pytest.fixture(scope="module", autouse=True)
def _device():
    if not torch.cuda.is_available() or R.device_count() == 0:
        pytest.skip("no B200")
    yield


def _rhs(n, seed):
    faces = W.uniform_faces(n, seed=seed)
    st, rhs = O.build_rhs(O.grid(n), 1.0, faces, 0.25)
    assert st == O.OK
    return rhs


def test_static_solve_matches_workspace_solve_on_two_calls_in_a_row():
    n = (32, 32, 32)  # the largest grid the static scratch holds
    g = R.GridGeometry(n)
    op = R.PressureOperator(g, 1.0)
    settings = R.PressureSettings(1e-10, 0.0, MAXF, 5000)
    ws = R.PressureWorkspace(g, 1 << 30)
    lib = N.lib()
    out = torch.empty(g.cell_len(), dtype=torch.float64, device="cuda")
    for seed in (11, 12):
        rhs = _rhs(n, seed)
        rhs_dev = torch.from_numpy(rhs).cuda()
        torch.cuda.synchronize()
        expected_report = ws.solve_rhs(op, rhs_dev, 0.25, settings)
        expected = ws.pressure()
        out.fill_(np.nan)
        torch.cuda.synchronize()
        rep = N.Report()
        st = lib.rb200_pressure_solve_static(C.byref(g.c()), 1.0, rhs_dev.data_ptr(), out.data_ptr(),
                                             g.cell_len(), 0.25, C.byref(settings.c()), C.byref(rep), None)
        assert st == N.OK, R.status_name(st)
        got = out.cpu().numpy()
        assert rep.iterations == expected_report.iterations
        err = np.linalg.norm(got - expected) / np.linalg.norm(expected)
        assert err <= 1e-12, err
        assert abs(rep.true_residual_l2 - expected_report.true_residual_l2) <= 1e-12 * expected_report.true_residual_l2
        assert got[0] == 0.0


def test_static_solve_rejects_grids_beyond_its_scratch():
    g = R.GridGeometry([33, 32, 32])
    lib = N.lib()
    rep = N.Report()
    settings = R.PressureSettings(1e-8, 0.0, MAXF, 100)
    buf = torch.zeros(g.cell_len(), dtype=torch.float64, device="cuda")
    st = lib.rb200_pressure_solve_static(C.byref(g.c()), 1.0, buf.data_ptr(), buf.data_ptr(), g.cell_len(), 0.25,
                                         C.byref(settings.c()), C.byref(rep), None)
    assert st == N.UNSUPPORTED
