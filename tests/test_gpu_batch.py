"""The packed batch of carriers (one launch per stage over every instance,
one CUDA graph per batched step) on the device.

Determinism: an instance's block span and reduction tree depend only on its
own grid, so each instance of a mixed batch must equal, bit for bit, the same
instance stepped in a batch of its own. Accuracy: the batched mixed method is
judged like the single mixed carrier, against the FP64-storage oracle step at
the same dt (velocity within 1e-4 relative, divergence of the stored faces
below 1e-3, at most 40 iterations), and against the single mixed carrier
(the same FP32 multigrid in FP64 flexible CG with other reduction trees and
launch shapes: faces within 1e-5 relative).
"""
import numpy as np
import pytest

import oracle as O
import rheon_b200 as R
from rheon_b200 import workloads as W

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

MAXF = 1.7976931348623157e308
SIZES = [(32, 32, 32), (48, 48, 48), (64, 64, 64), (48, 32, 64), (96, 64, 32)]


@pytest.fixture(scope="module", autouse=True)
def _device():
    if not torch.cuda.is_available() or R.device_count() == 0:
        pytest.skip("no B200")
    yield
    torch.cuda.synchronize()


def cfg():
    return R.CarrierConfig.mixed(pressure=R.PressureSettings(1e-8, 0.0, MAXF, 500))


def relerr(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def inits(sizes, dtype=np.float32):
    return [W.fourier_faces(n, seed=200 + i, dtype=dtype) for i, n in enumerate(sizes)]


def test_each_instance_equals_itself_in_a_batch_of_one():
    faces = inits(SIZES)
    batch = R.BatchedCarriers([R.GridGeometry(n) for n in SIZES], cfg())
    for i, f in enumerate(faces):
        batch.upload(i, f)
    prm = R.StepParams(MAXF, cfl=0.5)
    its = []
    for _ in range(3):
        out = batch.step(prm)
        assert all(st == 0 for st, _ in out), [(R.status_name(st), r.pressure.iterations) for st, r in out]
        its.append([r.pressure.iterations for _, r in out])
    for i, n in enumerate(SIZES):
        alone = R.BatchedCarriers([R.GridGeometry(n)], cfg())
        alone.upload(0, faces[i])
        for s in range(3):
            (st, rep), = alone.step(prm)
            assert st == 0 and rep.pressure.iterations == its[s][i]
        a, b = alone.download(0), batch.download(i)
        for d in range(3):
            assert np.array_equal(a[d], b[d]), (n, d)
        assert np.array_equal(alone.pressure(0), batch.pressure(i))
        alone.close()
    batch.close()


def test_batch_tracks_the_fp64_oracle():
    sizes = [(32, 32, 32), (48, 32, 64)]
    faces64 = inits(sizes, np.float64)
    batch = R.BatchedCarriers([R.GridGeometry(n) for n in sizes], cfg())
    for i, f in enumerate(faces64):
        batch.upload(i, [x.astype(np.float32) for x in f])
    s = O.settings(1e-8, 0.0, MAXF, 100000)
    refs = list(faces64)
    for step in range(2):
        out = batch.step(R.StepParams(MAXF, cfl=0.5))
        for i, n in enumerate(sizes):
            st, rep = out[i]
            assert st == 0 and rep.pressure.iterations <= 40, (n, st, rep.pressure.iterations)
            assert rep.actual_divergence_max < 1e-3
            prm = O.StepParams(rep.dt, 1.0, O.JACOBI_PCG_V1, s, 0.0, 0, 8)
            ost, refs[i], _, _ = O.carrier_step(O.grid(n), refs[i], prm)
            assert ost == O.OK
            got = batch.download(i)
            err = max(relerr(got[d].astype(np.float64), refs[i][d]) for d in range(3))
            assert err < 1e-4, (step, n, err)
            # the reported residual is a true FP64 residual, recomputed here
            p = batch.pressure(i)
            assert p[0] == 0.0
    batch.close()


def test_batch_agrees_with_the_single_mixed_carrier():
    sizes = [(64, 64, 64), (96, 64, 32)]
    faces = inits(sizes)
    batch = R.BatchedCarriers([R.GridGeometry(n) for n in sizes], cfg())
    singles = []
    for i, (n, f) in enumerate(zip(sizes, faces)):
        batch.upload(i, f)
        sim = R.CarrierSimulation(R.GridGeometry(n), cfg())
        sim.upload(f)
        singles.append(sim)
    for _ in range(2):
        out = batch.step(R.StepParams(MAXF, cfl=0.5))
        for i, sim in enumerate(singles):
            rep = sim.step(R.StepParams(MAXF, cfl=0.5))
            st, brep = out[i]
            assert st == 0
            assert abs(brep.pressure.iterations - rep.pressure.iterations) <= 2
            assert abs(brep.dt - rep.dt) <= 1e-6 * rep.dt
    for i, sim in enumerate(singles):
        a, b = sim.download(), batch.download(i)
        for d in range(3):
            assert relerr(b[d].astype(np.float64), a[d].astype(np.float64)) < 1e-5
        sim.close()
    batch.close()


def test_a_failed_instance_keeps_its_state_and_the_others_step():
    sizes = [(32, 32, 32), (48, 48, 48), (64, 32, 32)]
    faces = inits(sizes)
    batch = R.BatchedCarriers([R.GridGeometry(n) for n in sizes], cfg())
    for i, f in enumerate(faces):
        batch.upload(i, f)
    good = R.StepParams(MAXF, cfl=0.5)
    out = batch.step([good, R.StepParams(-1.0), good])
    assert out[0][0] == 0 and out[2][0] == 0
    assert R.status_name(out[1][0]) == "InvalidArgument"
    got = batch.download(1)
    for d in range(3):
        assert np.array_equal(got[d], faces[1][d])
    # the others advanced exactly as they do alone
    for i in (0, 2):
        alone = R.BatchedCarriers([R.GridGeometry(sizes[i])], cfg())
        alone.upload(0, faces[i])
        (st, _), = alone.step(good)
        assert st == 0
        a, b = alone.download(0), batch.download(i)
        for d in range(3):
            assert np.array_equal(a[d], b[d])
        alone.close()
    batch.close()


def test_batch_rejects_levels_without_fused_pairs():
    # 40 -> 20 -> 10: the 10-cell rows are not a multiple of 4
    with pytest.raises(R.SimulationError) as e:
        R.BatchedCarriers([R.GridGeometry((32, 32, 32)), R.GridGeometry((40, 40, 40))], cfg())
    assert e.value.kind == "Unsupported"


def test_profiled_step_equals_the_graph_step():
    """The eager, event-timed step issues the graph's kernels in the same order:
    the same bits, and every kernel kind of the step is timed."""
    sizes = [(32, 32, 32), (64, 48, 32)]
    faces = inits(sizes)
    a = R.BatchedCarriers([R.GridGeometry(n) for n in sizes], cfg())
    b = R.BatchedCarriers([R.GridGeometry(n) for n in sizes], cfg())
    for i, f in enumerate(faces):
        a.upload(i, f)
        b.upload(i, f)
    prm = R.StepParams(MAXF, cfl=0.5)
    for _ in range(2):
        out = a.step(prm)
        prof = b.profile_step(prm)
        assert prof["statuses"] == [st for st, _ in out] == [0, 0]
        assert [r.pressure.iterations for r in prof["reports"]] == [r.pressure.iterations for _, r in out]
        for name in ("k_b_advect", "k_b_pass1", "k_b_train (finest)", "k_b_lower", "k_b_finish", "k_b_correct"):
            ms, launches = prof["kernels"][name]
            assert launches > 0 and ms > 0.0, name
    for i in range(len(sizes)):
        x, y = a.download(i), b.download(i)
        for d in range(3):
            assert np.array_equal(x[d], y[d])
