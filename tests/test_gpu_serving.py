"""The serving loop on the device: step and projection requests, each result
alone equals it in the mix, and the mix really overlaps on the device.

Requests of uneven edges arrive together, so their work overlaps on the
device through the continuous-batching loop. Every request records CUDA events
on its carrier's stream before its first launch and after its last one; the
test requires device intervals of different requests to overlap. Every final
state (and, for projections, the pressure) must equal the same request run
alone on a fresh carrier, bit for bit (the kernels and their reduction trees
are deterministic and independent of what else runs).
"""
import numpy as np
import pytest

import oracle as O
import rheon_b200 as R
from rheon_b200 import serving as S
from rheon_b200 import workloads as W

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _device():
    if not torch.cuda.is_available() or R.device_count() == 0:
        pytest.skip("no B200")
    yield


def relerr(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def test_each_request_alone_equals_it_in_the_mix():
    cfg = R.CarrierConfig.mixed(pressure=R.PressureSettings(1e-8, 0.0, S.MAXF, 500))
    reqs = S.make_requests(12, rate_hz=1e6, seed=3, edge_min=32, edge_max=64, max_steps=4, projection_share=0.5)
    assert {r.kind for r in reqs} == {"step", "projection"}
    loop = S.ServingLoop(cfg, budget_bytes=8 << 30, device_times=True)
    comps = loop.run(reqs, keep_state=True)
    assert len(comps) == len(reqs) and all(c.status == 0 for c in comps)
    # the device intervals of the mix overlap
    assert all(c.device_end_ms > c.device_start_ms for c in comps)
    assert S.overlapping_pairs(comps) >= 1
    for req in reqs:
        alone = R.CarrierSimulation(R.GridGeometry((req.edge,) * 3), cfg)
        alone.init_fourier(req.seed)
        if req.kind == "projection":
            alone.project(req.dt)
        else:
            for _ in range(req.steps):
                alone.step(R.StepParams(S.MAXF, cfl=0.5))
        got = alone.download()
        for d in range(3):
            assert np.array_equal(got[d], loop.final_states[req.rid][d]), (req.rid, req.kind, d)
        assert np.array_equal(alone.pressure(), loop.final_pressures[req.rid])
        alone.close()
    summary = S.summarize(comps, loop.elapsed)
    assert set(summary["by_kind"]) == {"step", "projection"}
    loop.close()


def test_projection_matches_the_oracle():
    """A projection of a supplied f32 velocity (the reference's storage) with
    Jacobi-PCG: the same iterations as the oracle's build_rhs -> solve ->
    correct_candidate_in_place, faces within f32 rounding."""
    n = (24, 20, 16)
    g = R.GridGeometry(n)
    faces = W.fourier_faces(n, seed=11, dtype=np.float32)
    dt = 0.02
    cfg = R.CarrierConfig(pressure=R.PressureSettings(1e-10, 0.0, S.MAXF, 10000), storage="f32")
    sim = R.CarrierSimulation(g, cfg)
    sim.upload(faces)
    rep = sim.project(dt)
    og = O.grid(n)
    st, rhs = O.build_rhs(og, 1.0, faces, dt)
    assert st == O.OK
    ref = O.solve_rhs(og, 1.0, O.JACOBI_PCG_V1, rhs, dt, O.settings(1e-10, 0.0, S.MAXF, 10000))
    assert ref.status == O.OK
    assert rep.pressure.iterations == ref.report.iterations
    assert rep.dt == dt
    st, corrected = O.correct(og, 1.0, ref.pressure, dt, faces)
    assert st == O.OK
    got = sim.download()
    for d in range(3):
        assert relerr(got[d].astype(np.float64), corrected[d].astype(np.float64)) < 1e-6
    assert relerr(sim.pressure(), ref.pressure) < 1e-10
    _, div = O.divergence(og, got)
    assert np.max(np.abs(div)) == rep.actual_divergence_max
    sim.close()


def test_device_fourier_init_matches_the_host_generator():
    n = (40, 32, 24)
    sim = R.CarrierSimulation(R.GridGeometry(n), R.CarrierConfig(storage="f64"))
    sim.init_fourier(77)
    got = sim.download()
    ref = W.fourier_faces(n, seed=77, dtype=np.float64)
    for d in range(3):
        assert np.max(np.abs(got[d] - ref[d])) < 1e-13


def test_admission_respects_the_hbm_budget():
    cfg = R.CarrierConfig.mixed(pressure=R.PressureSettings(1e-8, 0.0, S.MAXF, 500))
    budget = 2 * S.carrier_bytes_estimate(64, cfg)
    reqs = S.make_requests(6, rate_hz=1e6, seed=9, edge_min=64, edge_max=64, max_steps=2, projection_share=0.3)
    loop = S.ServingLoop(cfg, budget_bytes=budget)
    comps = loop.run(reqs)
    assert all(c.status == 0 for c in comps)
    assert loop.pool.created <= 2 and loop.pool.used <= budget
    loop.close()
