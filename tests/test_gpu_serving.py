"""The serving loop on the device: each result alone equals it in the mix.

Requests of uneven edges arrive together, so their steps overlap on the
device through the continuous-batching loop; every final state must equal the
same request run alone on a fresh carrier, bit for bit (the kernels and their
reduction trees are deterministic and independent of what else runs).
"""
import numpy as np
import pytest

import rheon_b200 as R
from rheon_b200 import serving as S

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _device():
    if not torch.cuda.is_available() or R.device_count() == 0:
        pytest.skip("no B200")
    yield


def test_each_request_alone_equals_it_in_the_mix():
    cfg = R.CarrierConfig.mixed(pressure=R.PressureSettings(1e-8, 0.0, S.MAXF, 500))
    reqs = S.make_requests(10, rate_hz=1e6, seed=3, edge_min=32, edge_max=64, max_steps=4)
    loop = S.ServingLoop(cfg, budget_bytes=8 << 30)
    comps = loop.run(reqs, keep_state=True)
    assert len(comps) == len(reqs) and all(c.status == 0 for c in comps)
    assert max(c.admitted for c in comps) < min(c.finished for c in comps) + 10.0
    for req in reqs:
        alone = R.CarrierSimulation(R.GridGeometry((req.edge,) * 3), cfg)
        alone.init_fourier(req.seed)
        for _ in range(req.steps):
            alone.step(R.StepParams(S.MAXF, cfl=0.5))
        got = alone.download()
        for d in range(3):
            assert np.array_equal(got[d], loop.final_states[req.rid][d]), (req.rid, d)
        alone.close()
    loop.close()


def test_device_fourier_init_matches_the_host_generator():
    n = (40, 32, 24)
    sim = R.CarrierSimulation(R.GridGeometry(n), R.CarrierConfig(storage="f64"))
    sim.init_fourier(77)
    got = sim.download()
    from rheon_b200 import workloads as W

    ref = W.fourier_faces(n, seed=77, dtype=np.float64)
    for d in range(3):
        assert np.max(np.abs(got[d] - ref[d])) < 1e-13


def test_admission_respects_the_hbm_budget():
    cfg = R.CarrierConfig.mixed(pressure=R.PressureSettings(1e-8, 0.0, S.MAXF, 500))
    budget = 2 * S.carrier_bytes_estimate(64, cfg)
    reqs = S.make_requests(6, rate_hz=1e6, seed=9, edge_min=64, edge_max=64, max_steps=2)
    loop = S.ServingLoop(cfg, budget_bytes=budget)
    comps = loop.run(reqs)
    assert all(c.status == 0 for c in comps)
    assert loop.pool.created <= 2 and loop.pool.used <= budget
    loop.close()
