"""On-device qualification of candidate pressures and projections.

The provider's host qualification (src/solver_provider.rs:239-270) and the
supplied-projection momentum witness (solver_provider/composition/
projection.rs:515-542) run on the device; they are compared with the oracle's
qualification and with the oracle's correction, bit for bit where the
reference compares bits.
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


@pytest.fixture(scope="module", autouse=True)
def _device():
    if not torch.cuda.is_available() or R.device_count() == 0:
        pytest.skip("no B200")
    yield
    torch.cuda.synchronize()


def og(g):
    return O.grid(g.counts, g.spacing, g.origin)


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


GRIDS = [R.GridGeometry([4, 3, 2], [0.25, 0.3, 0.4]), R.GridGeometry([17, 10, 9], [0.5, 0.75, 1.25]),
         R.GridGeometry([48, 40, 24])]


def case(g, density=1.25, seed=3):
    faces = W.uniform_faces(g.counts, seed=seed, dtype=np.float64)
    st, rhs = O.build_rhs(og(g), density, faces, 0.1)
    assert st == O.OK
    r = O.solve_rhs(og(g), density, O.JACOBI_PCG_V1, rhs, 0.1, O.settings(1e-10, 0.0, MAXF, 100000), threads=8)
    assert r.status == O.OK
    return rhs, r.pressure


@pytest.mark.parametrize("g", GRIDS, ids=str)
def test_qualification_matches_the_oracle(g):
    density = 1.25
    rhs, p = case(g, density)
    op = R.PressureOperator(g, density)
    for settings, perturb in ((R.PressureSettings(1e-8, 0.0, MAXF, 1), 0.0),
                              (R.PressureSettings(1e-8, 0.0, MAXF, 1), 1e-3),
                              (R.PressureSettings(0.0, 1e-3, 1e-12, 1), 0.0)):
        cand = p.copy()
        cand[1:] += perturb * np.sin(np.arange(1, cand.size))
        ost, orep = O.qualify_pressure(og(g), density, rhs, 0.1,
                                       O.settings(settings.relative_residual, settings.absolute_residual,
                                                  settings.divergence_limit, 1), cand)
        try:
            rep = op.qualify_pressure(dev(rhs), dev(cand), 0.1, settings)
            st = O.OK
        except R.ProviderRejection as e:
            st, rep = e.status, e.report
        assert st == ost, (st, ost)
        assert abs(rep.true_residual_l2 - orep.true_residual_l2) <= 1e-12 * max(orep.true_residual_l2, 1e-300)
        assert rep.true_residual_max == orep.true_residual_max
        assert abs(rep.predicted_divergence_max - orep.predicted_divergence_max) <= \
            1e-15 * max(orep.predicted_divergence_max, 1e-300)


def test_qualification_rejects_nonfinite_and_gauge():
    # tests/solver_provider_contract.rs:97-169: non-finite output, non-zero gauge
    g = GRIDS[1]
    rhs, p = case(g)
    op = R.PressureOperator(g, 1.25)
    s = R.PressureSettings(1e-8, 0.0, MAXF, 1)
    bad = p.copy()
    bad[5] = math.nan
    with pytest.raises(R.ProviderRejection) as e:
        op.qualify_pressure(dev(rhs), dev(bad), 0.1, s)
    assert e.value.kind == "NonFiniteOutput"
    shifted = p + 1.0
    with pytest.raises(R.ProviderRejection) as e:
        op.qualify_pressure(dev(rhs), dev(shifted), 0.1, s)
    assert e.value.kind == "NonZeroGauge"
    assert O.qualify_pressure(og(g), 1.25, rhs, 0.1, O.settings(1e-8, 0.0, MAXF, 1), shifted)[0] == O.NONZERO_GAUGE


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("g", GRIDS, ids=str)
def test_projection_witness_is_bitwise(g, dtype):
    density = 1.25
    faces = [f.astype(dtype) for f in W.uniform_faces(g.counts, seed=9, dtype=np.float64)]
    st, rhs = O.build_rhs(og(g), density, faces, 0.1)
    assert st == O.OK
    _, p = case(g, density, seed=9)
    st, corrected = O.correct(og(g), density, p, 0.1, faces)
    assert st == O.OK
    op = R.PressureOperator(g, density)
    vin = [dev(f) for f in faces]
    assert op.projection_witness(dev(p), 0.1, vin, [dev(f) for f in corrected]) is None
    # one interior face of axis 1 off by one unit in the last place
    interior1 = np.flatnonzero(~W.wall_mask(g.counts, 1))
    interior2 = np.flatnonzero(~W.wall_mask(g.counts, 2))
    axis, idx = 1, int(interior1[len(interior1) // 2])
    off = [c.copy() for c in corrected]
    off[axis][idx] = np.nextafter(off[axis][idx], dtype(np.inf))
    assert op.projection_witness(dev(p), 0.1, vin, [dev(f) for f in off]) == (axis, idx)
    # the witness reports the lowest index of the first axis that differs
    off[2][int(interior2[0])] += dtype(1.0)
    off[1][int(interior1[-1])] += dtype(0.5)
    assert op.projection_witness(dev(p), 0.1, vin, [dev(f) for f in off]) == (axis, idx)
