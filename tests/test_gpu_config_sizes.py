"""Parity at the workloads' own sizes: 128^3 carrier steps against the oracle.

At 128^3 the device takes paths that the small-grid tests do not reach: the
solver vectors stay in L2 between passes, the persistent Jacobi-PCG kernel
streams 32x8x8 bricks through its TMA ring over 148 blocks, and the step
graph's WHILE node runs many iteration chunks. These tests run the bench's
own workload (random-Fourier velocity, seed 20261203, CFL 0.5, relative
residual 1e-8) for one step and compare with the oracle at all host threads.

Tolerances: the plain Jacobi-PCG step tracks the oracle per iteration, so the
iteration count is equal, dt is equal bit for bit and the faces agree within
1e-10 relative. Red-black SGS is a different preconditioner: it is judged at
convergence, by the oracle's own recomputation of the true residual of the
device's pressure and by the divergence of the corrected faces. The mixed
method (FP32 faces and multigrid) is compared with the FP64-storage oracle step
within 1e-4 relative, the bound of the smaller mixed tests.
"""
import os

import numpy as np
import pytest

import oracle as O
import rheon_b200 as R
from rheon_b200 import workloads as W

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

MAXF = 1.7976931348623157e308
SEED = 20261203
N128 = (128, 128, 128)
THREADS = os.cpu_count() or 1


@pytest.fixture(scope="module", autouse=True)
def _device():
    if not torch.cuda.is_available() or R.device_count() == 0:
        pytest.skip("no B200")
    yield
    torch.cuda.synchronize()


def og(g: R.GridGeometry):
    return O.grid(g.counts, g.spacing, g.origin)


def relerr(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


@pytest.fixture(scope="module")
def fourier128():
    return W.fourier_faces(N128, seed=SEED, dtype=np.float64)


@pytest.fixture(scope="module")
def oracle_step128(fourier128):
    """The oracle's Jacobi-PCG step of the bench's 128^3 workload."""
    g = O.grid(N128)
    _, rate = O.velocity_rate(g, fourier128)
    dt = min(MAXF, 0.5 / rate)
    prm = O.StepParams(dt, 1.0, O.JACOBI_PCG_V1, O.settings(1e-8, 0.0, MAXF, 1000000), 0.0, 0, THREADS)
    st, faces, _, rep = O.carrier_step(g, fourier128, prm)
    assert st == O.OK
    return dt, faces, rep


def test_jacobi_step_at_128_matches_the_oracle(fourier128, oracle_step128):
    dt, ref, orep = oracle_step128
    g = R.GridGeometry(N128)
    cfg = R.CarrierConfig(pressure=R.PressureSettings(1e-8, 0.0, MAXF, 1000000), storage="f64",
                          implementation=R.PressureImplementation.JACOBI_PCG_V1, max_courant=1.0)
    sim = R.CarrierSimulation(g, cfg)
    sim.upload(fourier128)
    rep = sim.step(R.StepParams(MAXF, cfl=0.5))
    assert rep.dt == dt
    assert rep.pressure.iterations == orep.pressure.iterations, (rep.pressure.iterations,
                                                                 orep.pressure.iterations)
    assert abs(rep.pressure.true_residual_l2 - orep.pressure.true_residual_l2) <= \
        1e-10 * orep.pressure.true_residual_l2
    got = sim.download()
    for d in range(3):
        e = relerr(got[d], ref[d])
        assert e <= 1e-10, (d, e)
    assert abs(rep.actual_divergence_max - orep.actual_divergence_max) <= \
        1e-8 * orep.actual_divergence_max + 1e-15
    sim.close()


def test_rbsgs_step_at_128_converges_like_the_oracle(fourier128, oracle_step128):
    dt, ref, orep = oracle_step128
    g = R.GridGeometry(N128)
    cfg = R.CarrierConfig(pressure=R.PressureSettings(1e-8, 0.0, MAXF, 1000000), storage="f64",
                          implementation=R.PressureImplementation.RBSGS_PCG, max_courant=1.0)
    sim = R.CarrierSimulation(g, cfg)
    sim.upload(fourier128)
    rep = sim.step(R.StepParams(MAXF, cfl=0.5))
    assert rep.dt == dt
    assert rep.pressure.iterations < orep.pressure.iterations
    # the right-hand side of the step, from the oracle's advection of the same state
    og128 = O.grid(N128)
    st, adv = O.advect_velocity(og128, fourier128, dt, threads=THREADS)
    assert st == O.OK
    st, rhs = O.build_rhs(og128, 1.0, adv, dt)
    assert st == O.OK
    p = sim.pressure()
    assert p[0] == 0.0
    st, q = O.qualify_pressure(og128, 1.0, rhs, dt, O.settings(1e-8, 0.0, MAXF, 1), p)
    assert st == O.OK, (q.true_residual_l2, 1e-8 * np.linalg.norm(rhs))
    assert abs(q.true_residual_l2 - rep.pressure.true_residual_l2) <= 1e-9 * q.true_residual_l2
    # final divergence: the corrected faces, recomputed by the oracle
    got = sim.download()
    _, div = O.divergence(og128, got)
    assert np.max(np.abs(div)) == rep.actual_divergence_max
    assert rep.actual_divergence_max <= 10 * orep.actual_divergence_max + 1e-12
    for d in range(3):
        assert relerr(got[d], ref[d]) <= 1e-6
    sim.close()


def test_mixed_step_at_128_tracks_the_fp64_oracle(fourier128, oracle_step128):
    dt, ref, orep = oracle_step128
    g = R.GridGeometry(N128)
    sim = R.CarrierSimulation(g, R.CarrierConfig.mixed(pressure=R.PressureSettings(1e-8, 0.0, MAXF, 500)))
    sim.upload([f.astype(np.float32) for f in fourier128])
    rep = sim.step(R.StepParams(MAXF, cfl=0.5))
    # the FP32 faces give a slightly different rate, hence dt
    assert abs(rep.dt - dt) <= 1e-6 * dt
    assert rep.pressure.iterations <= 40
    got = sim.download()
    err = max(relerr(got[d].astype(np.float64), ref[d]) for d in range(3))
    assert err < 1e-4, err
    assert rep.actual_divergence_max < 1e-3
    sim.close()
