"""Liquid-volume transport on the device against the oracle and the reference's answers.

The device LiquidVolumeState (src/liquid_volume.rs:520-776) must produce the
oracle's candidate fraction bit for bit, the same error with the same payload
(the first failing cell in x-fastest order), and the same ledger; a rejected
interval leaves the accepted state untouched. The known-answer cases restate
tests/liquid_volume_contract.rs.
"""
import math

import numpy as np
import pytest

import oracle as O
import rheon_b200 as R
from rheon_b200 import liquid as L

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _device():
    if not torch.cuda.is_available() or R.device_count() == 0:
        pytest.skip("no B200")
    yield
    torch.cuda.synchronize()


SETTINGS = L.LiquidVolumeSettings(1.0, 1e-9)


def dev(a, dtype):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=dtype)).cuda()


def fields(counts):
    g = O.grid(counts)
    return [np.zeros(O.face_len(g, a), np.float32) for a in range(3)]


def fidx(counts, axis, p):
    fc = list(counts)
    fc[axis] += 1
    return p[0] + fc[0] * (p[1] + fc[1] * p[2])


def run_both(counts, spacing, density, fraction, vel, start, dt, inlet, source=None, settings=SETTINGS,
             origin=(0.0, 0.0, 0.0)):
    """One interval on the device and in the oracle; returns (device report or
    error, oracle triple, device state)."""
    grid = R.GridGeometry(counts, spacing, origin)
    st = L.LiquidVolumeState(grid, density, (1, 0), np.asarray(fraction, np.float64))
    og = O.grid(counts, spacing, origin)
    want = O.liquid_advance(og, density, fraction, vel, start, dt, inlet, source=source,
                            max_outward_courant=settings.max_outward_courant,
                            actual_divergence_limit=settings.actual_divergence_limit, state_time=start)
    if start != 0.0:  # bring the device state to `start` with a zero-velocity interval
        st.advance([dev(np.zeros(O.face_len(og, a)), np.float32) for a in range(3)], 0.0, start, (9, 9),
                   L.LiquidInlet((4, 2), [[0.0, 0.0]] * 3), settings)
    try:
        got = st.advance([dev(v, np.float32) for v in vel], start, dt, (2, 3), L.LiquidInlet((4, 2), inlet), settings,
                         source=dev(source, np.float64) if source is not None else None, source_stamp=(3, 7))
    except L.LiquidVolumeError as e:
        got = e
    return got, want, st


def same_report(got: L.LiquidVolumeReport, want: dict):
    for k in ("dt", "time", "max_outward_courant", "actual_divergence_max", "fraction_min", "fraction_max",
              "dry_cells", "mixed_cells", "full_cells"):
        assert getattr(got, k) == want[k], k
    for k in ("liquid_volume_before", "liquid_volume_after", "inward_boundary_volume", "outward_boundary_volume",
              "source_volume", "liquid_mass_before", "liquid_mass_after"):
        assert abs(getattr(got, k) - want[k]) <= 1e-15 * max(abs(want[k]), 1e-300), k
    scale = abs(want["liquid_volume_before"]) + abs(want["liquid_volume_after"])
    assert abs(got.volume_balance_error - want["volume_balance_error"]) <= 4e-16 * max(scale, 1e-300)


@pytest.mark.parametrize("axis", [0, 1, 2])
@pytest.mark.parametrize("speed", [-0.5, 0.5])
def test_upwind_inlet_outlet_hand_volumes(axis, speed):
    """tests/liquid_volume_contract.rs:53-100"""
    counts = [1, 1, 1]
    counts[axis] = 4
    vel = fields(counts)
    vel[axis][:] = speed
    alpha = [[0.0, 0.0] for _ in range(3)]
    alpha[axis] = [0.5, 0.125]
    got, want, st = run_both(tuple(counts), (1.0, 1.0, 1.0), 1000.0, [0.0, 0.25, 0.75, 1.0], vel, 0.0, 1.0, alpha,
                             origin=(2.0, 3.0, 4.0))
    assert want[0] == "Ok" and isinstance(got, L.LiquidVolumeReport)
    expected = [0.25, 0.125, 0.5, 0.875] if speed > 0 else [0.125, 0.5, 0.875, 0.5625]
    assert list(st.fraction()) == expected
    same_report(got, want[2])
    assert got.stamp == (1, 1) and got.flow == (2, 3) and got.inlet == (4, 2) and got.time == 1.0
    assert (got.inward_boundary_volume, got.outward_boundary_volume) == ((0.25, 0.5) if speed > 0 else (0.0625, 0.0))
    assert st.occupancy(0) == L.LiquidOccupancy.MIXED and st.occupancy(4) is None


def test_closed_circulation_and_sources():
    """tests/liquid_volume_contract.rs:101-151"""
    counts = (2, 2, 2)
    vel = fields(counts)
    for z in range(2):
        vel[0][fidx(counts, 0, (1, 0, z))] = 0.25
        vel[0][fidx(counts, 0, (1, 1, z))] = -0.25
        vel[1][fidx(counts, 1, (0, 1, z))] = -0.5
        vel[1][fidx(counts, 1, (1, 1, z))] = 0.5
    got, want, st = run_both(counts, (0.5, 1.0, 2.0), 1000.0, [1.0, 0.0, 0.0, 0.0, 0.0, 0.5, 0.0, 0.25], vel, 0.0,
                             0.5, [[1.0, 1.0]] * 3)
    assert list(st.fraction()) == [0.75, 0.25, 0.0, 0.0, 0.0, 0.375, 0.0625, 0.3125]
    same_report(got, want[2])
    for density in (1.0, 1000.0):
        got, want, st = run_both((2, 1, 1), (1.0, 1.0, 1.0), density, [0.25, 0.75], fields((2, 1, 1)), 0.0, 0.5,
                                 [[0.0, 0.0]] * 3, source=np.array([0.25, -0.125]))
        assert list(st.fraction()) == [0.375, 0.6875]
        assert got.source == (3, 7) and got.source_volume == 0.0625 and got.liquid_mass_after == density * 1.0625


def test_translated_slab_matches_the_binomial_over_many_intervals():
    """tests/liquid_volume_contract.rs:219-270 (n = 64, Courant 0.5)"""
    n, courant = 64, 0.5
    h = 1.0 / n
    grid = R.GridGeometry((n, 1, 1), (h, 1.0, 1.0))
    init = np.array([1.0 if n // 4 <= i < n // 2 else 0.0 for i in range(n)])
    st = L.LiquidVolumeState(grid, 1000.0, (1, 0), init)
    vel = fields((n, 1, 1))
    vel[0][:] = 0.25
    dv = [dev(v, np.float32) for v in vel]
    dt = courant * h / 0.25
    steps = int(0.5 / dt)
    f, t = init.copy(), 0.0
    og = O.grid((n, 1, 1), (h, 1.0, 1.0))
    for k in range(steps):
        r = st.advance(dv, st.time, dt, (2, k), L.LiquidInlet((4, 2), [[0.0, 0.0]] * 3), SETTINGS)
        _, f, _ = O.liquid_advance(og, 1000.0, f, vel, t, dt, [[0.0, 0.0]] * 3)
        t = r.time
    got = st.fraction()
    assert np.array_equal(got.view(np.uint64), f.view(np.uint64))
    for i, value in enumerate(got):
        binomial = sum(math.comb(steps, k) * courant ** k * (1 - courant) ** (steps - k) * init[i - k]
                       for k in range(0, min(steps, i) + 1))
        assert abs(value - binomial) <= 2e-12 * max(abs(value), abs(binomial), 1.0)
    assert st.stamp == (1, steps)


@pytest.mark.parametrize("counts", [(7, 5, 3), (16, 9, 12), (33, 20, 17)], ids=str)
def test_random_intervals_match_the_oracle_bitwise(counts):
    rng = np.random.default_rng(sum(counts))
    spacing = (0.5, 0.75, 1.25)
    g = O.grid(counts, spacing)
    f = rng.uniform(0.2, 0.8, int(np.prod(counts)))
    vel = [rng.uniform(-0.05, 0.05, O.face_len(g, a)).astype(np.float32) for a in range(3)]
    src = rng.uniform(-1e-3, 1e-3, f.size)
    inlet = [[0.25, 0.5], [0.0, 1.0], [0.125, 0.75]]
    settings = L.LiquidVolumeSettings(1.0, 10.0)
    grid = R.GridGeometry(counts, spacing)
    st = L.LiquidVolumeState(grid, 800.0, (5, 0), f)
    dv = [dev(v, np.float32) for v in vel]
    ds = dev(src, np.float64)
    t = 0.0
    for k in range(4):
        err, f2, want = O.liquid_advance(g, 800.0, f, vel, t, 0.05, inlet, source=src, max_outward_courant=1.0,
                                         actual_divergence_limit=10.0)
        assert err == "Ok"
        got = st.advance(dv, t, 0.05, (2, k), L.LiquidInlet((4, 2), inlet), settings, source=ds, source_stamp=(3, k))
        assert np.array_equal(st.fraction().view(np.uint64), f2.view(np.uint64))
        same_report(got, want)
        assert got.stamp == (5, k + 1) and got.source == (3, k)
        f, t = f2, got.time
    # a strongly compressive random flow: the same first failure and payload
    vel = [rng.uniform(-3.0, 3.0, O.face_len(g, a)).astype(np.float32) for a in range(3)]
    f = rng.uniform(0.0, 1.0, f.size)
    for lim in (1.0, 0.5):
        err, _, want = O.liquid_advance(g, 800.0, f, vel, 0.0, 0.05, inlet, max_outward_courant=lim,
                                        actual_divergence_limit=100.0)
        st2 = L.LiquidVolumeState(grid, 800.0, (5, 0), f)
        with pytest.raises(L.LiquidVolumeError) as e:
            st2.advance([dev(v, np.float32) for v in vel], 0.0, 0.05, (2, 0), L.LiquidInlet((4, 2), inlet),
                        L.LiquidVolumeSettings(lim, 100.0))
        assert e.value.kind == err != "Ok"
        if err in ("CourantLimit", "FractionBounds"):
            assert e.value.cell == want["error_cell"] and e.value.actual == want["error_actual"]
        assert np.array_equal(st2.fraction(), f)


def test_errors_payloads_and_transactions():
    """tests/liquid_volume_contract.rs:293-345 and the first-failing-cell rule"""
    # Courant limit: actual 2.0 in cell 0, state unchanged
    vel = fields((1, 1, 1))
    vel[0][:] = 2.0
    got, want, st = run_both((1, 1, 1), (1.0, 1.0, 1.0), 1000.0, [0.25], vel, 0.0, 1.0, [[0.25, 0.25]] * 3)
    assert isinstance(got, L.LiquidVolumeError) and got.kind == "CourantLimit" and got.actual == 2.0
    assert want[0] == "CourantLimit"
    assert st.fraction()[0] == 0.25 and st.stamp == (1, 0) and st.time == 0.0
    # fraction bounds from a raw source, both signs
    for rate in (1.0, -1.0):
        got, want, _ = run_both((1, 1, 1), (1.0, 1.0, 1.0), 1000.0, [0.25], fields((1, 1, 1)), 0.0, 1.0,
                                [[0.0, 0.0]] * 3, source=np.array([rate]))
        assert got.kind == want[0] == "FractionBounds"
    # divergence limit 0.25, then accepted with the relaxed limit; overfull cells fail with fraction 1.25
    vel = fields((2, 1, 1))
    vel[0][1] = 0.25
    got, want, _ = run_both((2, 1, 1), (1.0, 1.0, 1.0), 1000.0, [0.25, 0.5], vel, 0.0, 1.0, [[0.0, 0.0]] * 3)
    assert got.kind == want[0] == "DivergenceLimit" and got.actual == 0.25
    relaxed = L.LiquidVolumeSettings(1.0, 0.25)
    got, want, _ = run_both((2, 1, 1), (1.0, 1.0, 1.0), 1000.0, [0.25, 0.5], vel, 0.0, 1.0, [[0.0, 0.0]] * 3,
                            settings=relaxed)
    assert got.liquid_volume_after == 0.75
    got, want, _ = run_both((2, 1, 1), (1.0, 1.0, 1.0), 1000.0, [1.0, 1.0], vel, 0.0, 1.0, [[1.0, 1.0]] * 3,
                            settings=relaxed)
    assert got.kind == "FractionBounds" and got.actual == 1.25 and got.cell == want[2]["error_cell"]
    # several failing cells: the first in x-fastest order is reported, with its own payload
    counts = (6, 4, 3)
    f = np.full(72, 0.5)
    src = np.zeros(72)
    for c in (50, 17, 63):
        f[c] = 1.0
        src[c] = 0.5
    got, want, _ = run_both(counts, (1.0, 1.0, 1.0), 1000.0, f, fields(counts), 0.0, 1.0, [[1.0, 1.0]] * 3,
                            source=src)
    assert want[0] == "FractionBounds" and want[2]["error_cell"] == 17
    assert got.kind == "FractionBounds" and got.cell == 17 and got.actual == want[2]["error_actual"] == 1.5
    vel = fields(counts)
    vel[0][fidx(counts, 0, (1, 1, 0))] = 5.0  # outward Courant 5 in cell (0, 1, 0) = 6, before cell 17
    got, want, _ = run_both(counts, (1.0, 1.0, 1.0), 1000.0, f, vel, 0.0, 1.0, [[1.0, 1.0]] * 3, source=src,
                            settings=L.LiquidVolumeSettings(1.0, 100.0))
    assert want[0] == "CourantLimit" and want[2]["error_cell"] == 6
    assert got.kind == "CourantLimit" and got.cell == 6 and got.actual == want[2]["error_actual"] == 5.0


def test_validation_order():
    """src/liquid_volume.rs:84-96, :123-150, :185-190, :485-529"""
    counts = (3, 2, 2)
    grid = R.GridGeometry(counts)
    st = L.LiquidVolumeState(grid, 1.0, (1, 0), np.full(12, 0.5))
    z = [dev(v, np.float32) for v in fields(counts)]
    ok = L.LiquidInlet((4, 2), [[0.0, 0.0]] * 3)

    def kind(*args, **kw):
        with pytest.raises(L.LiquidVolumeError) as e:
            st.advance(*args, **kw)
        return e.value.kind

    assert kind(z, 0.0, 0.0, (2, 0), ok, SETTINGS) == "InvalidTimeStep"
    assert kind(z, 1e300, 1e-300, (2, 0), ok, SETTINGS) == "TimeResolution"
    bad = fields(counts)
    bad[1][3] = np.nan
    assert kind([dev(v, np.float32) for v in bad], 0.5, 0.5, (2, 0), L.LiquidInlet((4, 2), [[2.0, 0.0]] * 3),
                SETTINGS) == "NonFiniteVelocity"
    assert kind(z, 0.5, 0.5, (2, 0), L.LiquidInlet((4, 2), [[2.0, 0.0]] * 3), SETTINGS) == "InvalidInlet"
    nan_src = dev(np.array([np.nan] + [0.0] * 11), np.float64)
    assert kind(z, 0.5, 0.5, (2, 0), ok, SETTINGS, source=nan_src) == "InvalidSource"
    assert kind(z, 0.5, 0.5, (2, 0), ok, SETTINGS) == "TimeMismatch"
    assert kind(z, 0.0, 0.5, (2, 0), ok, L.LiquidVolumeSettings(0.0, 1.0)) == "InvalidSettings"
    assert st.stamp == (1, 0) and np.all(st.fraction() == 0.5)
    with pytest.raises(L.LiquidVolumeError) as e:
        L.LiquidVolumeState(grid, 1.0, (1, 0), np.array([0.5] * 11 + [1.5]))
    assert e.value.kind == "InvalidFraction" and e.value.cell == 11
    with pytest.raises(L.LiquidVolumeError) as e:
        L.LiquidVolumeState(grid, -1.0, (1, 0), np.full(12, 0.5))
    assert e.value.kind == "InvalidDensity"
    with pytest.raises(L.LiquidVolumeError) as e:
        L.LiquidVolumeState(grid, 1.0, (1, 0), np.full(12, 0.5), limit=100)
    assert e.value.kind == "BufferLimit"


MAXF = 1.7976931348623157e308


def blob(counts, center, radius):
    """A ball of represented liquid at 0.875 occupancy: below one, so that the
    carrier's accepted residual divergence (about 1e-9 per step) cannot push
    a full cell over one (the reference rejects that as FractionBounds)."""
    z, y, x = np.meshgrid(*[np.arange(n) + 0.5 for n in counts[::-1]], indexing="ij")
    r = np.sqrt((x - center[0]) ** 2 + (y - center[1]) ** 2 + (z - center[2]) ** 2)
    return 0.875 * np.clip(radius + 0.5 - r, 0.0, 1.0).reshape(-1)


@pytest.mark.parametrize("mixed", [False, True], ids=["jacobi_f32", "mixed"])
def test_liquid_step_moves_the_fraction_through_the_step_faces(mixed):
    """src/liquid_step.rs:828-900: the transport uses the step's corrected faces
    over [time, time + dt] and commits with the carrier."""
    counts = (24, 20, 16)
    grid = R.GridGeometry(counts)
    cfg = R.CarrierConfig.mixed(with_tracer=True) if mixed else R.CarrierConfig(storage="f32", with_tracer=True)
    sim = R.CarrierSimulation(grid, cfg)
    sim.init_fourier(seed=11)
    f = blob(counts, (12.0, 10.0, 8.0), 5.0)
    lts = L.LiquidTransportSimulation(sim, 800.0, (41, 0), f, flow_id=43)
    inlet = L.LiquidInlet((4, 0), [[0.0, 0.0]] * 3)
    settings = L.LiquidVolumeSettings(1.0, 1e-3)
    og = O.grid(counts)
    t = 0.0
    for k in range(3):
        r = lts.step(R.StepParams(requested_dt=MAXF, cfl=0.5), inlet, settings)
        faces = sim.download()
        err, f2, want = O.liquid_advance(og, 800.0, f, faces, t, r.carrier.dt, inlet.fraction,
                                         max_outward_courant=1.0, actual_divergence_limit=1e-3)
        assert err == "Ok"
        assert np.array_equal(lts.fraction().view(np.uint64), f2.view(np.uint64))
        same_report(r.liquid, want)
        assert r.liquid.flow == (43, r.carrier.generation) and r.liquid.stamp == (41, k + 1)
        assert r.liquid.time == r.carrier.time == lts.time
        f, t = f2, r.liquid.time
    assert abs(want["liquid_volume_after"] - blob(counts, (12.0, 10.0, 8.0), 5.0).sum()) < 1e-9


def test_rejected_transport_rejects_the_whole_step():
    counts = (16, 12, 10)
    grid = R.GridGeometry(counts)
    sim = R.CarrierSimulation(grid, R.CarrierConfig(storage="f32"))
    sim.init_fourier(seed=5)
    f = blob(counts, (8.0, 6.0, 5.0), 3.0)
    lts = L.LiquidTransportSimulation(sim, 1000.0, (41, 0), f, flow_id=43)
    before_faces = sim.download()
    inlet = L.LiquidInlet((4, 0), [[0.0, 0.0]] * 3)
    prm = R.StepParams(requested_dt=MAXF, cfl=0.5)
    with pytest.raises(L.LiquidVolumeError) as e:
        lts.step(prm, inlet, L.LiquidVolumeSettings(1e-6, 1e-3))
    assert e.value.kind == "CourantLimit" and e.value.limit == 1e-6
    with pytest.raises(L.LiquidVolumeError) as e:
        lts.step(prm, L.LiquidInlet((4, 0), [[0.0, 2.0]] * 3), L.LiquidVolumeSettings(1.0, 1e-3))
    assert e.value.kind == "InvalidInlet"
    # neither state moved
    after = sim.download()
    assert all(np.array_equal(a.view(np.uint32), b.view(np.uint32)) for a, b in zip(before_faces, after))
    assert lts.stamp == (41, 0) and lts.time == 0.0 and np.array_equal(lts.fraction(), f)
    r = lts.step(prm, inlet, L.LiquidVolumeSettings(1.0, 1e-3))
    assert r.carrier.generation == 1 and r.liquid.stamp == (41, 1) and lts.time == r.carrier.time


def test_dense3d_frame_carries_the_liquid_fraction():
    from rheon_b200 import dense3d as D

    counts = (12, 10, 8)
    grid = R.GridGeometry(counts)
    sim = R.CarrierSimulation(grid, R.CarrierConfig(storage="f32", with_tracer=True))
    sim.init_fourier(seed=3)
    lts = L.LiquidTransportSimulation(sim, 800.0, (41, 0), blob(counts, (6.0, 5.0, 4.0), 2.5), flow_id=43)
    r = lts.step(R.StepParams(requested_dt=MAXF, cfl=0.5), L.LiquidInlet((4, 0), [[0.0, 0.0]] * 3),
                 L.LiquidVolumeSettings(1.0, 1e-3))
    info = D.Dense3dFrameInfo(frame=1, time_s=r.carrier.time, dt_s=r.carrier.dt, carrier_stamp=(43, 1),
                              liquid_stamp=r.liquid.stamp,
                              diagnostics=dict(pressure_iterations=r.carrier.pressure.iterations,
                                               volume_before_m3=r.liquid.liquid_volume_before,
                                               volume_after_m3=r.liquid.liquid_volume_after,
                                               mass_after_kg=r.liquid.liquid_mass_after))
    line = D.Dense3dEncoder(grid).encode(info, D.Dense3dFields.from_carrier(sim))
    faces, tracer = sim.download(with_tracer=True)
    st, want = O.dense3d_frame_text(O.grid(counts), frame=1, time_s=r.carrier.time, dt_s=r.carrier.dt,
                                    carrier_stamp=(43, 1), liquid_stamp=r.liquid.stamp, diagnostics=info.diagnostics,
                                    faces=faces, tracer=tracer, fraction=lts.fraction(), pressure=sim.pressure())
    assert st == 0 and line == want


# ---- periodic boundary (src/liquid_volume.rs:389-406)

def periodic_both(counts, spacing, density, fraction, vel, dt, source=None, settings=L.LiquidVolumeSettings(1.0, 0.0)):
    grid = R.GridGeometry(counts, spacing)
    st = L.LiquidVolumeState(grid, density, (1, 0), np.asarray(fraction, np.float64))
    want = O.liquid_advance(O.grid(counts, spacing), density, fraction, vel, 0.0, dt, [[0.0, 0.0]] * 3, source=source,
                            max_outward_courant=settings.max_outward_courant,
                            actual_divergence_limit=settings.actual_divergence_limit, periodic=True)
    try:
        got = st.advance_periodic([dev(v, np.float32) for v in vel], 0.0, dt, (2, 0), (9, 0), settings,
                                  source=dev(source, np.float64) if source is not None else None, source_stamp=(3, 0))
    except L.LiquidVolumeError as e:
        got = e
    return got, want, st


def uniform(counts, u):
    g = O.grid(counts)
    return [np.full(O.face_len(g, d), u[d], np.float32) for d in range(3)]


def test_periodic_known_answers():
    """tests/liquid_volume_periodic_contract.rs:17-68, 122-156"""
    init = [0.0, 0.25, 0.5, 1.0, 0.75, 0.125, 0.625, 0.875]
    got, want, st = periodic_both((2, 2, 2), (0.5, 0.5, 0.5), 998.2, init, uniform((2, 2, 2), [0.25, -0.125, 0.0625]),
                                  0.25)
    assert want[0] == "Ok" and got.periodic and got.inlet == (9, 0)
    assert np.array_equal(st.fraction(), want[1])
    assert got.inward_boundary_volume == 0.0 and got.outward_boundary_volume == 0.0
    got, want, st = periodic_both((1, 1, 1), (1.0, 1.0, 1.0), 2.0, [0.25], uniform((1, 1, 1), [-0.5, 0.25, -0.125]),
                                  0.25, source=np.array([0.5]))
    assert list(st.fraction()) == [0.375] and got.source_volume == 0.125 and got.volume_balance_error == 0.0
    for d in range(3):
        for sign in (-1.0, 1.0):
            counts = [1, 1, 1]
            counts[d] = 3
            spacing = [1.0, 1.0, 1.0]
            spacing[d] = 1.0 / 3.0
            speed = [0.0, 0.0, 0.0]
            speed[d] = sign
            got, want, st = periodic_both(tuple(counts), tuple(spacing), 1.0, [1.0, 0.0, 0.0],
                                          uniform(tuple(counts), speed), spacing[d] * 0.5)
            assert np.array_equal(st.fraction(), want[1])
            exact = [0.5, 0.5, 0.0] if sign > 0 else [0.5, 0.0, 0.5]
            assert all(abs(a - b) < 1e-14 for a, b in zip(st.fraction(), exact))


def test_periodic_seam_mismatch_and_random_parity():
    """tests/liquid_volume_periodic_contract.rs:69-104; random periodic flows bit for bit"""
    u = uniform((2, 2, 2), [0.25, 0.0, 0.0])
    u[0][2] = 0.125
    got, want, st = periodic_both((2, 2, 2), (0.5, 0.5, 0.5), 998.2, [0.5] * 8, u, 0.25)
    assert want[0] == got.kind == "PeriodicVelocityMismatch" and got.cell == 0 and got.actual == 0.0
    assert np.all(st.fraction() == 0.5) and st.time == 0.0
    u[1][fidx((2, 2, 2), 1, (1, 2, 1))] = 0.5  # a Y seam too: the X seam comes first
    got, want, _ = periodic_both((2, 2, 2), (0.5, 0.5, 0.5), 998.2, [0.5] * 8, u, 0.25)
    assert got.kind == "PeriodicVelocityMismatch" and got.actual == 0.0
    u = uniform((2, 2, 2), [0.25, 0.0, 0.0])
    got, _, _ = periodic_both((2, 2, 2), (0.5, 0.5, 0.5), 998.2, [0.5] * 8, u, 10.0)
    assert got.kind == "CourantLimit"
    for counts in [(8, 6, 5), (17, 12, 9)]:
        rng = np.random.default_rng(sum(counts))
        g = O.grid(counts, (0.5, 0.75, 1.25))
        vel = [rng.uniform(-0.05, 0.05, O.face_len(g, a)).astype(np.float32) for a in range(3)]
        for d in range(3):  # make every seam consistent: upper face = lower face
            fc = list(counts)
            fc[d] += 1
            arr = vel[d].reshape(fc[2], fc[1], fc[0])
            sl_lo = [slice(None)] * 3
            sl_hi = [slice(None)] * 3
            sl_lo[2 - d] = 0
            sl_hi[2 - d] = counts[d]
            arr[tuple(sl_hi)] = arr[tuple(sl_lo)]
        f = rng.uniform(0.2, 0.8, int(np.prod(counts)))
        src = rng.uniform(-1e-3, 1e-3, f.size)
        got, want, st = periodic_both(counts, (0.5, 0.75, 1.25), 800.0, f, vel, 0.05, source=src,
                                      settings=L.LiquidVolumeSettings(1.0, 10.0))
        assert want[0] == "Ok", want[0]
        assert np.array_equal(st.fraction().view(np.uint64), want[1].view(np.uint64))
        same_report(got, want[2])


# ------------------------------------------------------------------ cancellation stages
def _stage_sequence(counts, periodic):
    """The reference's VolumeStage sequence of one accepted interval
    (prepare_with_boundary, src/liquid_volume.rs:558-830)."""
    flux = (counts[2] + 0) * 2 + (counts[2] + 1)   # z planes of the X, Y and Z face arrays
    seq = ["BeforeFlux"] + ["FaceFluxSlice"] * (flux * (2 if periodic else 1))
    return seq + ["CellUpdateSlice"] * counts[2] + ["BeforeCommit"]


@pytest.mark.parametrize("periodic", [False, True], ids=["inlet", "periodic"])
def test_cancellation_stages_leave_the_state_untouched(periodic):
    """VolumeStage (src/liquid_volume.rs:18-23) polled at :568, 578, 610, 689,
    830: the callback sees the reference's sequence; a cancel at any point
    ends the interval with Cancelled { stage } and the accepted fraction,
    stamp and time unchanged; a retry equals a fresh run bit for bit."""
    counts = (12, 10, 6)
    rng = np.random.default_rng(7)
    spacing = (0.5, 0.75, 1.25)
    grid = R.GridGeometry(counts, spacing)
    g = O.grid(counts, spacing)
    f = rng.uniform(0.2, 0.8, int(np.prod(counts)))
    vel = [rng.uniform(-0.05, 0.05, O.face_len(g, a)).astype(np.float32) for a in range(3)]
    if periodic:  # equal velocities on the two faces of every seam
        for a in range(3):
            fc = list(counts)
            fc[a] += 1
            v = vel[a].reshape(fc[2], fc[1], fc[0])
            if a == 0:
                v[:, :, -1] = v[:, :, 0]
            elif a == 1:
                v[:, -1, :] = v[:, 0, :]
            else:
                v[-1, :, :] = v[0, :, :]
    dv = [dev(v, np.float32) for v in vel]
    inlet = L.LiquidInlet((4, 2), [[0.25, 0.5], [0.0, 1.0], [0.125, 0.75]])
    settings = L.LiquidVolumeSettings(1.0, 10.0)

    def run(state, cancel=None):
        if periodic:
            return state.advance_periodic(dv, 0.0, 0.05, (2, 0), (6, 1), settings, cancel=cancel)
        return state.advance(dv, 0.0, 0.05, (2, 0), inlet, settings, cancel=cancel)

    fresh = L.LiquidVolumeState(grid, 800.0, (5, 0), f)
    seen = []
    want = run(fresh, cancel=lambda s: seen.append(s) or False)
    assert seen == _stage_sequence(counts, periodic)
    want_f = fresh.fraction()
    st = L.LiquidVolumeState(grid, 800.0, (5, 0), f)
    for at in sorted({0, 1, len(seen) // 2, len(seen) - 2, len(seen) - 1}):
        calls = []

        def cancel(s, at=at):
            calls.append(s)
            return len(calls) - 1 == at

        with pytest.raises(L.LiquidVolumeError) as e:
            run(st, cancel=cancel)
        assert e.value.kind == "Cancelled" and e.value.stage == seen[at]
        assert calls == seen[: at + 1]
        assert np.array_equal(st.fraction(), f) and st.stamp == (5, 0) and st.time == 0.0
    got = run(st)
    assert np.array_equal(st.fraction().view(np.uint64), want_f.view(np.uint64))
    assert got.stamp == want.stamp == (5, 1)


def test_an_error_before_a_cancellation_point_wins():
    """A cell's Courant failure lies in its z plane's CellUpdateSlice: the
    reference reports it without asking the later points."""
    counts = (6, 4, 3)
    vel = fields(counts)
    vel[0][fidx(counts, 0, (1, 1, 1))] = 5.0   # outward Courant 5 in cell (0, 1, 1), z plane 1
    grid = R.GridGeometry(counts)
    st = L.LiquidVolumeState(grid, 1000.0, (1, 0), np.full(72, 0.5))
    calls = []
    with pytest.raises(L.LiquidVolumeError) as e:
        st.advance([dev(v, np.float32) for v in vel], 0.0, 1.0, (2, 3), L.LiquidInlet((4, 2), [[0.5, 0.5]] * 3),
                   L.LiquidVolumeSettings(1.0, 100.0), cancel=lambda s: calls.append(s) or False)
    assert e.value.kind == "CourantLimit" and e.value.cell == 6 + 24
    flux = 3 * 2 + 4
    assert calls == ["BeforeFlux"] + ["FaceFluxSlice"] * flux + ["CellUpdateSlice"] * 2
