"""dense3D frames encoded on the device, compared byte for byte with the oracle.

write_dense3d_frame (src/dense3d_sequence.rs:412-564) is the contract: every
byte of the device line must equal the oracle's line for the same state. The
stream tests follow Dense3dSequence's output rules (src/dense3d_sequence.rs:
90-120, 224-341): limits, ordered frames, terminal errors, no bytes from a
rejected frame. The reference's fixture shape (16x8x4, spacing
0.0625/0.125/0.25; docs/implementation/dense3d-sequence.md) is one of the
grids.
"""
import json
import os
import struct

import numpy as np
import pytest

import oracle as O
import rheon_b200 as R
from rheon_b200 import dense3d as D

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _device():
    if not torch.cuda.is_available() or R.device_count() == 0:
        pytest.skip("no B200")
    yield
    torch.cuda.synchronize()


DIAG = dict(pressure_iterations=504, pressure_residual_m3_s2=1.5e-9, carrier_divergence_s_inv=3.25e-7,
            liquid_divergence_s_inv=2.0e-7, volume_before_m3=0.125, volume_after_m3=0.125, mass_after_kg=100.0,
            inward_m3=0.0, outward_m3=1e-300, source_m3=0.0, balance_m3=-1.3877787807814457e-17,
            rounding_budget_m3=4.440892098500626e-16)


def special_f32(n, rng):
    """Values that stress the digit routine: ties at the tenth digit,
    subnormals, extremes, powers of ten, signed zeros."""
    vals = [0.0, -0.0, 1.0, -1.0, 1048575.9375, 16777215.0, 3.4028234663852886e38, 1.1754943508222875e-38,
            1.401298464324817e-45, 1e-45, 1e38, 0.1, 1e-7, 123456.789]
    vals += [float(np.float32(rng.integers(1, 2 ** 24) * 2.0 ** -int(rng.integers(0, 12)))) for _ in range(64)]
    out = rng.uniform(-3, 3, n).astype(np.float32)
    k = min(n, len(vals))
    out[:k] = np.array(vals[:k], np.float32)
    return out


def special_f64(n, rng):
    vals = [0.0, -0.0, 5e-324, 2.2250738585072014e-308, 1.7976931348623157e308, 1e18, 1e17, 1e-300, 0.1,
            9.999999999999999e22, 1048576.0625, -123456789012345678.0]
    out = rng.normal(0, 1e3, n)
    k = min(n, len(vals))
    out[:k] = vals[:k]
    return out


def state(counts, seed, f64_faces=False, tracer=True, fraction=True, special=True):
    rng = np.random.default_rng(seed)
    g = O.grid(counts)
    n = int(np.prod(counts))
    faces = []
    for a in range(3):
        m = O.face_len(g, a)
        f = special_f32(m, rng) if special else rng.uniform(-2, 2, m).astype(np.float32)
        faces.append(f.astype(np.float64) + (rng.uniform(-1e-9, 1e-9, m) if f64_faces else 0.0)
                     if f64_faces else f)
    tr = rng.uniform(0, 1, n).astype(np.float32) if tracer else None
    fr = np.clip(rng.uniform(-0.1, 1.1, n), 0.0, 1.0) if fraction else None
    p = special_f64(n, rng) if special else rng.normal(0, 1, n)
    return faces, tr, fr, p


def device_fields(faces, tr, fr, p):
    ts = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in faces]
    return D.Dense3dFields.from_tensors(ts[0], ts[1], ts[2],
                                        torch.from_numpy(tr).cuda() if tr is not None else None,
                                        torch.from_numpy(fr).cuda() if fr is not None else None,
                                        torch.from_numpy(p).cuda() if p is not None else None)


def oracle_line(counts, info: D.Dense3dFrameInfo, faces, tr, fr, p):
    f32 = [np.asarray(f, dtype=np.float32) for f in faces]  # f64 faces print as the f32 they round to
    st, line = O.dense3d_frame_text(O.grid(counts), frame=info.frame, time_s=info.time_s, dt_s=info.dt_s,
                                    carrier_stamp=info.carrier_stamp, liquid_stamp=info.liquid_stamp,
                                    diagnostics=info.diagnostics, faces=f32, tracer=tr, fraction=fr, pressure=p)
    assert st == 0
    return line


GRIDS = [(16, 8, 4), (1, 1, 1), (17, 10, 9), (33, 7, 5), (64, 48, 40)]


@pytest.mark.parametrize("counts", GRIDS, ids=str)
@pytest.mark.parametrize("f64_faces", [False, True], ids=["f32faces", "f64faces"])
def test_device_frame_is_byte_identical(counts, f64_faces):
    faces, tr, fr, p = state(counts, seed=sum(counts), f64_faces=f64_faces)
    info = D.Dense3dFrameInfo(frame=7, time_s=0.4375, dt_s=0.0625, carrier_stamp=(43, 7), liquid_stamp=(41, 7),
                              diagnostics=DIAG)
    enc = D.Dense3dEncoder(R.GridGeometry(counts))
    got = enc.encode(info, device_fields(faces, tr, fr, p))
    want = oracle_line(counts, info, faces, tr, fr, p)
    assert len(got) <= enc.bound()
    assert got == want


@pytest.mark.parametrize("counts", [(16, 8, 4), (9, 5, 3)], ids=str)
def test_constructor_frame_with_absent_fields(counts):
    faces, _, _, _ = state(counts, seed=5)
    info = D.Dense3dFrameInfo(carrier_stamp=(43, 0), liquid_stamp=(41, 0))
    enc = D.Dense3dEncoder(R.GridGeometry(counts))
    got = enc.encode(info, device_fields(faces, None, None, None))
    want = oracle_line(counts, info, faces, None, None, np.zeros(int(np.prod(counts))))
    assert got == want
    obj = json.loads(got)
    assert obj["diagnostics"] is None and set(obj["fields"]["pressure"]) == {0.0}


def test_rejected_frames_write_no_bytes():
    counts = (12, 6, 5)
    enc = D.Dense3dEncoder(R.GridGeometry(counts))
    faces, tr, fr, p = state(counts, seed=11)
    info = D.Dense3dFrameInfo(frame=1, time_s=0.25, dt_s=0.25, diagnostics=DIAG)
    out = torch.full((enc.bound(),), 0x5A, dtype=torch.uint8, device="cuda")
    cases = []
    bad = [f.copy() for f in faces]
    bad[2][17] = np.nan
    cases.append(("nonfinite velocity", (bad, tr, fr, p)))
    badp = p.copy()
    badp[3] = np.inf
    cases.append(("nonfinite or invalid cell field", (faces, tr, fr, badp)))
    badf = fr.copy()
    badf[0] = 1.0000000000000002
    cases.append(("nonfinite or invalid cell field", (faces, tr, badf, p)))
    badt = tr.copy()
    badt[-1] = np.float32(np.inf)
    cases.append(("nonfinite or invalid cell field", (faces, badt, fr, p)))
    for message, st in cases:
        with pytest.raises(D.Dense3dError) as e:
            enc.encode_into(info, device_fields(*st), out.data_ptr(), out.numel())
        assert e.value.kind == "InvalidState" and message in str(e.value)
    with pytest.raises(D.Dense3dError) as e:  # report continuity: a finite, positive dt
        enc.encode_into(D.Dense3dFrameInfo(frame=1, time_s=0.25, dt_s=0.0, diagnostics=DIAG),
                        device_fields(faces, tr, fr, p), out.data_ptr(), out.numel())
    assert e.value.kind == "InvalidState"
    assert bool((out == 0x5A).all())
    with pytest.raises(D.Dense3dError) as e:  # too small a buffer: nothing written either
        enc.encode_into(info, device_fields(faces, tr, fr, p), out.data_ptr(), 100)
    assert e.value.kind == "Limit"
    assert bool((out == 0x5A).all())


def test_frame_stream_limits_and_terminal_errors(tmp_path):
    counts = (16, 8, 4)
    grid = R.GridGeometry(counts, (0.0625, 0.125, 0.25))
    faces, tr, fr, p = state(counts, seed=2, special=False)
    fields = device_fields(faces, tr, fr, p)
    zero = device_fields(faces, tr, fr, None)
    infos = [D.Dense3dFrameInfo(carrier_stamp=(43, 0), liquid_stamp=(41, 0))]
    for k in range(1, 4):
        infos.append(D.Dense3dFrameInfo(frame=k, time_s=0.0625 * k, dt_s=0.0625, carrier_stamp=(43, k),
                                        liquid_stamp=(41, k), diagnostics=dict(DIAG, pressure_iterations=k)))
    lines = [oracle_line(counts, infos[0], faces, tr, fr, np.zeros(512))]
    lines += [oracle_line(counts, i, faces, tr, fr, p) for i in infos[1:]]
    path = tmp_path / "frames.jsonl"
    with D.Dense3dFrameWriter(grid, str(path), D.Dense3dLimits(512, 3, 1 << 20)) as w:
        w.write_frame(infos[0], zero)
        w.write_frame(infos[1], fields)
        w.write_frame(infos[2], fields)
        w.flush()
        assert w.frame_count() == 3 and w.bytes_written() == sum(len(x) for x in lines[:3])
        with pytest.raises(D.Dense3dError) as e:  # the frame limit includes the constructor frame
            w.write_frame(infos[3], fields)
        assert e.value.kind == "Limit" and w.is_aborted()
        with pytest.raises(D.Dense3dError) as e:
            w.write_frame(infos[3], fields)
        assert e.value.kind == "Aborted"
    assert path.read_bytes() == b"".join(lines[:3])
    with pytest.raises(FileExistsError):  # never overwrite
        D.Dense3dFrameWriter(grid, str(path), D.Dense3dLimits(512, 3, 1 << 20))
    # byte budget: the second frame does not fit; nothing of it is written
    budget = len(lines[0]) + len(lines[1]) - 1
    p2 = tmp_path / "budget.jsonl"
    with D.Dense3dFrameWriter(grid, str(p2), D.Dense3dLimits(512, 9, budget)) as w:
        w.write_frame(infos[0], zero)
        with pytest.raises(D.Dense3dError) as e:
            w.write_frame(infos[1], fields)
        assert e.value.kind == "Io" and "budget" in str(e.value)
    assert p2.read_bytes() == lines[0]
    # frames out of order, a preflight failure: terminal too
    with D.Dense3dFrameWriter(grid, str(tmp_path / "order.jsonl"), D.Dense3dLimits(512, 9, 1 << 20)) as w:
        with pytest.raises(D.Dense3dError) as e:
            w.write_frame(infos[1], fields)
        assert e.value.kind == "InvalidState" and w.is_aborted()
    # a failed write (the pipe's reader is gone) surfaces at the next call and is terminal
    r, wfd = os.pipe()
    os.close(r)
    w = D.Dense3dFrameWriter(grid, wfd, D.Dense3dLimits(512, 9, 1 << 20))
    w.write_frame(infos[0], zero)
    with pytest.raises(D.Dense3dError) as e:
        w.flush()
    assert e.value.kind == "Io" and w.is_aborted()
    with pytest.raises(D.Dense3dError):
        w.write_frame(infos[1], fields)
    w.close()
    os.close(wfd)
    # creation limits (Dense3dSequence::new): zero frames or bytes, too many cells
    for lim in (D.Dense3dLimits(512, 0, 10), D.Dense3dLimits(512, 3, 0), D.Dense3dLimits(511, 3, 10)):
        with pytest.raises(D.Dense3dError) as e:
            D.Dense3dFrameWriter(grid, os.open(os.devnull, os.O_WRONLY), lim)
        assert e.value.kind == "Limit"


@pytest.mark.parametrize("storage", ["f32", "f64"])
def test_carrier_frames_match_the_oracle(storage, tmp_path):
    counts = (24, 16, 12)
    grid = R.GridGeometry(counts)
    sim = R.CarrierSimulation(grid, R.CarrierConfig(storage=storage, with_tracer=True))
    sim.init_fourier(seed=7)
    faces0, tr0 = sim.download(with_tracer=True)
    path = tmp_path / f"carrier_{storage}.jsonl"
    expect = []
    with D.Dense3dFrameWriter(grid, str(path), D.Dense3dLimits(1 << 20, 4, 1 << 26)) as w:
        info = D.Dense3dFrameInfo(carrier_stamp=(1, 0), liquid_stamp=(2, 0))
        w.write_frame(info, D.Dense3dFields.from_carrier(sim))
        expect.append(oracle_line(counts, info, faces0, tr0, None, np.zeros(grid.cell_len())))
        for k in range(1, 4):
            rep = sim.step(R.StepParams(requested_dt=0.02, cfl=0.5))
            faces, tr = sim.download(with_tracer=True)
            p = sim.pressure()
            info = D.Dense3dFrameInfo(frame=k, time_s=rep.time, dt_s=rep.dt, carrier_stamp=(1, rep.generation),
                                      liquid_stamp=(2, rep.generation),
                                      diagnostics=dict(pressure_iterations=rep.pressure.iterations,
                                                       pressure_residual_m3_s2=rep.pressure.true_residual_max,
                                                       carrier_divergence_s_inv=rep.actual_divergence_max))
            w.write_frame(info, D.Dense3dFields.from_carrier(sim))
            expect.append(oracle_line(counts, info, faces, tr, None, p))
    assert path.read_bytes() == b"".join(expect)
