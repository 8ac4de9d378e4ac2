"""dense3D frame text on the CPU: the oracle and the library's number routine.

The frame format is write_dense3d_frame (src/dense3d_sequence.rs:412-564):
Rust's `{:.9e}` for the f32 fields and `{:.17e}` for the f64 ones. Python's
'%.*e' is correctly rounded (ties to even on the exact binary value), like
Rust's LowerExp with a precision; only the exponent spelling differs. The
oracle (glibc "%.*e") and the encoder's own digit routine (run here through
its host build) are both checked against it. Device frames are compared with
the oracle in test_gpu_dense3d.py.
"""
import json
import random
import struct

import numpy as np
import pytest

import oracle as O
from rheon_b200 import dense3d as D


def rust_exp(x: float, precision: int) -> str:
    m, e = ("%.*e" % (precision, x)).split("e")
    return f"{m}e{int(e)}"


def f32(bits: int) -> float:
    return struct.unpack("<f", struct.pack("<I", bits))[0]


def f64(bits: int) -> float:
    return struct.unpack("<d", struct.pack("<Q", bits))[0]


# Rust's own spellings: tests/dense3d_controls_contract.rs:196 ("0.00000000000000000e0"
# for 0.0 with {:.17e}) and the LowerExp rules (no '+', no exponent padding, -0.0 signed).
KNOWN = [
    (0.0, 17, "0.00000000000000000e0"),
    (0.0625, 17, "6.25000000000000000e-2"),
    (0.5, 17, "5.00000000000000000e-1"),
    (1.0, 9, "1.000000000e0"),
    (-0.0, 9, "-0.000000000e0"),
    (1e21, 17, "1.00000000000000000e21"),
    (5e-324, 17, "4.94065645841246544e-324"),
]


@pytest.mark.parametrize("x,precision,text", KNOWN)
def test_known_spellings(x, precision, text):
    assert rust_exp(x, precision) == text
    got = D.text_f64(x) if precision == 17 else D.text_f32(x)
    assert got == text


def test_library_digits_match_correct_rounding():
    rng = random.Random(20261203)
    xs = [f64(rng.getrandbits(64) & 0x7FEFFFFFFFFFFFFF | rng.getrandbits(1) << 63) for _ in range(20000)]
    xs += [10.0 ** k for k in range(-300, 301)] + [float(rng.randint(1, 10 ** 19)) for _ in range(2000)]
    xs += [5e-324, 2.2250738585072014e-308, 1.7976931348623157e308, 1e18, 1e17, 9.999999999999999e22]
    for x in xs:
        assert D.text_f64(x) == rust_exp(x, 17), x
    ys = [f32(rng.getrandbits(32) & 0x7F7FFFFF | rng.getrandbits(1) << 31) for _ in range(20000)]
    # exact ties at the tenth digit: m 2^-k with few significant decimal digits
    ys += [float(np.float32(rng.randint(1, 2 ** 24 - 1) * 2.0 ** -rng.randint(0, 12))) for _ in range(20000)]
    ys += [1048575.9375, 16777215.0, f32(1), f32(0x7F7FFFFF), f32(0x00800000)]
    for y in ys:
        assert D.text_f32(y) == rust_exp(y, 9), y


def test_ties_round_to_even():
    # 1048575.9375 = 1.0485759375e6 exactly: a tie at the tenth digit (odd 7 rounds up)
    assert D.text_f32(1048575.9375) == "1.048575938e6"
    # 1048576.0625 is not representable as f32; 2^20 + 2^-4 in f64 keeps 18 digits exactly
    assert rust_exp(1048576.0625, 17) == D.text_f64(1048576.0625)


def small_state(counts, seed=3, with_tracer=True, with_fraction=True):
    rng = np.random.default_rng(seed)
    n = int(np.prod(counts))
    faces = [rng.uniform(-2, 2, O.face_len(O.grid(counts), a)).astype(np.float32) for a in range(3)]
    faces[0][0] = -0.0
    tracer = rng.uniform(0, 1, n).astype(np.float32) if with_tracer else None
    fraction = rng.uniform(0, 1, n) if with_fraction else None
    pressure = rng.normal(0, 1e3, n)
    pressure[0] = 0.0
    return faces, tracer, fraction, pressure


DIAG = dict(pressure_iterations=42, pressure_residual_m3_s2=1.5e-9, carrier_divergence_s_inv=3.25e-7,
            liquid_divergence_s_inv=2.0e-7, volume_before_m3=0.125, volume_after_m3=0.125, mass_after_kg=100.0,
            inward_m3=0.0, outward_m3=0.0, source_m3=0.0, balance_m3=-1.3877787807814457e-17,
            rounding_budget_m3=4.440892098500626e-16)


def test_oracle_frame_layout_and_round_trip():
    counts = (16, 8, 4)
    g = O.grid(counts, (0.0625, 0.125, 0.25))
    faces, tracer, fraction, pressure = small_state(counts)
    st, line = O.dense3d_frame_text(g, frame=3, time_s=0.1875, dt_s=0.0625, carrier_stamp=(43, 3),
                                    liquid_stamp=(41, 3), diagnostics=DIAG, faces=faces, tracer=tracer,
                                    fraction=fraction, pressure=pressure)
    assert st == 0
    assert line.endswith(b"}\n") and line.count(b"\n") == 1
    obj = json.loads(line)
    assert list(obj) == ["frame", "time_s", "dt_s", "carrier_stamp", "liquid_stamp", "fields", "diagnostics"]
    assert obj["carrier_stamp"] == {"id": "43", "version": "3"}
    assert obj["liquid_stamp"] == {"id": "41", "version": "3"}
    assert list(obj["fields"]) == ["velocity_x", "velocity_y", "velocity_z", "tracer", "fraction", "pressure"]
    for a, name in enumerate(["velocity_x", "velocity_y", "velocity_z"]):
        got = np.array(obj["fields"][name], dtype=np.float32)
        assert got.size == faces[a].size and np.array_equal(got.view(np.uint32)[1:], faces[a].view(np.uint32)[1:])
    assert np.array_equal(np.array(obj["fields"]["tracer"], np.float32), tracer)
    assert np.array_equal(np.array(obj["fields"]["fraction"], np.float64), fraction)
    assert np.array_equal(np.array(obj["fields"]["pressure"], np.float64), pressure)
    assert list(obj["diagnostics"]) == ["pressure_iterations"] + list(O.DENSE3D_DIAGNOSTICS)
    text = line.decode()
    assert '"velocity_x":[-0.000000000e0,' in text
    assert '"time_s":1.87500000000000000e-1,"dt_s":6.25000000000000000e-2,' in text
    for v in pressure[:50]:
        assert rust_exp(float(v), 17) in text


def test_oracle_constructor_frame_and_preflight():
    counts = (5, 3, 2)
    g = O.grid(counts)
    faces, tracer, fraction, pressure = small_state(counts, with_tracer=False, with_fraction=False)
    st, line = O.dense3d_frame_text(g, faces=faces, pressure=np.zeros(30))
    assert st == 0
    obj = json.loads(line)
    assert obj["diagnostics"] is None and obj["dt_s"] == 0.0
    assert '"dt_s":0.00000000000000000e0' in line.decode()
    assert all(t == "0.000000000e0" for t in line.decode().split('"tracer":[')[1].split("]")[0].split(","))
    # a constructor frame must be frame 0 at time 0 (src/dense3d_sequence.rs:487-492)
    assert O.dense3d_frame_text(g, frame=1, faces=faces)[0] == 23
    bad = [f.copy() for f in faces]
    bad[1][2] = np.inf
    assert O.dense3d_frame_text(g, faces=bad)[0] == 23
    assert O.dense3d_frame_text(g, faces=faces, fraction=np.full(30, 1.5))[0] == 23
    assert O.dense3d_frame_text(g, faces=faces, time_s=0.5, diagnostics=dict(DIAG, mass_after_kg=np.nan),
                                dt_s=0.5)[0] == 23
