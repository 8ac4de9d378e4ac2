"""Host-side checks of the C ABI and the input generators (no GPU needed)."""
import ctypes as C
import os
import re

import numpy as np

import rheon_b200 as R
from rheon_b200 import _native as N
from rheon_b200 import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "rheon_b200.h")


def declared_symbols():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"RB200_API [^;(]*?\b(rb200_[a-z0-9_]+)\s*\(", src)))


def test_library_loads_and_exports_every_declared_symbol():
    lib = N.lib()
    names = declared_symbols()
    assert len(names) >= 30
    for name in names:
        assert hasattr(lib, name), name
    # and the Python declarations cover exactly the header
    assert sorted(N.SIGNATURES) == names


def test_abi_version_and_status_strings():
    lib = N.lib()
    assert lib.rb200_abi_version() == 1
    for code in range(0, 19):
        assert lib.rb200_status_string(code)
    assert lib.rb200_status_string(999) == b"unknown status"


def test_struct_layouts_match_the_header():
    # Sizes of the C structs as declared in include/rheon_b200.h (x86-64).
    assert C.sizeof(N.Grid) == 72
    assert C.sizeof(N.Settings) == 32
    assert C.sizeof(N.Report) == 56
    assert C.sizeof(N.Trace) == 48
    assert C.sizeof(N.Request) == 72 + 8 + 8 + 8 + 8
    assert C.sizeof(N.StepParams) == 32
    assert C.sizeof(N.BatchConfig) == 8 + 32 + 8 + 8 + 4 + 4


def test_device_count_without_gpu_is_safe():
    # On a host without an sm_100 device this is 0; on the box it is >= 1.
    assert R.device_count() >= 0


def test_creation_without_device_fails_cleanly():
    if R.device_count() > 0:
        return
    g = R.GridGeometry([4, 4, 4])
    try:
        R.PressureWorkspace(g, 1 << 30)
    except R.PressureError as e:
        assert e.kind in ("NoDevice", "Execution")
    else:
        raise AssertionError("workspace creation must fail without a device")


def test_invalid_grids_are_rejected_before_touching_a_device():
    lib = N.lib()
    g = R.GridGeometry([4, 4, 4]).c()
    g.counts[1] = 0
    h = C.c_void_p()
    assert lib.rb200_workspace_create(C.byref(g), 1.0, 0, 1 << 30, 0, C.byref(h)) == N.INVALID_ARGUMENT
    g = R.GridGeometry([4, 4, 4]).c()
    assert lib.rb200_workspace_create(C.byref(g), -1.0, 0, 1 << 30, 0, C.byref(h)) == N.INVALID_ARGUMENT
    assert lib.rb200_workspace_create(C.byref(g), 1.0, 0, 10, 0, C.byref(h)) == N.OUT_OF_MEMORY


def test_splitmix_inputs_are_deterministic_and_walls_zero():
    n = (5, 4, 3)
    a = W.uniform_faces(n, seed=7)
    b = W.uniform_faces(n, seed=7)
    for d in range(3):
        assert np.array_equal(a[d], b[d])
        assert np.all(a[d][W.wall_mask(n, d)] == 0.0)
        assert np.all(np.abs(a[d]) <= 1.0)
    f = W.fourier_faces((8, 8, 8), seed=3)
    for d in range(3):
        assert np.all(f[d][W.wall_mask((8, 8, 8), d)] == 0.0)
    k, phase, amp = W.fourier_modes(3)
    assert k.min() >= 1 and k.max() <= 8
    assert np.allclose(np.sum(amp * amp, axis=1), 1.0)


def test_splitmix64_known_values():
    # SplitMix64 reference outputs for state increments from 0.
    assert int(W.splitmix64(np.array([0], np.uint64))[0]) == 0xE220A8397B1DCDAF
    assert int(W.splitmix64(np.array([0x9E3779B97F4A7C15], np.uint64))[0]) == 0x6E789E6AA1B965F4
