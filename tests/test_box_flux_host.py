"""Host-side contracts of the box-flux workspace (no device needed).

BoxFluxWorkspace::new (src/box_flux.rs:132-186) checks the operator, the cell
mass, the side areas and the buffer limit before it touches a device; the
C structs match include/rheon_b200.h.
"""
import ctypes as C

import pytest

import rheon_b200 as R
from rheon_b200 import _native as N
from rheon_b200.box_flux import BoxFluxError, BoxFluxStamp, BoxFluxWorkspace, PrescribedBoxFlux


def test_struct_layouts():
    assert C.sizeof(N.BoxFluxBoundary) == 40
    assert C.sizeof(N.BoxFluxReport) == 192


def test_invalid_boundary():
    """box_flux_contract.rs:484-487"""
    with pytest.raises(BoxFluxError) as e:
        PrescribedBoxFlux(BoxFluxStamp(0, 0), [[float("nan")] * 2] * 3)
    assert e.value.kind == "InvalidBoundary"
    b = PrescribedBoxFlux(BoxFluxStamp(37, 8), [[-0.375, 0.0], [0.0, 0.5], [0.0, 0.0]])
    assert b.stamp() == BoxFluxStamp(37, 8) and b.outward_speeds()[1] == (0.0, 0.5)
    c = b.c()
    assert (c.id, c.version) == (37, 8) and list(c.outward) == [-0.375, 0.0, 0.0, 0.5, 0.0, 0.0]


def test_invalid_density_and_mass():
    """box_flux_contract.rs:488-503"""
    g = R.GridGeometry([2, 1, 1])
    with pytest.raises(BoxFluxError) as e:
        BoxFluxWorkspace(g, 0.0, 4096)
    assert (e.value.kind, e.value.inner) == ("Operator", "InvalidDensity")
    for spacing, density in [([1e-100, 1e-100, 1.0], 1e-200), ([1e100, 1e100, 1.0], 1e200)]:
        with pytest.raises(BoxFluxError) as e:
            BoxFluxWorkspace(R.GridGeometry([2, 1, 1], spacing), density, 4096)
        assert e.value.kind == "InvalidMass"


@pytest.mark.parametrize("method", [0, 1])
def test_buffer_limit_is_56_bytes_per_cell(method):
    """box_flux_contract.rs:452-460"""
    g = R.GridGeometry([1, 1, 1], [0.5, 1.0, 2.0])
    with pytest.raises(BoxFluxError) as e:
        BoxFluxWorkspace(g, 1.0, 55, method)
    assert e.value.kind == "BufferLimit" and (e.value.required, e.value.limit) == (56, 55)
    if R.device_count() == 0:
        with pytest.raises(BoxFluxError) as e:
            BoxFluxWorkspace(g, 1.0, 56, method)
        assert e.value.status == N.NO_DEVICE
