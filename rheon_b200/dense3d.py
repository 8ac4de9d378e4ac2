"""dense3D accepted-state frames (src/dense3d_sequence.rs), encoded on the device.

A frame is one JSON line byte-identical to the reference's
write_dense3d_frame (src/dense3d_sequence.rs:412-564): the header (frame,
time_s, dt_s, carrier and liquid stamps), the fields velocity_x/y/z and tracer
as `{:.9e}` f32 text, fraction and pressure as `{:.17e}` f64 text, then the
diagnostics object or null. Dense3dEncoder formats a device-resident state on
the device; Dense3dFrameWriter streams frames to a file with the limits and
terminal errors of Dense3dSequence's output side
(src/dense3d_sequence.rs:42-120, :224-341).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from typing import Optional

from . import _native as N
from ._native import lib

__all__ = ["Dense3dError", "Dense3dFrameInfo", "Dense3dFields", "Dense3dLimits", "Dense3dEncoder",
           "Dense3dFrameWriter", "text_f64", "text_f32"]


class Dense3dError(RuntimeError):
    """Dense3dError (src/dense3d_sequence.rs:21-27): kind is InvalidState,
    Limit, Aborted or Io (or the library status name for argument and device
    errors)."""

    def __init__(self, status: int, message: str = ""):
        self.status = status
        self.kind = N.STATUS_NAMES.get(status, f"Status{status}")
        super().__init__(message or f"dense3D export: {self.kind}")


@dataclass
class Dense3dLimits:
    """Dense3dLimits (src/dense3d_sequence.rs:13-19)."""
    max_cells: int
    max_frames: int
    max_bytes: int


@dataclass
class Dense3dFrameInfo:
    """The scalars of one frame: LiquidTransportView clocks and stamps, and
    for an accepted step the diagnostics of its LiquidStepReport. Without
    diagnostics it is the constructor frame (frame 0, time 0)."""
    frame: int = 0
    time_s: float = 0.0
    dt_s: float = 0.0
    carrier_stamp: tuple = (0, 0)  # (id, version)
    liquid_stamp: tuple = (0, 0)
    diagnostics: Optional[dict] = None  # keys of DIAGNOSTICS; pressure_iterations an int

    DIAGNOSTICS = ("pressure_residual_m3_s2", "carrier_divergence_s_inv", "liquid_divergence_s_inv",
                   "volume_before_m3", "volume_after_m3", "mass_after_kg", "inward_m3", "outward_m3", "source_m3",
                   "balance_m3", "rounding_budget_m3")

    def c(self) -> N.Dense3dFrame:
        f = N.Dense3dFrame()
        f.frame = int(self.frame)
        f.time_s = float(self.time_s)
        f.dt_s = float(self.dt_s)
        f.carrier_stamp_id, f.carrier_stamp_version = (int(x) for x in self.carrier_stamp)
        f.liquid_stamp_id, f.liquid_stamp_version = (int(x) for x in self.liquid_stamp)
        if self.diagnostics is not None:
            f.has_diagnostics = 1
            f.pressure_iterations = int(self.diagnostics.get("pressure_iterations", 0))
            for k in self.DIAGNOSTICS:
                setattr(f, k, float(self.diagnostics.get(k, 0.0)))
        return f


@dataclass
class Dense3dFields:
    """Device pointers of one state (0 for an absent tracer, fraction or
    pressure: printed as zeros). velocity_f64: the face arrays hold f64 and
    are printed as the f32 each value rounds to."""
    u: int
    v: int
    w: int
    tracer: int = 0
    fraction: int = 0
    pressure: int = 0
    velocity_f64: bool = False
    keep: list = field(default_factory=list, repr=False)  # owners of the memory

    @classmethod
    def from_tensors(cls, u, v, w, tracer=None, fraction=None, pressure=None):
        """From CUDA tensors (contiguous; faces f32 or f64, tracer f32,
        fraction and pressure f64)."""
        import torch

        ts = [u, v, w, tracer, fraction, pressure]
        for t in ts:
            if t is not None and (not t.is_cuda or not t.is_contiguous()):
                raise ValueError("dense3D fields must be contiguous CUDA tensors")
        if tracer is not None and tracer.dtype != torch.float32:
            raise ValueError("tracer must be float32")
        for t in (fraction, pressure):
            if t is not None and t.dtype != torch.float64:
                raise ValueError("fraction and pressure must be float64")
        f64 = u.dtype == torch.float64
        return cls(u.data_ptr(), v.data_ptr(), w.data_ptr(), tracer.data_ptr() if tracer is not None else 0,
                   fraction.data_ptr() if fraction is not None else 0,
                   pressure.data_ptr() if pressure is not None else 0, f64, [t for t in ts if t is not None])

    @classmethod
    def from_carrier(cls, carrier, fraction=None):
        """The carrier's accepted state (faces, tracer, the liquid fraction
        of an attached liquid state, the last accepted pressure); `fraction`
        (an f64 CUDA tensor) replaces the fraction."""
        f = N.Dense3dFields()
        st = lib().rb200_carrier_dense3d_fields(carrier._handle, C.byref(f))
        if st != N.OK:
            raise Dense3dError(st)
        out = cls(f.u or 0, f.v or 0, f.w or 0, f.tracer or 0, f.fraction or 0, f.pressure or 0,
                  f.velocity_storage == 1, [carrier])
        if fraction is not None:
            out.fraction = fraction.data_ptr()
            out.keep.append(fraction)
        return out

    def c(self) -> N.Dense3dFields:
        f = N.Dense3dFields()
        f.velocity_storage = 1 if self.velocity_f64 else 0
        f.u, f.v, f.w = self.u, self.v, self.w
        f.tracer = self.tracer or None
        f.fraction = self.fraction or None
        f.pressure = self.pressure or None
        return f


def text_f64(x: float) -> str:
    """`{:.17e}` text of a double, by the encoder's own routine (host)."""
    buf = C.create_string_buffer(32)
    n = lib().rb200_dense3d_text_f64(float(x), buf, 32)
    return buf.raw[:n].decode()


def text_f32(x: float) -> str:
    """`{:.9e}` text of a float (the value is rounded to f32 first)."""
    buf = C.create_string_buffer(32)
    n = lib().rb200_dense3d_text_f32(float(x), buf, 32)
    return buf.raw[:n].decode()


class Dense3dEncoder:
    """Encodes frames of one grid on a device into a device byte buffer."""

    def __init__(self, grid, device: int = 0):
        h = C.c_void_p()
        st = lib().rb200_dense3d_encoder_create(C.byref(grid.c()), device, C.byref(h))
        if st != N.OK:
            raise Dense3dError(st)
        self._h = h
        self.grid = grid
        self.device = device

    def close(self):
        if getattr(self, "_h", None):
            lib().rb200_dense3d_encoder_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def bound(self) -> int:
        """Upper bound on the bytes of one frame line of this grid."""
        return int(lib().rb200_dense3d_frame_bound(self._h))

    def encode_into(self, info: Dense3dFrameInfo, fields: Dense3dFields, out_ptr: int, capacity: int,
                    stream: int = 0) -> int:
        """Encode into device memory at out_ptr; returns the line's length."""
        n = C.c_uint64()
        st = lib().rb200_dense3d_encode(self._h, C.byref(info.c()), C.byref(fields.c()), out_ptr, capacity,
                                        C.byref(n), stream or None)
        if st != N.OK:
            raise Dense3dError(st, (lib().rb200_dense3d_encoder_error(self._h) or b"").decode())
        return int(n.value)

    def encode(self, info: Dense3dFrameInfo, fields: Dense3dFields) -> bytes:
        """The frame line as bytes (device encode, then a copy to the host)."""
        import torch

        buf = torch.empty(self.bound(), dtype=torch.uint8, device=f"cuda:{self.device}")
        n = self.encode_into(info, fields, buf.data_ptr(), buf.numel())
        return bytes(buf[:n].cpu().numpy().tobytes())


class Dense3dFrameWriter:
    """Bounded frame stream to a file (Dense3dSequence's output side).

    `output` is a path (a new file is created; an existing one is refused, as
    the reference's exporter refuses to overwrite) or an open file descriptor.
    Frames must come in order 0, 1, 2, ...; any failure is terminal.
    write_frame encodes on the device and returns; the copy to the host and
    the write run behind it (two frames in flight), so a write error surfaces
    at the next write_frame, flush or sync."""

    def __init__(self, grid, output, limits: Dense3dLimits, device: int = 0):
        self._own_fd = False
        if isinstance(output, (str, os.PathLike)):
            fd = os.open(output, os.O_WRONLY | os.O_CREAT | os.O_EXCL, 0o644)
            self._own_fd = True
        else:
            fd = int(output)
        self._fd = fd
        h = C.c_void_p()
        lim = N.Dense3dLimits(limits.max_cells, limits.max_frames, limits.max_bytes)
        st = lib().rb200_dense3d_writer_create(C.byref(grid.c()), C.byref(lim), fd, device, C.byref(h))
        if st != N.OK:
            if self._own_fd:
                os.close(fd)
            raise Dense3dError(st)
        self._h = h
        self.grid = grid

    def write_frame(self, info: Dense3dFrameInfo, fields: Dense3dFields, stream: int = 0) -> None:
        st = lib().rb200_dense3d_writer_frame(self._h, C.byref(info.c()), C.byref(fields.c()), stream or None)
        if st != N.OK:
            raise Dense3dError(st, (lib().rb200_dense3d_writer_error(self._h) or b"").decode())

    def flush(self) -> None:
        """Dense3dSequence::flush: returns once every accepted frame is
        written (the copies and writes run behind write_frame)."""
        st = lib().rb200_dense3d_writer_flush(self._h)
        if st != N.OK:
            raise Dense3dError(st, (lib().rb200_dense3d_writer_error(self._h) or b"").decode())

    def sync(self) -> None:
        """flush, then fsync of the file."""
        st = lib().rb200_dense3d_writer_sync(self._h)
        if st != N.OK:
            raise Dense3dError(st, (lib().rb200_dense3d_writer_error(self._h) or b"").decode())

    def frame_count(self) -> int:
        """Frames accepted (encoded and queued for writing)."""
        return int(lib().rb200_dense3d_writer_frames(self._h))

    def bytes_written(self) -> int:
        """Bytes written so far (all accepted frames after flush())."""
        return int(lib().rb200_dense3d_writer_bytes(self._h))

    def is_aborted(self) -> bool:
        return bool(lib().rb200_dense3d_writer_aborted(self._h))

    def close(self):
        if getattr(self, "_h", None):
            lib().rb200_dense3d_writer_destroy(self._h)
            self._h = None
        if getattr(self, "_own_fd", False):
            os.close(self._fd)
            self._own_fd = False

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
