"""Seeded synthetic inputs for the carrier-step workloads.

All inputs are generated on the host once, in float64, and cast to the face
storage type, so the oracle and the device see identical bits. The generator is
counter-based SplitMix64: u = splitmix64(seed ^ (stream << 48) ^ index), mapped
to [-1, 1) as 2*(u >> 11)*2^-53 - 1.

Workloads (cubic boxes, unit spacing, origin 0, density 1, walls everywhere):
  uniform_faces   interior faces i.i.d. U(-1, 1), wall-normal faces 0
  fourier_faces   8 random Fourier modes (integer wavevectors in [1, 8]^3,
                  random phase, random unit amplitude direction) + 0.05*U(-1,1)
  gaussian_blob   cell density, Gaussian of sigma 20 cells, peak 1
"""
from __future__ import annotations

import numpy as np

DEFAULT_SEED = 20261203
_M1 = np.uint64(0x9E3779B97F4A7C15)
_M2 = np.uint64(0xBF58476D1CE4E5B9)
_M3 = np.uint64(0x94D049BB133111EB)


def splitmix64(x: np.ndarray) -> np.ndarray:
    x = np.asarray(x, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = x + _M1
        z = (z ^ (z >> np.uint64(30))) * _M2
        z = (z ^ (z >> np.uint64(27))) * _M3
        return z ^ (z >> np.uint64(31))


def uniform(seed: int, stream: int, n: int, start: int = 0) -> np.ndarray:
    """n values in [-1, 1) of the given stream."""
    idx = np.arange(start, start + n, dtype=np.uint64)
    key = np.uint64((seed ^ (stream << 48)) & 0xFFFFFFFFFFFFFFFF)
    u = splitmix64(idx ^ key)
    return 2.0 * (u >> np.uint64(11)).astype(np.float64) * (2.0 ** -53) - 1.0


def face_counts(n, axis):
    f = list(n)
    f[axis] += 1
    return f


def wall_mask(n, axis) -> np.ndarray:
    """Boolean mask (x-fastest flat) of the wall-normal faces of `axis`."""
    f = face_counts(n, axis)
    c = np.arange(f[axis])
    wall = (c == 0) | (c == n[axis])
    shape = [1, 1, 1]
    shape[2 - axis] = f[axis]  # arrays are [k][j][i]
    m = np.broadcast_to(wall.reshape(shape), (f[2], f[1], f[0]))
    return np.ascontiguousarray(m).reshape(-1)


def uniform_faces(n, seed=DEFAULT_SEED, dtype=np.float64):
    faces = []
    for a in range(3):
        f = face_counts(n, a)
        vals = uniform(seed, a, f[0] * f[1] * f[2])
        vals[wall_mask(n, a)] = 0.0
        faces.append(vals.astype(dtype))
    return faces


def fourier_modes(seed=DEFAULT_SEED, modes=8, kmax=8):
    """(k[m,3], phase[m], amplitude[m,3]) of the random Fourier field."""
    r = uniform(seed, 8, modes * 7)
    k = np.minimum(kmax, 1 + np.floor((r[: 3 * modes].reshape(modes, 3) + 1.0) * 0.5 * kmax)).astype(np.float64)
    phase = np.pi * r[3 * modes: 4 * modes]
    a = r[4 * modes: 7 * modes].reshape(modes, 3)
    norm = np.sqrt(np.sum(a * a, axis=1, keepdims=True))
    norm[norm == 0.0] = 1.0
    return k, phase, a / norm


def fourier_faces(n, seed=DEFAULT_SEED, modes=8, kmax=8, amplitude=1.0, noise=0.05, dtype=np.float64):
    k, phase, amp = fourier_modes(seed, modes, kmax)
    L = np.array(n, dtype=np.float64)
    faces = []
    for a in range(3):
        f = face_counts(n, a)
        xs = [np.arange(f[d], dtype=np.float64) + (0.0 if d == a else 0.5) for d in range(3)]
        Z, Y, X = np.meshgrid(xs[2], xs[1], xs[0], indexing="ij")
        val = np.zeros((f[2], f[1], f[0]), np.float64)
        for m in range(len(phase)):
            arg = 2.0 * np.pi * (k[m, 0] * X / L[0] + k[m, 1] * Y / L[1] + k[m, 2] * Z / L[2]) + phase[m]
            val += amplitude * amp[m, a] * np.sin(arg)
        flat = val.reshape(-1)
        flat += noise * uniform(seed, 16 + a, flat.size)
        flat[wall_mask(n, a)] = 0.0
        faces.append(flat.astype(dtype))
    return faces


def gaussian_blob(n, sigma=20.0, peak=1.0, center=None):
    if center is None:
        center = (n[0] / 2.0, n[1] / 4.0, n[2] / 2.0)
    xs = [np.arange(n[d], dtype=np.float64) + 0.5 for d in range(3)]
    Z, Y, X = np.meshgrid(xs[2], xs[1], xs[0], indexing="ij")
    r2 = (X - center[0]) ** 2 + (Y - center[1]) ** 2 + (Z - center[2]) ** 2
    return (peak * np.exp(-r2 / (2.0 * sigma * sigma))).reshape(-1).astype(np.float32)
