"""Shared cases and numpy restatements for the box-flux tests.

The helpers restate the independent checks of tests/box_flux_contract.rs
(imposed, independent_divergence, dense_pressure, mixed) and the per-face
arithmetic of BoxFluxWorkspace::project (src/box_flux.rs:297-362) in float64
numpy, one IEEE operation at a time in the reference's order, so that a
device result can be recomputed bit for bit from the device's own pressure.
"""
import numpy as np


def face_counts(counts, axis):
    fc = list(counts)
    fc[axis] += 1
    return fc


def component(outward, d, upper):
    speed = np.float32(outward[d][1 if upper else 0])
    if speed == 0:
        return np.float32(0.0)
    return speed if upper else -speed


def _side(axis, index):
    sl = [slice(None)] * 3
    sl[2 - axis] = index
    return tuple(sl)


def imposed(counts, old, outward):
    """tests/box_flux_contract.rs:40-56: the outer samples replaced by the sides' components."""
    v = [np.array(o, dtype=np.float32, copy=True) for o in old]
    for d in range(3):
        fc = face_counts(counts, d)
        arr = v[d].reshape(fc[2], fc[1], fc[0])
        arr[_side(d, 0)] = component(outward, d, False)
        arr[_side(d, counts[d])] = component(outward, d, True)
    return v


def divergence(counts, spacing, faces):
    """divergence() (src/box_flux.rs:405-434): value = 0; value += (hi - lo)/h_d, per cell."""
    n = counts
    value = np.zeros((n[2], n[1], n[0]))
    for d in range(3):
        fc = face_counts(n, d)
        f = np.asarray(faces[d], np.float32).reshape(fc[2], fc[1], fc[0]).astype(np.float64)
        hi = f[_side(d, slice(1, None))]
        lo = f[_side(d, slice(None, -1))]
        value = value + (hi - lo) / spacing[d]
    return value.reshape(-1)


def dense_pressure(counts, spacing, old, outward, rho, dt):
    """The gauge-eliminated dense solve of tests/box_flux_contract.rs:140-207."""
    n = int(np.prod(counts))
    h = spacing
    area = [h[1] * h[2], h[0] * h[2], h[0] * h[1]]
    m = np.zeros((n, n))
    for k in range(counts[2]):
        for j in range(counts[1]):
            for i in range(counts[0]):
                p = [i, j, k]
                row = i + counts[0] * (j + counts[1] * k)
                for d in range(3):
                    if p[d] + 1 < counts[d]:
                        q = list(p)
                        q[d] += 1
                        col = q[0] + counts[0] * (q[1] + counts[1] * q[2])
                        wgt = area[d] / (rho * h[d])
                        m[row, row] += wgt
                        m[col, col] += wgt
                        m[row, col] -= wgt
                        m[col, row] -= wgt
    vol = h[0] * h[1] * h[2]
    rhs = -vol * divergence(counts, spacing, imposed(counts, old, outward)) / dt
    p = np.zeros(n)
    p[1:] = np.linalg.solve(m[1:, 1:], rhs[1:])
    return p


def mixed_old(counts):
    """tests/box_flux_contract.rs:209-219: old[d][i] = ((3 i + d) mod 7) 0.13 - 0.2."""
    out = []
    for d in range(3):
        fc = face_counts(counts, d)
        m = fc[0] * fc[1] * fc[2]
        out.append(np.array([((i * 3 + d) % 7) * 0.13 - 0.2 for i in range(m)], np.float32))
    return out


MIXED = dict(counts=(3, 2, 1), spacing=(0.5, 1.0, 2.0), origin=(-1.0, 2.0, 0.0),
             outward=[[-0.375, 0.0], [0.0, 0.5], [0.0, 0.0]], density=1.5, dt=0.2)


def correct_from_pressure(counts, spacing, density, old, p, dt, outward):
    """The stored output of the correction (src/box_flux.rs:297-328) for a given pressure:
    f32(f64(u) - (dt (1/(rho h_d))) (p_c - p_left)) on interior faces, side components outside."""
    n = counts
    P = np.asarray(p, np.float64).reshape(n[2], n[1], n[0])
    out = []
    for d in range(3):
        fc = face_counts(n, d)
        o = np.asarray(old[d], np.float32).reshape(fc[2], fc[1], fc[0]).astype(np.float64)
        res = np.empty((fc[2], fc[1], fc[0]), np.float32)
        dtf = dt * (1.0 / (density * spacing[d]))
        diff = P[_side(d, slice(1, None))] - P[_side(d, slice(None, -1))]
        res[_side(d, slice(1, n[d]))] = (o[_side(d, slice(1, n[d]))] - dtf * diff).astype(np.float32)
        res[_side(d, 0)] = component(outward, d, False)
        res[_side(d, n[d])] = component(outward, d, True)
        out.append(res.reshape(-1))
    return out


def work_terms(counts, spacing, density, old, out, p, dt, outward):
    """Per-face and per-cell terms of BoxFluxWork (src/box_flux.rs:318-362), each
    rounded as the reference rounds it, as flat arrays in the reference's order."""
    n = counts
    h = spacing
    area = [h[1] * h[2], h[0] * h[2], h[0] * h[1]]
    vol = h[0] * h[1] * h[2]
    mass = density * vol
    half = 0.5 * mass
    P = np.asarray(p, np.float64).reshape(n[2], n[1], n[0])
    kb, ka, ce, cr = [], [], [], []
    for d in range(3):
        fc = face_counts(n, d)
        inner = _side(d, slice(1, n[d]))
        u = np.asarray(old[d], np.float32).reshape(fc[2], fc[1], fc[0])[inner].astype(np.float64)
        v = np.asarray(out[d], np.float32).reshape(fc[2], fc[1], fc[0])[inner].astype(np.float64)
        diff = P[_side(d, slice(1, None))] - P[_side(d, slice(None, -1))]
        delta = v - u
        kb.append((half * u * u).reshape(-1))
        ka.append((half * v * v).reshape(-1))
        ce.append((half * delta * delta).reshape(-1))
        cr.append(((mass * delta + (dt * area[d]) * diff) * v).reshape(-1))
    div = divergence(n, h, out)
    q = np.zeros((n[2], n[1], n[0]))
    for d in range(3):
        lo = np.zeros(n[d], bool)
        lo[0] = True
        hi = np.zeros(n[d], bool)
        hi[-1] = True
        shape = [1, 1, 1]
        shape[2 - d] = n[d]
        q = q + np.where(lo.reshape(shape), area[d] * float(np.float32(outward[d][0])), 0.0)
        q = q + np.where(hi.reshape(shape), area[d] * float(np.float32(outward[d][1])), 0.0)
    q = q.reshape(-1)
    dtp = dt * np.asarray(p, np.float64)
    return dict(kinetic_before=np.concatenate(kb), kinetic_after=np.concatenate(ka),
                correction_energy=np.concatenate(ce), correction_residual_work=np.concatenate(cr),
                boundary_pressure_work=-(dtp * q), divergence_residual_work=dtp * vol * div), div


def balanced_outward(counts, spacing, scale=2.0 ** -8):
    """A boundary with zero net flux. On dyadic spacings: inflow through the
    lower x side, outflow through the upper y side with side_x a + side_y b = 0
    exactly (a = -side_y t, b = side_x t), and a uniform -z through-flow;
    otherwise through-flows along x and y (equal and opposite terms)."""
    h = spacing
    side_x = h[1] * h[2] * counts[1] * counts[2]
    side_y = h[0] * h[2] * counts[0] * counts[2]
    a, b = -side_y * scale, side_x * scale
    if float(np.float32(a)) == a and float(np.float32(b)) == b:
        return [[a, 0.0], [0.0, b], [0.125, -0.125]]
    return [[-0.25, 0.25], [0.375, -0.375], [0.0, 0.0]]
