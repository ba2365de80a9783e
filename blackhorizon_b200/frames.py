"""Observer frames for interior cameras (camera set-up on the host).

Mirrors blackhorizon/frames.py:33-218: metric inner products and index
raising/lowering with g = eta + 2 H l l (Kerr-Schild), the rain (Doran)
free-fall 4-velocity, an orthonormal tetrad by metric Gram-Schmidt, and the
past-directed traced momenta of tetrad camera rays (unit camera-frame
frequency).  These prepare a handful of vectors per camera; H and l come
from the device (``KerrSpacetime.geometry``), the rest is NumPy on (n, 4)
host arrays.
"""

from __future__ import annotations

import numpy

from .kerr import KerrSpacetime


def _hl(spacetime: KerrSpacetime, positions):
    p = numpy.asarray(positions, dtype=float)
    geo = spacetime.geometry(numpy.ascontiguousarray(p[:, 0]), numpy.ascontiguousarray(p[:, 1]),
                             numpy.ascontiguousarray(p[:, 2]))
    return numpy.asarray(geo.h), numpy.asarray(geo.l)


def metric_dot(spacetime: KerrSpacetime, positions, a_vec, b_vec):
    """g(A, B) of contravariant 4-vectors (frames.py:33-60)."""
    h, l = _hl(spacetime, positions)
    a = numpy.asarray(a_vec, dtype=float)
    b = numpy.asarray(b_vec, dtype=float)
    eta = -a[:, 0] * b[:, 0] + numpy.sum(a[:, 1:4] * b[:, 1:4], axis=-1)
    l_a = a[:, 0] + numpy.sum(l * a[:, 1:4], axis=-1)
    l_b = b[:, 0] + numpy.sum(l * b[:, 1:4], axis=-1)
    return eta + 2.0 * h * l_a * l_b


def lower_index(spacetime: KerrSpacetime, positions, vectors):
    """v_mu = g_mu_nu v^nu (frames.py:63-77)."""
    h, l = _hl(spacetime, positions)
    v = numpy.asarray(vectors, dtype=float)
    l_v = v[:, 0] + numpy.sum(l * v[:, 1:4], axis=-1)
    out = numpy.empty_like(v)
    out[:, 0] = -v[:, 0] + 2.0 * h * l_v
    out[:, 1:4] = v[:, 1:4] + (2.0 * h * l_v)[:, None] * l
    return out


def raise_index(spacetime: KerrSpacetime, positions, covectors):
    """v^mu = g^mu_nu v_nu with g^-1 = eta - 2 H l^ l^ (frames.py:80-99)."""
    h, l = _hl(spacetime, positions)
    c = numpy.asarray(covectors, dtype=float)
    l_up = -c[:, 0] + numpy.sum(l * c[:, 1:4], axis=-1)
    out = numpy.empty_like(c)
    out[:, 0] = -c[:, 0] + 2.0 * h * l_up
    out[:, 1:4] = c[:, 1:4] - (2.0 * h * l_up)[:, None] * l
    return out


def rain_four_velocity(spacetime: KerrSpacetime, positions):
    """Contravariant 4-velocity of the rain observer, E = 1 free fall with
    covariant momentum (-1, w l), w = -sqrt(2H) / (1 + sqrt(2H))
    (frames.py:102-127)."""
    p = numpy.asarray(positions, dtype=float)
    h, l = _hl(spacetime, p)
    root = numpy.sqrt(numpy.maximum(2.0 * h, 0.0))
    w = -root / (1.0 + root)
    cov = numpy.empty(p.shape[:-1] + (4,))
    cov[:, 0] = -1.0
    cov[:, 1:4] = w[:, None] * l
    return raise_index(spacetime, p, cov)


def build_tetrad(spacetime: KerrSpacetime, position, four_velocity, forward, up):
    """Orthonormal tetrad (e0 = u, e1 view, e2 right, e3 up) by metric
    Gram-Schmidt from the seeds (forward, forward x up, up)
    (frames.py:130-180).  Raises ValueError for a non-timelike u or
    degenerate seeds."""
    pos = numpy.asarray(position, dtype=float)[None, :]

    def dot(a, b):
        return float(metric_dot(spacetime, pos, a[None, :], b[None, :])[0])

    e0 = numpy.asarray(four_velocity, dtype=float)
    norm0 = dot(e0, e0)
    if norm0 >= 0.0:
        raise ValueError("observer 4-velocity must be timelike")
    e0 = e0 / numpy.sqrt(-norm0)
    fwd = numpy.asarray(forward, dtype=float)
    upv = numpy.asarray(up, dtype=float)
    seeds = [numpy.concatenate([[0.0], fwd]),
             numpy.concatenate([[0.0], numpy.cross(fwd, upv).astype(float)]),
             numpy.concatenate([[0.0], upv])]
    basis = [e0]
    for seed in seeds:
        vec = seed + dot(seed, e0) * e0
        for spatial in basis[1:]:
            vec = vec - dot(seed, spatial) * spatial
        nrm = dot(vec, vec)
        if nrm <= 1e-14:
            raise ValueError("degenerate tetrad seed directions")
        basis.append(vec / numpy.sqrt(nrm))
    return numpy.stack(basis)


def tetrad_ray_momenta(spacetime: KerrSpacetime, position, tetrad, local_directions):
    """Past-directed traced covariant momenta (n, 4) of tetrad camera rays
    looking along local directions (components on e1, e2, e3): minus the
    lowered physical momentum e0 - n.e, so every ray has unit camera-frame
    frequency (frames.py:182-218)."""
    d = numpy.asarray(local_directions, dtype=float)
    t = numpy.asarray(tetrad, dtype=float)
    n = d.shape[0]
    spatial = d[:, 0:1] * t[1][None, :] + d[:, 1:2] * t[2][None, :] + d[:, 2:3] * t[3][None, :]
    physical = t[0][None, :] - spatial
    positions = numpy.tile(numpy.asarray(position, dtype=float)[None, :], (n, 1))
    return lower_index(spacetime, positions, -physical)
