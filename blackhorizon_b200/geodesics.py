"""Geodesic dynamics in Kerr-Schild coordinates, b200 backend.

Same functions and state layout as blackhorizon/geodesics.py: a batch is an
(n, 8) array of (t, x, y, z, p_t, p_x, p_y, p_z) with covariant momenta.
``geodesic_rhs``, ``hamiltonian``, ``coordinate_velocity`` and
``null_momentum_from_velocity`` run as CUDA kernels.

``GeodesicRhs(spacetime)`` is the callable form of ``geodesic_rhs`` that the
b200 integrators recognise (the reference passes a closure; an arbitrary
Python callable cannot be moved onto the device, so the b200
``dormand_prince_step`` / ``rk4_step`` accept this object, or
``functools.partial(geodesic_rhs, spacetime)``).
"""

from __future__ import annotations

import functools

import numpy
import torch

from . import _lib
from .backend import (Array, is_device_array, out_like, ptr, stream_handle,
                      to_device_f64)
from .kerr import KerrSpacetime


def _check_state(s):
    if s.dim() != 2 or s.shape[1] != 8:
        raise ValueError("state must have shape (n, 8)")


def build_state(positions: Array, momenta: Array, t0: float = 0.0) -> Array:
    """(n, 8) state from positions (n, 3) and momenta (n, 4)
    (geodesics.py:25-39), in the positions' array type."""
    if is_device_array(positions):
        n = positions.shape[0]
        state = torch.empty((n, 8), dtype=positions.dtype, device=positions.device)
        state[:, 0] = t0
        state[:, 1:4] = positions
        state[:, 4:8] = torch.as_tensor(momenta, device=positions.device)
        return state
    positions = numpy.asarray(positions)
    n = positions.shape[0]
    state = numpy.empty((n, 8), dtype=positions.dtype)
    state[:, 0] = t0
    state[:, 1:4] = positions
    state[:, 4:8] = momenta
    return state


class GeodesicRhs:
    """d(state)/d(lambda) for one spacetime; the RHS object of the b200
    integrators."""

    def __init__(self, spacetime: KerrSpacetime) -> None:
        self.spacetime = spacetime

    def __call__(self, state: Array) -> Array:
        return geodesic_rhs(self.spacetime, state)


def spacetime_of_rhs(rhs) -> KerrSpacetime:
    """The spacetime behind a recognised RHS callable, else TypeError."""
    if isinstance(rhs, GeodesicRhs):
        return rhs.spacetime
    if isinstance(rhs, functools.partial) and rhs.func is geodesic_rhs and rhs.args:
        return rhs.args[0]
    raise TypeError(
        "the b200 integrators run the geodesic RHS on the device: pass "
        "GeodesicRhs(spacetime) or functools.partial(geodesic_rhs, spacetime)"
    )


def geodesic_rhs(spacetime: KerrSpacetime, state: Array) -> Array:
    """Hamilton's equations for a batch (geodesics.py:42-74)."""
    s, host = to_device_f64(state, "state")
    _check_state(s)
    out = torch.empty_like(s)
    _lib.check(_lib.load().bh_geodesic_rhs(spacetime.mass, spacetime.spin, ptr(s),
                                           ptr(out), s.shape[0], stream_handle()),
               "geodesic_rhs")
    return out_like(out, host, state)


def hamiltonian(spacetime: KerrSpacetime, state: Array) -> Array:
    """Super-Hamiltonian per geodesic (geodesics.py:77-85)."""
    s, host = to_device_f64(state, "state")
    _check_state(s)
    out = torch.empty(s.shape[0], dtype=torch.float64, device=s.device)
    _lib.check(_lib.load().bh_hamiltonian(spacetime.mass, spacetime.spin, ptr(s),
                                          ptr(out), s.shape[0], stream_handle()),
               "hamiltonian")
    return out_like(out, host, state)


def conserved_quantities(state: Array):
    """E = -p_t and L_z = x p_y - y p_x (geodesics.py:88-92)."""
    energy = -state[:, 4]
    l_z = state[:, 1] * state[:, 6] - state[:, 2] * state[:, 5]
    return energy, l_z


def coordinate_velocity(spacetime: KerrSpacetime, state: Array) -> Array:
    """dx^mu/dlambda = g^mu^nu p_nu, shape (n, 4) (geodesics.py:95-106)."""
    s, host = to_device_f64(state, "state")
    _check_state(s)
    out = torch.empty((s.shape[0], 4), dtype=torch.float64, device=s.device)
    _lib.check(_lib.load().bh_coordinate_velocity(
        spacetime.mass, spacetime.spin, ptr(s), ptr(out), s.shape[0],
        stream_handle()), "coordinate_velocity")
    return out_like(out, host, state)


def null_momentum_from_velocity(
    spacetime: KerrSpacetime,
    positions: Array,
    directions: Array,
    time_orientation: str = "past",
    normalize: bool = True,
) -> Array:
    """Covariant null momentum for a spatial direction (geodesics.py:109-170).

    ``spacetime.spin`` may be an (n,) array (one spin per ray)."""
    if time_orientation not in ("past", "future"):
        raise ValueError("time_orientation must be 'past' or 'future'")
    pos, host = to_device_f64(positions, "positions")
    d, _ = to_device_f64(directions, "directions")
    if pos.dim() != 2 or pos.shape[1] != 3 or d.shape != pos.shape:
        raise ValueError("positions and directions must have shape (n, 3)")
    n = pos.shape[0]
    spins = None
    spin = spacetime.spin
    if numpy.ndim(spin) != 0 or is_device_array(spin):
        spins, _ = to_device_f64(spin, "spin")
        if spins.shape != (n,):
            raise ValueError("per-ray spin must have shape (n,)")
        spin = 0.0
    out = torch.empty((n, 4), dtype=torch.float64, device=pos.device)
    _lib.check(_lib.load().bh_null_momentum(
        float(spacetime.mass), float(spin), ptr(spins), ptr(pos), ptr(d), n,
        int(time_orientation == "past"), int(bool(normalize)), ptr(out),
        stream_handle()), "null_momentum_from_velocity")
    return out_like(out, host, positions)


def timelike_momentum(spacetime: KerrSpacetime, positions: Array,
                      coordinate_velocities: Array) -> Array:
    """Unit-mass covariant momentum from dx^i/dt (geodesics.py:173-209).

    Not on the ray-tracing path; assembled on the device from the
    ``bh_geometry`` kernel's H and l."""
    pos, host = to_device_f64(positions, "positions")
    v, _ = to_device_f64(coordinate_velocities, "coordinate_velocities")
    geo = spacetime.geometry(pos[:, 0].contiguous(), pos[:, 1].contiguous(),
                             pos[:, 2].contiguous())
    h, l = geo.h, geo.l
    l_dot_big_v = 1.0 + (l * v).sum(-1)
    norm2 = -1.0 + (v * v).sum(-1) + 2.0 * h * l_dot_big_v * l_dot_big_v
    if bool((norm2 >= 0.0).any()):
        raise ValueError("coordinate velocity is not timelike at one or more positions")
    u_t = 1.0 / torch.sqrt(-norm2)
    l_dot_u = u_t * l_dot_big_v
    mom = torch.empty((pos.shape[0], 4), dtype=torch.float64, device=pos.device)
    mom[:, 0] = -u_t + 2.0 * h * l_dot_u
    mom[:, 1:4] = u_t[:, None] * v + (2.0 * h * l_dot_u)[:, None] * l
    return out_like(mom, host, positions)
