"""The doomed-observer plunge of the offline renderer on the b200 backend.

Mirrors blackhorizon/offline/infall.py:38-192: ``radial_momentum`` (the
E-parameterised radial infaller), ``build_plunge`` (the camera's timelike
worldline) and ``plunge_tetrad`` (the camera frame at a worldline sample).
The worldline is one sequential trajectory and is integrated by the library
on the host (``bh_plunge_worldline``); each frame of the plunge is then
``emission.render_hdr`` with the tetrad and the interior stop, every ray on
the device (``plunge_frame``).
"""

from __future__ import annotations

import ctypes

import numpy

from . import _lib
from .kerr import KerrSpacetime


def radial_momentum(spacetime: KerrSpacetime, position, energy: float) -> numpy.ndarray:
    """Covariant momentum (1, 4) of a radial infaller with conserved energy
    E >= 0 (infall.py:38-91); ValueError where no future-directed inward
    root exists (for E = 0 outside the horizon)."""
    pos = numpy.ascontiguousarray(position, dtype=float)
    out = numpy.empty(4)
    _lib.check(_lib.load().bh_radial_momentum(
        float(spacetime.mass), float(spacetime.spin), pos.ctypes.data_as(ctypes.c_void_p),
        float(energy), out.ctypes.data_as(ctypes.c_void_p)), "radial_momentum")
    return out[None, :]


def build_plunge(spacetime: KerrSpacetime, start_radius: float, energy: float,
                 stop_radius: float, step: float = 5e-4):
    """(taus (k,), states (k, 8)): the plunge worldline from (start_radius,
    0, 0), every integration step (infall.py:94-153)."""
    lib = _lib.load()
    args = (float(spacetime.mass), float(spacetime.spin), float(start_radius), float(energy),
            float(stop_radius), float(step))
    count = lib.bh_plunge_worldline(*args, 0, None, None)
    if count < 0:
        raise ValueError(lib.bh_last_error().decode())
    taus = numpy.empty(count)
    states = numpy.empty((count, 8))
    got = lib.bh_plunge_worldline(*args, count, taus.ctypes.data_as(ctypes.c_void_p),
                                  states.ctypes.data_as(ctypes.c_void_p))
    if got != count:
        raise RuntimeError("plunge worldline changed between calls")
    return taus, states


def plunge_tetrad(spacetime: KerrSpacetime, state, look: str):
    """(position, tetrad) of the camera at a worldline sample
    (infall.py:156-189): the sample's 4-velocity, forward along the outward
    radial direction, its opposite, or sideways, up toward +z (+y near the
    axis)."""
    from .frames import build_tetrad, raise_index

    state = numpy.asarray(state, dtype=float)
    position = state[1:4]
    velocity = raise_index(spacetime, position[None, :], state[None, 4:8])[0]
    outward = position / max(numpy.linalg.norm(position), 1e-12)
    up_seed = numpy.array([0.0, 0.0, 1.0])
    if abs(float(numpy.dot(outward, up_seed))) > 0.98:
        up_seed = numpy.array([0.0, 1.0, 0.0])
    if look == "outward":
        forward = outward
    elif look == "inward":
        forward = -outward
    else:
        forward = numpy.cross(up_seed, outward)
        forward = forward / max(numpy.linalg.norm(forward), 1e-12)
    return position, build_tetrad(spacetime, position, velocity, forward, up_seed)


def terminal_stop(spacetime: KerrSpacetime, stop: float = 0.02,
                  journey: str = "realistic") -> float:
    """The stop radius of the plunge (infall.py:202-217): on the realistic
    journey through a spinning hole the terminal surface is the Cauchy
    horizon, so the stop is raised to at least 1.02 r_minus; the idealized
    journey keeps the requested stop."""
    inner = float(spacetime.inner_horizon_radius)
    if journey != "idealized" and inner > 0.0 and stop < inner * 1.02:
        return inner * 1.02
    return float(stop)


def plunge_frame(spacetime: KerrSpacetime, state, width: int, height: int, settings,
                 look: str = "inward", stop: float = 0.02, journey: str = "realistic",
                 **kwargs):
    """One frame of the plunge (infall.py:246-262): render_hdr from the
    camera at a worldline sample with its tetrad and the interior stop
    (``terminal_stop``); a float32 (height, width, 3) device tensor."""
    from .emission import render_hdr
    from .offline import FlyCamera

    position, tetrad = plunge_tetrad(spacetime, state, look)
    stop = terminal_stop(spacetime, stop, journey)
    camera = FlyCamera(position=numpy.asarray(position, dtype=float).copy(), yaw=0.0, pitch=0.0)
    return render_hdr(camera, width, height, settings, camera_tetrad=tetrad,
                      interior_stop=stop, **kwargs)
