"""Pinhole camera, b200 backend.

The interface is the reference's PinholeCamera (blackhorizon/camera.py:25-120):
the same fields, defaults, errors and pixel convention (horizontal field of
view, pixel centres, row-major from the top-left), since those decide which
ray each pixel gets.  ``initial_states(spacetime)`` builds the past-directed
null initial states of every pixel on the device (``bh_camera_states``:
pinhole direction, null momentum and state in one kernel); ``ray_directions``
and ``ray_origins`` are host arrays, computed here component plane by
component plane with the reference's floating-point operations, so that they
equal its arrays bit for bit.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy
import torch

from . import _lib
from .backend import ptr, stream_handle

# Second choice of the horizontal axis when the view is parallel to the up
# hint (camera.py:59-61).
_FALLBACK_UP = numpy.array([0.0, 1.0, 0.0])


def _unit(v: numpy.ndarray) -> numpy.ndarray:
    length = numpy.linalg.norm(v)
    if length == 0.0:
        raise ValueError("zero-length vector cannot be normalized")
    return v / length


def look_at_frame(position, target, up_hint):
    """(forward, right, up) of a camera at `position` looking at `target`:
    forward is the unit view direction, right = forward x up_hint
    normalised (forward x +y when the view is parallel to the hint), and up
    completes the right-handed frame as right x forward."""
    eye = numpy.asarray(position, dtype=numpy.float64)
    view = _unit(numpy.asarray(target, dtype=numpy.float64) - eye)
    side = numpy.cross(view, numpy.asarray(up_hint, dtype=numpy.float64))
    if numpy.linalg.norm(side) < 1e-12:
        side = numpy.cross(view, _FALLBACK_UP)
    side = _unit(side)
    return view, side, numpy.cross(side, view)


def pixel_offsets(count: int, half_extent: float) -> numpy.ndarray:
    """Image-plane coordinate of each pixel centre along one axis, from -1 to
    +1 times half_extent (the left edge, or the bottom row when negated)."""
    centres = (numpy.arange(count) + 0.5) / count
    return (centres * 2.0 - 1.0) * half_extent


@dataclass(frozen=True)
class PinholeCamera:
    """A pinhole camera looking at a target point (camera.py:25-66)."""

    position: tuple[float, float, float]
    target: tuple[float, float, float] = (0.0, 0.0, 0.0)
    up_hint: tuple[float, float, float] = (0.0, 0.0, 1.0)
    fov_degrees: float = 20.0
    width: int = 320
    height: int = 240

    forward: numpy.ndarray = field(init=False, repr=False)
    right: numpy.ndarray = field(init=False, repr=False)
    up: numpy.ndarray = field(init=False, repr=False)

    def __post_init__(self) -> None:
        if self.width <= 0 or self.height <= 0:
            raise ValueError("image dimensions must be positive")
        if not 0.0 < self.fov_degrees < 180.0:
            raise ValueError("fov_degrees must be in (0, 180)")
        for name, axis in zip(("forward", "right", "up"),
                              look_at_frame(self.position, self.target, self.up_hint)):
            object.__setattr__(self, name, axis)

    @classmethod
    def from_orbit(cls, distance: float, inclination_degrees: float,
                   azimuth_degrees: float = 0.0, **kwargs) -> "PinholeCamera":
        """Camera at `distance` from the origin, `inclination_degrees` from the
        +z axis and `azimuth_degrees` from +x (camera.py:69-94)."""
        if distance <= 0.0:
            raise ValueError("distance must be positive")
        polar = math.radians(inclination_degrees)
        azimuth = math.radians(azimuth_degrees)
        rho = distance * math.sin(polar)  # distance from the z axis
        return cls(position=(rho * math.cos(azimuth), rho * math.sin(azimuth),
                             distance * math.cos(polar)), **kwargs)

    def half_extents(self) -> tuple[float, float]:
        """Half width and half height of the image plane at unit distance: the
        field of view is horizontal."""
        half_w = math.tan(math.radians(self.fov_degrees) / 2.0)
        return half_w, half_w * self.height / self.width

    def ray_directions(self) -> numpy.ndarray:
        """Unit directions per pixel, (height*width, 3), row-major from the
        top-left (camera.py:96-113), on the host."""
        half_w, half_h = self.half_extents()
        u = pixel_offsets(self.width, half_w)[None, :]    # grows to the right
        v = -pixel_offsets(self.height, half_h)[:, None]  # row 0 is the top
        planes = [f + u * r + v * w for f, r, w in zip(self.forward, self.right, self.up)]
        length = numpy.sqrt((planes[0] * planes[0] + planes[1] * planes[1])
                            + planes[2] * planes[2])
        return numpy.stack([p / length for p in planes], axis=-1).reshape(-1, 3)

    def ray_origins(self) -> numpy.ndarray:
        """Camera position per pixel, (height*width, 3) (camera.py:115-120)."""
        eye = numpy.asarray(self.position, dtype=numpy.float64)
        return numpy.tile(eye, (self.height * self.width, 1))

    def initial_states(self, spacetime, capture_margin: float = 1e-3,
                       escape_radius: float = 0.0):
        """(height*width, 8) past-directed null states on the device: the
        reference's ray_origins / ray_directions -> null_momentum_from_velocity
        ('past', normalised) -> build_state chain (render_shadow.py:69-75)."""
        from .tracer import CameraScene, camera_struct

        cam = camera_struct(CameraScene(spacetime, self, escape_radius or 1.0,
                                        capture_margin))
        n = self.width * self.height
        out = torch.empty((n, 8), dtype=torch.float64,
                          device=torch.device("cuda", torch.cuda.current_device()))
        _lib.check(_lib.load().bh_camera_states(cam, ptr(out), stream_handle()),
                   "initial_states")
        return out
