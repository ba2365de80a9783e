"""Pinhole camera, b200 backend.

The camera basis and the host-side ``ray_directions`` / ``ray_origins`` are
the reference's (blackhorizon/camera.py:25-120, NumPy, unchanged behaviour
and errors).  ``initial_states(spacetime)`` generates the past-directed
null initial states of every pixel on the device (``bh_camera_states``):
pinhole direction, null_momentum_from_velocity and build_state in one kernel.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy
import torch

from . import _lib
from .backend import ptr, stream_handle


def _normalize(v: numpy.ndarray) -> numpy.ndarray:
    norm = numpy.linalg.norm(v)
    if norm == 0.0:
        raise ValueError("zero-length vector cannot be normalized")
    return v / norm


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
        forward = _normalize(
            numpy.asarray(self.target, dtype=numpy.float64)
            - numpy.asarray(self.position, dtype=numpy.float64)
        )
        up_hint = numpy.asarray(self.up_hint, dtype=numpy.float64)
        right = numpy.cross(forward, up_hint)
        if numpy.linalg.norm(right) < 1e-12:
            # Looking along the up hint: the reference's fallback axis.
            right = numpy.cross(forward, numpy.array([0.0, 1.0, 0.0]))
        right = _normalize(right)
        up = numpy.cross(right, forward)
        object.__setattr__(self, "forward", forward)
        object.__setattr__(self, "right", right)
        object.__setattr__(self, "up", up)

    @classmethod
    def from_orbit(cls, distance: float, inclination_degrees: float,
                   azimuth_degrees: float = 0.0, **kwargs) -> "PinholeCamera":
        """Camera on a sphere around the origin (camera.py:69-94)."""
        if distance <= 0.0:
            raise ValueError("distance must be positive")
        inc = math.radians(inclination_degrees)
        azi = math.radians(azimuth_degrees)
        position = (
            distance * math.sin(inc) * math.cos(azi),
            distance * math.sin(inc) * math.sin(azi),
            distance * math.cos(inc),
        )
        return cls(position=position, **kwargs)

    def ray_directions(self) -> numpy.ndarray:
        """Unit directions per pixel, (height*width, 3), row-major from the
        top-left (camera.py:96-113); host NumPy as in the reference."""
        half_w = math.tan(math.radians(self.fov_degrees) / 2.0)
        half_h = half_w * self.height / self.width
        cols = (numpy.arange(self.width) + 0.5) / self.width * 2.0 - 1.0
        rows = 1.0 - (numpy.arange(self.height) + 0.5) / self.height * 2.0
        u, v = numpy.meshgrid(cols * half_w, rows * half_h)
        directions = (
            self.forward[None, None, :]
            + u[..., None] * self.right[None, None, :]
            + v[..., None] * self.up[None, None, :]
        )
        directions /= numpy.linalg.norm(directions, axis=-1, keepdims=True)
        return directions.reshape(-1, 3)

    def ray_origins(self) -> numpy.ndarray:
        """Camera position per pixel, (height*width, 3) (camera.py:115-120)."""
        origin = numpy.asarray(self.position, dtype=numpy.float64)
        return numpy.broadcast_to(origin, (self.height * self.width, 3)).copy()

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
