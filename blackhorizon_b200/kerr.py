"""Kerr spacetime in Cartesian Kerr-Schild coordinates, b200 backend.

Same API as blackhorizon/kerr.py: ``KerrSpacetime(mass, spin)`` with the
analytic radii (kerr.py:73-112, host scalars), ``geometry(x, y, z,
gradients)`` (kerr.py:118-193) and ``kerr_schild_radius`` evaluated by the
``bh_geometry`` kernel, and ``metric`` / ``inverse_metric`` (kerr.py:201-235)
assembled on the device from the kernel's H and l.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import torch

from . import _lib
from .backend import Array, out_like, ptr, stream_handle, to_device_f64


@dataclass(frozen=True)
class KerrSchildGeometry:
    """Pointwise geometry (kerr.py:32-49); grad_l[..., i, j] = d l_j / d x_i."""

    radius: Array
    h: Array
    l: Array
    grad_h: Array | None = None
    grad_l: Array | None = None


class KerrSpacetime:
    """A Kerr black hole; mass > 0 and |spin| <= mass (kerr.py:61-71)."""

    def __init__(self, mass: float = 1.0, spin: float = 0.0) -> None:
        if mass <= 0.0:
            raise ValueError("mass must be positive")
        if abs(spin) > mass:
            raise ValueError("Kerr bound violated: |spin| must be <= mass")
        self.mass = float(mass)
        self.spin = float(spin)

    # Analytic radii: kerr.py:73-112 (host-side scalar formulas).
    @property
    def outer_horizon_radius(self) -> float:
        m, a = self.mass, self.spin
        return m + math.sqrt(m * m - a * a)

    @property
    def inner_horizon_radius(self) -> float:
        m, a = self.mass, self.spin
        return m - math.sqrt(m * m - a * a)

    def ergosphere_radius(self, theta: float) -> float:
        m, a = self.mass, self.spin
        return m + math.sqrt(m * m - a * a * math.cos(theta) ** 2)

    def isco_radius(self, prograde: bool = True) -> float:
        chi = abs(self.spin) / self.mass
        z1 = 1.0 + (1.0 - chi * chi) ** (1.0 / 3.0) * (
            (1.0 + chi) ** (1.0 / 3.0) + (1.0 - chi) ** (1.0 / 3.0)
        )
        z2 = math.sqrt(3.0 * chi * chi + z1 * z1)
        root = math.sqrt((3.0 - z1) * (3.0 + z1 + 2.0 * z2))
        sign = -1.0 if prograde else 1.0
        return self.mass * (3.0 + z2 + sign * root)

    def photon_orbit_radius(self, prograde: bool = True) -> float:
        chi = abs(self.spin) / self.mass
        sign = -1.0 if prograde else 1.0
        angle = (2.0 / 3.0) * math.acos(sign * chi)
        return 2.0 * self.mass * (1.0 + math.cos(angle))

    def capture_radius(self, capture_margin: float) -> float:
        """r_plus (1 + margin), the tracer's capture test (tracer.py:84)."""
        return self.outer_horizon_radius * (1.0 + capture_margin)

    # ------------------------------------------------------------ device
    def geometry(self, x: Array, y: Array, z: Array,
                 gradients: bool = False) -> KerrSchildGeometry:
        """H, l and optionally their gradients at (x, y, z) (kerr.py:118-193).

        Inputs are 1-D arrays of one length (NumPy or CUDA tensors); the
        result uses the input's array type."""
        xs, host = to_device_f64(x, "x")
        ys, _ = to_device_f64(y, "y")
        zs, _ = to_device_f64(z, "z")
        if xs.dim() != 1 or xs.shape != ys.shape or xs.shape != zs.shape:
            raise ValueError("x, y, z must be 1-D arrays of equal length")
        n = xs.shape[0]
        dev = xs.device
        r = torch.empty(n, dtype=torch.float64, device=dev)
        h = torch.empty(n, dtype=torch.float64, device=dev)
        l = torch.empty((n, 3), dtype=torch.float64, device=dev)
        gh = torch.empty((n, 3), dtype=torch.float64, device=dev) if gradients else None
        gl = torch.empty((n, 3, 3), dtype=torch.float64, device=dev) if gradients else None
        _lib.check(_lib.load().bh_geometry(
            self.mass, self.spin, ptr(xs), ptr(ys), ptr(zs), 1, n, ptr(r), ptr(h),
            ptr(l), ptr(gh), ptr(gl), stream_handle()), "geometry")
        conv = lambda t: None if t is None else out_like(t, host, x)  # noqa: E731
        return KerrSchildGeometry(radius=conv(r), h=conv(h), l=conv(l),
                                  grad_h=conv(gh), grad_l=conv(gl))

    def kerr_schild_radius(self, x: Array, y: Array, z: Array) -> Array:
        """Kerr-Schild radius r (kerr.py:114-116)."""
        return self.geometry(x, y, z).radius

    def _l4(self, positions):
        pos, host = to_device_f64(positions, "positions")
        geo = self.geometry(pos[..., 1].contiguous(), pos[..., 2].contiguous(),
                            pos[..., 3].contiguous())
        ones = torch.ones_like(geo.h)
        return torch.cat([ones[:, None], geo.l], dim=-1), geo.h, pos, host

    def metric(self, positions: Array) -> Array:
        """g_mu_nu = eta + 2 H l_mu l_nu at (n, 4) positions (kerr.py:201-215)."""
        l4, h, pos, host = self._l4(positions)
        eta = torch.diag(torch.tensor([-1.0, 1.0, 1.0, 1.0], dtype=torch.float64,
                                      device=pos.device))
        g = eta + 2.0 * h[:, None, None] * l4[:, :, None] * l4[:, None, :]
        return out_like(g, host, positions)

    def inverse_metric(self, positions: Array) -> Array:
        """g^mu^nu = eta - 2 H l^mu l^nu at (n, 4) positions (kerr.py:217-235)."""
        l4, h, pos, host = self._l4(positions)
        l_up = torch.cat([-l4[:, :1], l4[:, 1:]], dim=-1)
        eta = torch.diag(torch.tensor([-1.0, 1.0, 1.0, 1.0], dtype=torch.float64,
                                      device=pos.device))
        g = eta - 2.0 * h[:, None, None] * l_up[:, :, None] * l_up[:, None, :]
        return out_like(g, host, positions)
