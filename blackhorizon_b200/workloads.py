"""Synthetic workloads of the geodesic hot path (host-side NumPy, no GPU).

These are the benchmark and parity inputs, built from seeds so that the
benchmark, the tests and the fixture generator all rebuild the same rays.

* ``raw_throughput_inputs`` -- photons with Kerr-Schild radius exactly 30 M,
  positions and directions uniform on the sphere, spin uniform in
  [-0.95, 0.95] per ray.  Three independent streams (spawned from one seed)
  keep every prefix of the batch identical to the same prefix of the full
  2^20-ray batch.
* ``SHADOW_SMALL`` / ``SHADOW_FULL_HD`` / ``DIFFERENTIABLE`` -- pinhole
  camera frames (camera.py:69-94 orbit placement).
* ``uneven_cameras`` -- the 64-camera batch of mixed resolution, spin,
  inclination and distance.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

RAW_SEED = 20260
RAW_RADIUS = 30.0
RAW_SPIN_MAX = 0.95
RAW_N = 1 << 20
RAW_STEPS = 2000
RAW_RTOL = 1e-8
RAW_ATOL = 1e-10
RAW_H0 = 0.1
RAW_MAX_STEP = 2.0

UNEVEN_SEED = 20264


def raw_throughput_inputs(n: int, seed: int = RAW_SEED, offset: int = 0):
    """Positions (n,3), directions (n,3) and spins (n,) of rays
    [offset, offset+n) of the raw-throughput workload."""
    ss = np.random.SeedSequence(seed)
    ru, rs, ra = (np.random.default_rng(s) for s in ss.spawn(3))
    total = offset + n
    u = ru.normal(size=(total, 3))[offset:]
    s = rs.normal(size=(total, 3))[offset:]
    spin = ra.uniform(-RAW_SPIN_MAX, RAW_SPIN_MAX, size=total)[offset:]
    u /= np.linalg.norm(u, axis=-1, keepdims=True)
    s /= np.linalg.norm(s, axis=-1, keepdims=True)
    r = RAW_RADIUS
    # x + iy on the circle of radius sqrt(r^2 + a^2), z = r u_z, which puts
    # the point exactly on the Kerr-Schild radius r.
    rho = np.sqrt(r * r + spin * spin)
    pos = np.stack([rho * u[:, 0], rho * u[:, 1], r * u[:, 2]], axis=-1)
    return pos, s, spin


@dataclass(frozen=True)
class ShadowConfig:
    """A pinhole-camera shadow frame and its tracer controls."""

    name: str
    spin: float
    distance: float
    inclination: float
    fov: float
    width: int
    height: int
    escape_radius: float
    max_steps: int
    rtol: float
    atol: float
    capture_margin: float

    @property
    def n(self) -> int:
        return self.width * self.height


SHADOW_SMALL = ShadowConfig(
    "shadow-160x120-a0.9-i60", 0.9, 50.0, 60.0, 30.0, 160, 120, 100.0, 5000,
    1e-8, 1e-10, 0.01,
)
SHADOW_FULL_HD = ShadowConfig(
    "shadow-1920x1080-a0.9-i80", 0.9, 50.0, 80.0, 25.0, 1920, 1080, 100.0,
    10000, 1e-9, 1e-12, 0.01,
)
DIFFERENTIABLE = ShadowConfig(
    "adjoint-256x256-a0.7-i60", 0.7, 50.0, 60.0, 30.0, 256, 256, 100.0, 10000,
    1e-9, 1e-12, 0.01,
)


@dataclass(frozen=True)
class OfflineFrameConfig:
    """An offline-renderer frame: FlyCamera on the orbit sphere looking at
    the hole, subpixel rays traced with disk crossings (two passes)."""

    name: str
    spin: float
    distance: float
    inclination: float
    azimuth: float
    width: int
    height: int
    supersample: int
    max_steps: int

    @property
    def n(self) -> int:
        return self.width * self.height * self.supersample ** 2


# The offline renderer's command-line defaults (render.py:684-707):
# 1280x800, supersample 2 (4,096,000 rays), a=0.9, D=26 M, inclination 82,
# fov 70, disk from the ISCO to 18 M, rtol 1e-9 then 1e-11, 12000 steps.
OFFLINE_FRAME = OfflineFrameConfig("offline-1280x800-ss2-a0.9-i82", 0.9, 26.0, 82.0, 0.0,
                                   1280, 800, 2, 12000)


@dataclass(frozen=True)
class RealtimeFrameConfig:
    """A real-time viewer frame: pinhole camera on the orbit sphere, the
    shader algorithm at a quality preset, disk from the ISCO to 18 M."""

    name: str
    spin: float
    distance: float
    inclination: float
    fov: float
    width: int
    height: int
    preset: str

    @property
    def n(self) -> int:
        return self.width * self.height

    @property
    def escape_radius(self) -> float:
        # realtime/settings.py:166-173 (effective_escape_radius)
        return max(2.0 * self.distance, 100.0)


# A 1280x720 frame at the MEDIUM preset (512 steps), a=0.9, r=30 M,
# inclination 80 deg, fov 60 deg (the real-time defaults).
REALTIME_FRAME = RealtimeFrameConfig("realtime-1280x720-medium-a0.9-i80", 0.9, 30.0, 80.0,
                                     60.0, 1280, 720, "medium")


@dataclass(frozen=True)
class UnevenCamera:
    spin: float
    inclination: float
    distance: float
    width: int
    height: int
    fov: float = 30.0

    @property
    def escape_radius(self) -> float:
        return 2.0 * self.distance


def uneven_cameras(count: int = 64, seed: int = UNEVEN_SEED):
    """Cameras with log-uniform pixel area between 64x64 and 1024x768 (4:3),
    spin in [-0.998, 0.998], inclination in [0, 90] deg, distance in
    [20, 200] M."""
    rng = np.random.default_rng(seed)
    area = np.exp(rng.uniform(np.log(64 * 64), np.log(1024 * 768), size=count))
    spin = rng.uniform(-0.998, 0.998, size=count)
    inc = rng.uniform(0.0, 90.0, size=count)
    dist = rng.uniform(20.0, 200.0, size=count)
    cams = []
    for k in range(count):
        w = int(np.clip(round(np.sqrt(area[k] * 4.0 / 3.0)), 64, 1024))
        h = int(np.clip(round(w * 3 / 4), 48, 768))
        cams.append(UnevenCamera(float(spin[k]), float(inc[k]), float(dist[k]), w, h))
    return cams


def ks_radius_np(states, spin):
    """Kerr-Schild radius of (n, 8) states with per-ray spin (kerr.py:135-141),
    NumPy, for host-side bookkeeping of end points."""
    x, y, z = states[:, 1], states[:, 2], states[:, 3]
    a2 = np.asarray(spin, dtype=np.float64) ** 2
    q = x * x + y * y + z * z - a2
    with np.errstate(invalid="ignore", over="ignore"):
        return np.sqrt(0.5 * (q + np.sqrt(q * q + 4.0 * a2 * z * z)))


# End points inside this Kerr-Schild radius belong to rays that fell through
# the horizon during a no-termination run; their coordinates run toward the
# singularity and are excluded (and counted) when end points are compared.
PLUNGE_RADIUS = 2.5


def shadow_edge(status, width: int, height: int):
    """Pixels of a row-major status image with a 4-neighbour of another status
    (the shadow edge, where classification is chaotic)."""
    st = np.asarray(status).reshape(height, width)
    e = np.zeros_like(st, dtype=bool)
    e[1:, :] |= st[1:, :] != st[:-1, :]
    e[:-1, :] |= st[:-1, :] != st[1:, :]
    e[:, 1:] |= st[:, 1:] != st[:, :-1]
    e[:, :-1] |= st[:, :-1] != st[:, 1:]
    return e.reshape(-1)
