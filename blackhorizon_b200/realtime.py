"""The real-time renderer's ray tracing on the b200 backend.

Mirrors blackhorizon/realtime/settings.py (``RenderSettings``,
``QualityPreset``, ``BackgroundMode``) and blackhorizon/realtime/reference.py
(``trace_like_shader``, ``ReferenceResult``): the fixed-step RK4 shader
algorithm runs as a persistent CUDA kernel (libbh_b200 ``bh_trace_realtime``)
writing into device buffers.  The reference's GL viewer (window, fragment
shader, framebuffers) is not part of this package: the kernel is the
headless equivalent of its tracing loop.
"""

from __future__ import annotations

from dataclasses import dataclass, replace
from enum import Enum

import numpy
import torch

from . import _lib
from .backend import Array, ptr, stream_handle, to_device_f64
from .kerr import KerrSpacetime


class BackgroundMode(int, Enum):
    """Celestial sphere styles (settings.py:13-17)."""

    CHECKERBOARD = 0
    STARFIELD = 1


class QualityPreset(str, Enum):
    """Named fidelity levels (settings.py:20-26)."""

    LOW = "low"
    MEDIUM = "medium"
    HIGH = "high"
    ULTRA = "ultra"


_PRESET_VALUES = {
    QualityPreset.LOW: {"max_steps": 256, "step_scale": 0.35, "resolution_scale": 0.5},
    QualityPreset.MEDIUM: {"max_steps": 512, "step_scale": 0.22, "resolution_scale": 0.75},
    QualityPreset.HIGH: {"max_steps": 1024, "step_scale": 0.14, "resolution_scale": 1.0},
    QualityPreset.ULTRA: {"max_steps": 2048, "step_scale": 0.08, "resolution_scale": 1.0},
}

MAX_STEPS_HARD_LIMIT = 4096
"""Largest step budget (the shader's compile-time loop bound)."""


@dataclass
class RenderSettings:
    """Tunables of the real-time tracer (settings.py:54-173); the tracing
    kernel uses max_steps, step_scale, min_step, max_step, capture_margin,
    momentum_bailout, escape_radius and the disk radius."""

    spin: float = 0.9
    fov_degrees: float = 60.0
    max_steps: int = 512
    step_scale: float = 0.22
    min_step: float = 1e-4
    max_step: float = 4.0
    resolution_scale: float = 0.75
    capture_margin: float = 2e-2
    escape_radius: float = 0.0
    momentum_bailout: float = 1e3
    background: BackgroundMode = BackgroundMode.CHECKERBOARD
    interior_mode: bool = False
    interior_journey: str = "realistic"
    interior_stop: float = 0.02
    disk_enabled: bool = True
    disk_outer_radius: float = 18.0
    disk_temperature: float = 6500.0
    disk_detail: float = 1.0
    exposure: float = 1.0

    def validate(self) -> None:
        """Raise ValueError if any field is outside its legal range."""
        if not -1.0 <= self.spin <= 1.0:
            raise ValueError("spin must be in [-1, 1]")
        if not 1.0 <= self.fov_degrees <= 170.0:
            raise ValueError("fov_degrees must be in [1, 170]")
        if not 1 <= self.max_steps <= MAX_STEPS_HARD_LIMIT:
            raise ValueError(f"max_steps must be in [1, {MAX_STEPS_HARD_LIMIT}]")
        if self.step_scale <= 0.0:
            raise ValueError("step_scale must be positive")
        if not 0.0 < self.min_step <= self.max_step:
            raise ValueError("require 0 < min_step <= max_step")
        if not 0.05 <= self.resolution_scale <= 1.0:
            raise ValueError("resolution_scale must be in [0.05, 1]")
        if self.capture_margin < 0.0:
            raise ValueError("capture_margin must be non-negative")
        if self.momentum_bailout <= 1.0:
            raise ValueError("momentum_bailout must exceed 1")
        if self.interior_journey not in ("realistic", "idealized"):
            raise ValueError("interior_journey must be realistic or idealized")
        if not 1e-4 <= self.interior_stop <= 1.0:
            raise ValueError("interior_stop must be in [1e-4, 1] M")
        if self.disk_outer_radius <= 1.0:
            raise ValueError("disk_outer_radius must exceed 1 M")
        if not 500.0 <= self.disk_temperature <= 40000.0:
            raise ValueError("disk_temperature must be in [500, 40000] K")
        if not 0.0 <= self.disk_detail <= 1.0:
            raise ValueError("disk_detail must be in [0, 1]")
        if self.exposure <= 0.0:
            raise ValueError("exposure must be positive")

    def apply_preset(self, preset: QualityPreset) -> "RenderSettings":
        """A copy with a quality preset applied."""
        return replace(self, **_PRESET_VALUES[QualityPreset(preset)])

    def effective_escape_radius(self, camera_distance: float) -> float:
        """Escape radius for a camera at the given distance."""
        if self.escape_radius > 0.0:
            return self.escape_radius
        return max(2.0 * camera_distance, 100.0)


@dataclass(frozen=True)
class ReferenceResult:
    """Rays traced with the shader algorithm (reference.py:24-38): status,
    final positions (n, 3) and momenta (n, 4); with a disk, the crossing
    radius, position and momentum of DISK rays (NaN elsewhere).  ``steps``
    is the number of RK4 steps all rays took together."""

    status: Array
    positions: Array
    momenta: Array
    hit_radii: Array | None = None
    hit_positions: Array | None = None
    hit_momenta: Array | None = None
    steps: int = 0


def trace_like_shader(spacetime: KerrSpacetime, state0: Array, settings: RenderSettings,
                      escape_radius: float, disk_radii=None, interior_stop=None, *,
                      precision: str = "fp64") -> ReferenceResult:
    """Trace rays as the real-time shader does (reference.py:41-188).

    ``precision='mixed'`` runs the RK4 stages in float32 (the shader's own
    precision) with the state kept in float64.  NumPy in, NumPy out; device
    tensor in, device tensors out."""
    s, host = to_device_f64(state0, "state0")
    if s.dim() != 2 or s.shape[1] != 8:
        raise ValueError("state0 must have shape (n, 8)")
    status, states, hit_r, hit_p, hit_m, steps = _trace_shader_device(
        spacetime, s, settings, escape_radius, disk_radii, interior_stop, precision)
    conv = (lambda t: t.cpu().numpy()) if host is not None else (lambda t: t)  # noqa: E731
    disk = disk_radii is not None
    return ReferenceResult(status=conv(status), positions=conv(states[:, 1:4].contiguous()),
                           momenta=conv(states[:, 4:8].contiguous()),
                           hit_radii=conv(hit_r) if disk else None,
                           hit_positions=conv(hit_p) if disk else None,
                           hit_momenta=conv(hit_m) if disk else None,
                           steps=steps)


def _trace_shader_device(spacetime, s, settings, escape_radius, disk_radii, interior_stop,
                         precision):
    """bh_trace_realtime on a device state tensor: (status, final states (n, 8),
    hit radii, hit positions, hit momenta, RK4 steps), all device tensors but
    the step count."""
    n = s.shape[0]
    dev = s.device
    lib = _lib.load()
    states = torch.empty_like(s)
    status = torch.empty(n, dtype=torch.int32, device=dev)
    hit_r = torch.empty(n, dtype=torch.float64, device=dev)
    hit_p = torch.empty((n, 3), dtype=torch.float64, device=dev)
    hit_m = torch.empty((n, 4), dtype=torch.float64, device=dev)
    ws = torch.empty(lib.bh_trace_workspace_bytes(), dtype=torch.uint8, device=dev)
    r_in, r_out = (0.0, 0.0) if disk_radii is None else (float(disk_radii[0]),
                                                          float(disk_radii[1]))
    cfg = _lib.RealtimeConfig(int(settings.max_steps), float(settings.step_scale),
                              float(settings.min_step), float(settings.max_step),
                              float(settings.capture_margin), float(settings.momentum_bailout),
                              float(escape_radius), r_in, r_out,
                              0.0 if interior_stop is None else float(interior_stop),
                              _lib.PRECISION[precision], 0)
    stream = stream_handle()
    _lib.check(lib.bh_trace_realtime(cfg, float(spacetime.mass), float(spacetime.spin), ptr(s),
                                     ptr(states), ptr(status), ptr(hit_r), ptr(hit_p), ptr(hit_m),
                                     n, ptr(ws), stream), "trace_like_shader")
    stats = _lib.TraceStats()
    _lib.check(lib.bh_trace_stats_read(ptr(ws), stats, stream), "trace_like_shader")
    return status, states, hit_r, hit_p, hit_m, int(stats.attempts)


# ------------------------------------------------------------ headless frame


def _viewer_tables(spin: float, outer: float):
    """The viewer's lookup textures (engine.py:55-58, 102-123): the 512-entry
    temperature table and the 256-row blackbody table, kept per (spin, outer)."""
    from .emission import blackbody_lut, temperature_lut

    key = (round(float(spin), 12), round(float(outer), 12))
    hit = _TABLE_CACHE.get(key)
    if hit is None:
        temperature, r_inner, _ = temperature_lut(spin, outer)
        blackbody, log_min, log_max = blackbody_lut()
        hit = (temperature, float(r_inner), blackbody, float(log_min), float(log_max))
        _TABLE_CACHE[key] = hit
    return hit


_TABLE_CACHE: dict = {}


def _interior_view(spacetime: KerrSpacetime, camera, settings: RenderSettings):
    """Tetrad, stop radius and blue-sheet uniforms of an interior camera
    (engine.py:125-215): the camera's 4-velocity when it carries a finite
    one, else the rain observer; the terminal surface at max(stop, 1.02
    r_minus) on the realistic journey; the amplification B of the camera
    radius, its display value clip(B, 1, 8), the glow and the whiteout."""
    from .emission import (blueshift_amplification, display_amplification, sheet_radiance,
                           whiteout_fraction)
    from .frames import build_tetrad, rain_four_velocity

    position = numpy.asarray(camera.position, dtype=float)
    stop = float(settings.interior_stop)
    radius = float(numpy.linalg.norm(position))
    if not numpy.isfinite(position).all() or radius < stop:
        direction = position / radius if radius > 1e-9 else numpy.array([1.0, 0.0, 0.0])
        position = direction * max(stop, 1e-3)
    forward, _, up = camera.basis()
    velocity = getattr(camera, "four_velocity", None)
    try:
        if velocity is None or not numpy.isfinite(velocity).all():
            raise ValueError("missing or non-finite 4-velocity")
        tetrad = build_tetrad(spacetime, position, velocity, forward, up)
    except ValueError:
        tetrad = build_tetrad(spacetime, position,
                              rain_four_velocity(spacetime, position[None, :])[0], forward, up)
    inner = float(spacetime.inner_horizon_radius)
    effective_stop = stop if settings.interior_journey == "idealized" else max(stop, inner * 1.02)
    amplification = 1.0
    if settings.interior_journey == "realistic" and inner > 1e-9:
        r_cam = float(numpy.asarray(spacetime.kerr_schild_radius(
            position[None, 0], position[None, 1], position[None, 2]))[0])
        amplification = float(blueshift_amplification(spacetime, numpy.array([r_cam]))[0])
    display = float(display_amplification(numpy.array([amplification]))[0])
    return {"tetrad": tetrad, "stop": effective_stop, "display": display,
            "glow": float(sheet_radiance(numpy.array([display]))[0]),
            "white": float(whiteout_fraction(numpy.array([amplification]))[0])}


def _static_lapse(spacetime: KerrSpacetime, position) -> float:
    """engine.py:217-233: 1 / sqrt(-g_tt), 1 where g_tt >= -1e-3."""
    p = numpy.asarray(position, dtype=float)
    geo = spacetime.geometry(p[None, 0], p[None, 1], p[None, 2])
    g_tt = 2.0 * float(numpy.asarray(geo.h)[0]) - 1.0
    return 1.0 if g_tt >= -1e-3 else 1.0 / float(numpy.sqrt(-g_tt))


def render_frame_device(settings: RenderSettings, camera, width: int, height: int, *,
                        precision: str = "fp64", return_rays: bool = False):
    """One frame of the real-time viewer as an (height, width, 3) uint8 device
    tensor, row 0 at the top (headless.py:32-48, engine.py:235-330): the
    camera's rays (pinhole, or the observer's tetrad in interior mode) built
    on the device, traced by the shader algorithm (``trace_like_shader``) and
    shaded as kerr_tracer.frag shades them (``bh_realtime_shade``).
    ``return_rays`` also returns the trace (a ReferenceResult of device
    tensors) and the shading uniforms with their tables."""
    from .offline import device_camera_rays, disk_inner_radius

    settings.validate()
    if width < 1 or height < 1:
        raise ValueError("width and height must be >= 1")
    spacetime = KerrSpacetime(mass=1.0, spin=settings.spin)
    inner = disk_inner_radius(spacetime)
    outer = max(settings.disk_outer_radius, inner + 1.0)
    temperature, t_inner, blackbody, log_min, log_max = _viewer_tables(settings.spin, outer)
    dev = torch.device("cuda", torch.cuda.current_device())
    interior = _interior_view(spacetime, camera, settings) if settings.interior_mode else None
    s0 = device_camera_rays(spacetime, camera, width, height, settings.fov_degrees, 1,
                            interior["tetrad"] if interior else None, dev)
    escape = settings.effective_escape_radius(camera.distance_from_origin)
    disk_radii = (inner, outer) if settings.disk_enabled else None
    # The shader reads the traced states and hits where the kernel wrote them
    # (it reads columns 1-7 of a state, and the hits only of disk rays).
    status, states, hit_r, hit_p, hit_m, steps = _trace_shader_device(
        spacetime, s0, settings, escape, disk_radii,
        interior["stop"] if interior else None, precision)
    cfg = _lib.RealtimeShading(
        mass=1.0, spin=float(settings.spin), disk_inner=t_inner, disk_outer=float(outer),
        disk_temperature=float(settings.disk_temperature),
        disk_detail=float(settings.disk_detail), exposure=float(settings.exposure),
        observer_lapse=interior["display"] if interior else _static_lapse(spacetime,
                                                                          camera.position),
        bb_log_min=log_min, bb_log_max=log_max,
        sky_amplification=interior["display"] if interior else 0.0,
        sheet_radiance=interior["glow"] if interior else 0.0,
        whiteout=interior["white"] if interior else 0.0,
        background=int(settings.background), temperature_size=int(temperature.size),
        blackbody_size=int(blackbody.shape[0]), reserved=0)
    t_dev = torch.as_tensor(temperature, device=dev)
    bb_dev = torch.as_tensor(blackbody, device=dev).contiguous()
    rgb = torch.empty((height, width, 3), dtype=torch.uint8, device=dev)
    _lib.check(_lib.load().bh_realtime_shade(
        cfg, ptr(status), ptr(states), ptr(hit_p), ptr(hit_m), width, height, ptr(t_dev),
        ptr(bb_dev), ptr(rgb), stream_handle()), "realtime shade")
    if return_rays:
        disk = disk_radii is not None
        res = ReferenceResult(status=status, positions=states[:, 1:4].contiguous(),
                              momenta=states[:, 4:8].contiguous(),
                              hit_radii=hit_r if disk else None,
                              hit_positions=hit_p if disk else None,
                              hit_momenta=hit_m if disk else None, steps=steps)
        shading = {k: getattr(cfg, k) for k, _ in _lib.RealtimeShading._fields_}
        shading.update(temperature=temperature, blackbody=blackbody, states=states,
                       hit_positions=hit_p, hit_momenta=hit_m)
        return rgb, res, shading
    return rgb


def render_frame(settings: RenderSettings, camera, width: int, height: int, ctx=None, *,
                 precision: str = "fp64") -> numpy.ndarray:
    """headless.render_frame (headless.py:32-48): one frame of the real-time
    viewer as a (height, width, 3) uint8 array, row 0 at the top, rendered by
    the device kernels instead of an OpenGL context (``ctx`` is accepted for
    signature parity and must be None)."""
    if ctx is not None:
        raise ValueError("the b200 backend renders without an OpenGL context")
    return render_frame_device(settings, camera, width, height, precision=precision).cpu().numpy()
