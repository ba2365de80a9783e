"""Emission stage of the offline renderer on the b200 backend.

Mirrors, for the offline frame:
- the host-side tables and scalars of blackhorizon/emission:
  - the Novikov-Thorne temperature table (novikov_thorne.py:48-120, the Page
    and Thorne 1974 flux);
  - the blackbody chromaticity table (blackbody.py:35-106: the Planck
    spectrum against the Wyman, Sloan and Shirley 2013 fits of the CIE 1931
    colour-matching functions, to linear sRGB);
  - the static-observer lapse (redshift.py:66-83);
  - the blue-sheet amplification and glow (bluesheet.py:50-118);
- ``render_hdr`` (offline/render.py:487-680): the b200 tile tracer
  (``offline.trace_frame``), then ``bh_offline_radiance``, which shades
  every ray on the device (starfield, redshifted disk, blue sheet) and
  averages the supersamples into a float32 HDR image.

The tables have a few thousand entries and are built once per frame with
NumPy, as the reference builds them; everything per ray runs on the device.
"""

from __future__ import annotations

import functools
import math

import numpy
import torch

from . import _lib
from .backend import ptr, stream_handle
from .kerr import KerrSpacetime
from .offline import (FlyCamera, OfflineSettings, camera_states, disk_inner_radius,
                      tetrad_camera_states, trace_frame)
from .tracer import DEFAULT_TIMEOUT_S

# ----------------------------------------------------------------- disk


def _radicand_roots(spin: float):
    """Roots of x^3 - 3 x + 2 a = 0 (x = sqrt(r / M)), largest first."""
    third = math.acos(max(-1.0, min(1.0, spin))) / 3.0
    return (2.0 * math.cos(third - math.pi / 3.0), 2.0 * math.cos(third + math.pi / 3.0),
            -2.0 * math.cos(third))


def page_thorne_flux(radii, spin: float):
    """Page-Thorne flux profile of the +phi disk, zero inside the ISCO
    (novikov_thorne.py:48-95): F(x) = 3 / (2 x^4 (x^3 - 3 x + 2 a)) [x - x0 -
    (3 a / 2) ln(x / x0) - sum_i 3 (x_i - a)^2 / (x_i (x_i - x_j) (x_i - x_k))
    ln((x - x_i) / (x0 - x_i))], x = sqrt(r)."""
    r = numpy.asarray(radii, dtype=float)
    r_isco = disk_inner_radius(KerrSpacetime(1.0, spin))
    x = numpy.sqrt(numpy.maximum(r, 1e-12))
    x0 = math.sqrt(r_isco)
    roots = _radicand_roots(spin)
    bracket = x - x0 - 1.5 * spin * numpy.log(numpy.maximum(x / x0, 1e-30))
    for i in range(3):
        xi, xj, xk = roots[i], roots[(i + 1) % 3], roots[(i + 2) % 3]
        if abs(xi) < 1e-12:
            continue  # (x_i - a)^2 / x_i -> 0 where a root sits at zero (a = 0)
        coefficient = 3.0 * (xi - spin) ** 2 / (xi * (xi - xj) * (xi - xk))
        bracket = bracket - coefficient * numpy.log(
            numpy.maximum((x - xi) / (x0 - xi), 1e-30))
    denominator = x ** 4 * (x ** 3 - 3.0 * x + 2.0 * spin)
    flux = numpy.where(r > r_isco, 1.5 * bracket / numpy.maximum(denominator, 1e-30), 0.0)
    return numpy.maximum(flux, 0.0)


def temperature_profile(radii, spin: float):
    """T(r) = F(r)^(1/4), dimensionless (novikov_thorne.py:98-100)."""
    return page_thorne_flux(radii, spin) ** 0.25


def temperature_lut(spin: float, outer_radius: float, size: int = 512):
    """(table float32 (size,), r_inner, r_outer): T / max T sampled linearly
    in radius from the ISCO to outer_radius (novikov_thorne.py:103-126)."""
    r_inner = disk_inner_radius(KerrSpacetime(1.0, spin))
    if outer_radius <= r_inner:
        raise ValueError("outer_radius must exceed the ISCO radius")
    profile = temperature_profile(numpy.linspace(r_inner, outer_radius, size), spin)
    peak = profile.max()
    if peak <= 0.0:
        raise RuntimeError("temperature profile unexpectedly vanished")
    return (profile / peak).astype(numpy.float32), float(r_inner), float(outer_radius)


# ------------------------------------------------------------ blackbody

# CODATA SI values (exact since 2019).
_PLANCK = 6.62607015e-34
_LIGHT = 2.99792458e8
_BOLTZMANN = 1.380649e-23
# Linear sRGB from CIE XYZ (IEC 61966-2-1).
_XYZ_TO_SRGB = numpy.array([[3.2406, -1.5372, -0.4986],
                            [-0.9689, 1.8758, 0.0415],
                            [0.0557, -0.2040, 1.0570]])
TEMPERATURE_MIN = 500.0
TEMPERATURE_MAX = 40000.0
# Wyman, Sloan and Shirley (2013) multi-lobe fits: (weight, mean nm, sigma
# below the mean, sigma above) per lobe.
_CMF_LOBES = (
    ((1.056, 599.8, 37.9, 31.0), (0.362, 442.0, 16.0, 26.7), (-0.065, 501.1, 20.4, 26.2)),
    ((0.821, 568.8, 46.9, 40.5), (0.286, 530.9, 16.3, 31.1)),
    ((1.217, 437.0, 11.8, 36.0), (0.681, 459.0, 26.0, 13.8)),
)


def _lobe(w, mean, sigma_low, sigma_high):
    sigma = numpy.where(w < mean, sigma_low, sigma_high)
    return numpy.exp(-0.5 * ((w - mean) / sigma) ** 2)


def color_matching_functions(wavelengths_nm):
    """CIE 1931 xbar, ybar, zbar (blackbody.py:37-49)."""
    out = []
    for lobes in _CMF_LOBES:
        weight, mean, lo, hi = lobes[0]
        total = weight * _lobe(wavelengths_nm, mean, lo, hi)
        for weight, mean, lo, hi in lobes[1:]:
            total = total + weight * _lobe(wavelengths_nm, mean, lo, hi)
        out.append(total)
    return tuple(out)


def planck_spectral_radiance(wavelengths_nm, temperature):
    """B_lambda(T) up to a common scale (blackbody.py:52-57)."""
    lam = wavelengths_nm * 1e-9
    exponent = numpy.minimum(_PLANCK * _LIGHT / (lam * _BOLTZMANN * temperature), 700.0)
    return 1.0 / (lam ** 5 * numpy.expm1(exponent))


def blackbody_rgb(temperature: float) -> numpy.ndarray:
    """Linear sRGB of a blackbody, largest channel 1 (blackbody.py:60-85)."""
    t = float(numpy.clip(temperature, TEMPERATURE_MIN, TEMPERATURE_MAX))
    wavelengths = numpy.linspace(380.0, 780.0, 200)
    spectrum = planck_spectral_radiance(wavelengths, t)
    xyz = numpy.array([numpy.trapezoid(spectrum * cmf, wavelengths)
                       for cmf in color_matching_functions(wavelengths)])
    rgb = numpy.maximum(_XYZ_TO_SRGB @ xyz, 0.0)
    peak = rgb.max()
    return numpy.array([1.0, 1.0, 1.0]) if peak <= 0.0 else rgb / peak


def blackbody_lut(size: int = 256):
    """(table float32 (size, 3), log_t_min, log_t_max) over log-spaced
    temperatures from 500 K to 40000 K (blackbody.py:88-106)."""
    log_min = float(numpy.log(TEMPERATURE_MIN))
    log_max = float(numpy.log(TEMPERATURE_MAX))
    temperatures = numpy.exp(numpy.linspace(log_min, log_max, size))
    table = numpy.stack([blackbody_rgb(t) for t in temperatures])
    return table.astype(numpy.float32), log_min, log_max


# ---------------------------------------------------- observers and sheet


def static_observer_lapse(spacetime: KerrSpacetime, position) -> float:
    """u^t = 1 / sqrt(-g_tt) of a static observer (redshift.py:66-83);
    ValueError inside the ergosphere."""
    p = numpy.asarray(position, dtype=float)
    geo = spacetime.geometry(p[None, 0], p[None, 1], p[None, 2])
    g_tt = 2.0 * float(numpy.asarray(geo.h)[0]) - 1.0
    if g_tt >= 0.0:
        raise ValueError("camera inside the ergosphere has no static frame")
    return 1.0 / numpy.sqrt(-g_tt)


DEFAULT_MATCHING_PROXIMITY = 0.5
DEFAULT_AMPLIFICATION_CAP = 60.0
SHEET_COLOR = (0.62, 0.78, 1.0)


def blueshift_amplification(spacetime: KerrSpacetime, radius,
                            matching_proximity: float = DEFAULT_MATCHING_PROXIMITY,
                            cap: float = DEFAULT_AMPLIFICATION_CAP):
    """B(r) = clip(x_match / x, 1, cap) with x = (r - r_minus) / (r_plus -
    r_minus) clamped to [1e-6, 1]; 1 without an inner horizon
    (bluesheet.py:50-95)."""
    r = numpy.asarray(radius, dtype=float)
    r_plus = float(spacetime.outer_horizon_radius)
    r_minus = float(spacetime.inner_horizon_radius)
    if r_minus <= 0.0:
        return numpy.ones_like(r)
    x = numpy.clip((r - r_minus) / max(r_plus - r_minus, 1e-12), 1e-6, 1.0)
    return numpy.clip(matching_proximity / x, 1.0, cap)


DISPLAY_CAP = 8.0
WHITEOUT_START = 8.0
WHITEOUT_END = 30.0


def display_amplification(amplification):
    """The amplification a display adapts to: clip(B, 1, 8) (bluesheet.py:126-136)."""
    return numpy.clip(numpy.asarray(amplification, dtype=float), 1.0, DISPLAY_CAP)


def whiteout_fraction(amplification):
    """0.92 smoothstep((B - 8) / 22) (bluesheet.py:139-155)."""
    t = numpy.clip((numpy.asarray(amplification, dtype=float) - WHITEOUT_START)
                   / (WHITEOUT_END - WHITEOUT_START), 0.0, 1.0)
    return 0.92 * t * t * (3.0 - 2.0 * t)


def sheet_radiance(amplification, base_intensity: float = 0.02):
    """Radiance of rays ending on the blue sheet: base (B - 1)^4
    (bluesheet.py:98-108)."""
    return base_intensity * (numpy.asarray(amplification, dtype=float) - 1.0) ** 4


# ------------------------------------------------------------- radiance


def radiance_image(spacetime: KerrSpacetime, status, escape_directions, hit_positions,
                   hit_momenta, width: int, height: int, settings: OfflineSettings,
                   observer_lapse: float, energy=None, sheet_rgb=None, tables=None):
    """float32 HDR image (height, width, 3) on the device from the per-ray
    outputs of a traced frame (pixel-major, supersample^2 rays per pixel).
    ``energy``: the rays' initial p_t (tetrad cameras); ``sheet_rgb``: the
    radiance of TERMINATED rays; ``tables``: the result of ``frame_tables``."""
    dev = status.device
    t = tables if tables is not None else frame_tables(spacetime, settings, dev)
    n_rays = width * height * settings.supersample ** 2
    for name, arr in (("status", status), ("escape_directions", escape_directions),
                      ("hit_positions", hit_positions), ("hit_momenta", hit_momenta)):
        if arr.shape[0] != n_rays:
            raise ValueError(f"{name} must hold width * height * supersample^2 rays")
    sheet = (0.0, 0.0, 0.0) if sheet_rgb is None else tuple(float(v) for v in sheet_rgb)
    cfg = _lib.EmissionConfig(
        mass=spacetime.mass, spin=spacetime.spin, disk_inner=t["disk_inner"],
        disk_temperature=float(settings.disk_temperature),
        disk_detail=float(settings.disk_detail), observer_lapse=float(observer_lapse),
        bb_log_min=t["bb_log_min"], bb_log_max=t["bb_log_max"], sheet_rgb=sheet,
        temperature_size=t["temperature"].numel(), blackbody_size=t["blackbody"].shape[0],
        supersample=int(settings.supersample), reserved=0)
    hdr = torch.empty((height, width, 3), dtype=torch.float32, device=dev)
    st = status.to(torch.int32).contiguous()
    e = None if energy is None else energy.to(torch.float64).contiguous()
    dirs, hp, hm = (a.to(torch.float64).contiguous()
                    for a in (escape_directions, hit_positions, hit_momenta))
    _lib.check(_lib.load().bh_offline_radiance(
        cfg, ptr(st), ptr(dirs), ptr(hp), ptr(hm), ptr(e) if e is not None else None,
        width, height, ptr(t["temperature"]), ptr(t["radii"]), ptr(t["blackbody"]), ptr(hdr),
        stream_handle()), "offline radiance")
    return hdr


@functools.lru_cache(maxsize=32)
def _host_tables(spin: float, disk_outer_radius: float):
    disk_inner = disk_inner_radius(KerrSpacetime(1.0, spin))
    disk_outer = max(disk_outer_radius, disk_inner + 1.0)
    temperature, _, _ = temperature_lut(spin, disk_outer, size=2048)
    radii = numpy.linspace(disk_inner, disk_outer, temperature.shape[0])
    return float(disk_inner), float(disk_outer), temperature, radii


@functools.lru_cache(maxsize=1)
def _host_blackbody():
    return blackbody_lut(size=1024)


def frame_tables(spacetime: KerrSpacetime, settings: OfflineSettings, device) -> dict:
    """The lookup tables of render_hdr (render.py:527-532) on the device:
    the 2048-entry temperature table on its radii, the 1024-row blackbody
    table and its log-temperature range.  The host tables are built once per
    (spin, outer radius) and kept."""
    if spacetime.mass != 1.0:
        raise ValueError("the offline renderer's tables assume M = 1")
    disk_inner, disk_outer, temperature, radii = _host_tables(float(spacetime.spin),
                                                              float(settings.disk_outer_radius))
    blackbody, log_min, log_max = _host_blackbody()
    return {"disk_inner": disk_inner, "disk_outer": disk_outer,
            "temperature": torch.as_tensor(temperature, device=device),
            "radii": torch.as_tensor(radii, device=device),
            "blackbody": torch.as_tensor(blackbody, device=device).contiguous(),
            "bb_log_min": log_min, "bb_log_max": log_max}


def render_hdr(camera: FlyCamera, width: int, height: int, settings: OfflineSettings,
               progress: bool = False, camera_tetrad=None, interior_stop: float | None = None,
               *, precision: str = "fp64", tile_rays: int | None = None,
               timeout_s: float = DEFAULT_TIMEOUT_S, return_rays: bool = False):
    """Linear HDR frame (height, width, 3) float32 on the device, as
    render_hdr computes it (render.py:487-680): the tile tracer with the
    photon-shell retrace (``offline.trace_frame``), then every ray shaded on
    the device and the supersamples averaged.  Exterior cameras see by the
    static-observer lapse (1 inside the ergosphere); tetrad cameras
    (``camera_tetrad``) by the blue-sheet amplification of the camera radius
    when the terminal surface is the inner horizon (``interior_stop`` >=
    0.99 r_minus), with each escaped ray shifted by B / E and TERMINATED rays
    glowing.  ``progress`` is accepted for signature parity and ignored.
    ``return_rays`` also returns the traced ``FrameRays``."""
    spacetime = KerrSpacetime(mass=1.0, spin=settings.spin)
    dev = torch.device("cuda", torch.cuda.current_device())
    if camera_tetrad is not None:
        inner = float(spacetime.inner_horizon_radius)
        sheet_active = inner > 1e-9 and interior_stop is not None and interior_stop >= inner * 0.99
        pos = numpy.asarray(camera.position, dtype=float)
        camera_radius = float(numpy.asarray(spacetime.kerr_schild_radius(
            pos[None, 0], pos[None, 1], pos[None, 2]))[0])
        lapse = float(blueshift_amplification(spacetime, numpy.array([camera_radius]))[0]) \
            if sheet_active else 1.0
        s0 = tetrad_camera_states(camera, spacetime, camera_tetrad, width, height, settings, dev)
        energy = s0[:, 4]
    else:
        try:
            lapse = float(static_observer_lapse(spacetime, camera.position))
        except ValueError:
            lapse = 1.0
        s0 = camera_states(camera, spacetime, width, height, settings, dev)
        energy = None
    rays = trace_frame(camera, width, height, settings, precision=precision, tile_rays=tile_rays,
                       timeout_s=timeout_s, state0=s0, camera_tetrad=camera_tetrad,
                       interior_stop=interior_stop)
    sheet = None
    if camera_tetrad is not None and lapse > 1.0:
        glow = float(sheet_radiance(numpy.array([lapse]))[0])
        sheet = glow * numpy.array(SHEET_COLOR, dtype=numpy.float32)  # float32, as render.py:646
    hdr = radiance_image(spacetime, rays.status, rays.escape_directions, rays.hit_positions,
                         rays.hit_momenta, width, height, settings, lapse, energy=energy,
                         sheet_rgb=sheet, tables=frame_tables(spacetime, settings, dev))
    return (hdr, rays) if return_rays else hdr


__all__ = ["page_thorne_flux", "temperature_profile", "temperature_lut",
           "color_matching_functions", "planck_spectral_radiance", "blackbody_rgb",
           "blackbody_lut", "static_observer_lapse", "blueshift_amplification",
           "sheet_radiance", "SHEET_COLOR", "radiance_image", "frame_tables", "render_hdr"]
