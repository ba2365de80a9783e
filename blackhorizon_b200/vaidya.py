"""The charged-Vaidya/Ori mass-inflation surrogate, b200 backend.

Mirrors blackhorizon/vaidya.py (``ChargedVaidyaSpacetime``,
``VaidyaGeometry``, ``FrozenVaidyaSlice``, ``vaidya_geodesic_rhs``) and the
tracing of the mass-inflation renderer (offline/inflation.py: ``rain_state``,
``camera_four_velocity``, ``_trace_vaidya_tile`` as ``trace_vaidya_tile``).

The shell table (the co-integrated Ori shell ODE) is integrated by the
library on the host (``bh_vaidya_shell_table``) and copied once to each
device that uses it; the mass function, the time-dependent geometry, the
Hamiltonian flow and the tile tracer run on the device.  The closed-form
Price-tail history (``ingoing_mass``, ``ingoing_mass_rate``,
``metric_function``) and table look-ups (``shell_radius``,
``inflated_mass_increment``) are host NumPy, as in the reference.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy
import torch

from . import _lib
from .backend import Array, ptr, stream_handle, to_device_f64


@dataclass(frozen=True)
class VaidyaGeometry:
    """Point samples of the surrogate (vaidya.py:68-84)."""

    h: Array
    l: Array
    h_spatial_scale: Array
    h_t: Array
    radius: Array


@dataclass
class ChargedVaidyaSpacetime:
    """The Ori surrogate in Cartesian Kerr-Schild form (vaidya.py:87-330)."""

    mass: float = 1.0
    charge: float = 0.9
    tail_mass: float = 0.01
    tail_start: float = 12.0
    tail_power: float = 12.0
    shell_energy: float = 1e-3
    shell_start_v: float = 14.0
    shell_start_radius: float = 1.0
    shell_width: float = 0.02
    mass_cap: float = 1e7
    time_dependent: bool = True
    _shell_v: numpy.ndarray = field(init=False, repr=False)
    _shell_r: numpy.ndarray = field(init=False, repr=False)
    _shell_m2: numpy.ndarray = field(init=False, repr=False)
    _device_tables: dict = field(init=False, repr=False, default_factory=dict)

    def __post_init__(self) -> None:
        if not 0.0 < self.charge < self.mass:
            raise ValueError("charge must lie in (0, mass)")
        if not (self.inner_horizon_radius < self.shell_start_radius < self.outer_horizon_radius):
            raise ValueError("shell must launch strictly between the horizons")
        lib = _lib.load()
        st = self._struct(None, 0)
        rows = int(lib.bh_vaidya_shell_table(st, None, None, None, 0))
        if rows < 1:
            raise RuntimeError("shell table integration failed")
        self._shell_v = numpy.empty(rows)
        self._shell_r = numpy.empty(rows)
        self._shell_m2 = numpy.empty(rows)
        lib.bh_vaidya_shell_table(st, self._shell_v.ctypes.data, self._shell_r.ctypes.data,
                                  self._shell_m2.ctypes.data, rows)

    # ---------------------------------------------------------- structure
    @property
    def outer_horizon_radius(self) -> float:
        return self.mass + math.sqrt(self.mass ** 2 - self.charge ** 2)

    @property
    def inner_horizon_radius(self) -> float:
        return self.mass - math.sqrt(self.mass ** 2 - self.charge ** 2)

    @property
    def inner_surface_gravity(self) -> float:
        """kappa_minus = (r_plus - r_minus) / (2 r_minus^2)."""
        return (self.outer_horizon_radius - self.inner_horizon_radius) / (
            2.0 * self.inner_horizon_radius ** 2)

    # ------------------------------------------------- host closed forms
    def ingoing_mass(self, v):
        """m1(v), the Price-tail-fed exterior mass (vaidya.py:153-159)."""
        v_safe = numpy.maximum(v, self.tail_start)
        return self.mass - self.tail_mass * (self.tail_start / v_safe) ** (self.tail_power - 1.0)

    def ingoing_mass_rate(self, v):
        """L(v) = dm1/dv, zero before the tail's onset (vaidya.py:161-171)."""
        rate = (self.tail_mass * (self.tail_power - 1.0)
                * self.tail_start ** (self.tail_power - 1.0)
                / numpy.maximum(v, self.tail_start) ** self.tail_power)
        return numpy.where(numpy.asarray(v) >= self.tail_start, rate, 0.0)

    def metric_function(self, v, radius):
        """f1 = 1 - 2 m1(v)/r + q^2/r^2 (vaidya.py:173-179)."""
        return 1.0 - 2.0 * self.ingoing_mass(v) / radius + self.charge ** 2 / radius ** 2

    def shell_radius(self, v):
        """R_s(v), held at the table's ends outside it (vaidya.py:239-242)."""
        return numpy.interp(v, self._shell_v, self._shell_r)

    def inflated_mass_increment(self, v):
        """m2(v) - m1(v) behind the shell (vaidya.py:244-258)."""
        m2 = numpy.interp(v, self._shell_v, self._shell_m2)
        inc = m2 - self.ingoing_mass(v)
        return numpy.where(numpy.asarray(v) < self.shell_start_v, 0.0,
                           numpy.clip(inc, 0.0, self.mass_cap))

    def kerr_schild_radius(self, x, y, z):
        """Areal radius; the surrogate is spherical (vaidya.py:280-283)."""
        if isinstance(x, torch.Tensor):
            return torch.sqrt(x * x + y * y + z * z)
        return numpy.sqrt(x * x + y * y + z * z)

    # ------------------------------------------------------------ device
    def _struct(self, dev, n_shell) -> "_lib.Vaidya":
        t = self._device_tables.get(dev) if dev is not None else None
        return _lib.Vaidya(self.mass, self.charge, self.tail_mass, self.tail_start,
                           self.tail_power, self.shell_energy, self.shell_start_v,
                           self.shell_start_radius, self.shell_width, self.mass_cap,
                           ptr(t[0]) if t else None, ptr(t[1]) if t else None,
                           ptr(t[2]) if t else None, n_shell)

    def device_struct(self, device) -> "_lib.Vaidya":
        """The C-ABI struct with the shell table copied to `device` (once)."""
        key = str(device)
        if key not in self._device_tables:
            self._device_tables[key] = tuple(
                torch.as_tensor(a, device=device).contiguous()
                for a in (self._shell_v, self._shell_r, self._shell_m2))
        return self._struct(key, int(self._shell_v.size))

    def mass_function(self, v, radius):
        """m(v, r) (vaidya.py:260-269), on the device."""
        return self._masses(v, radius)[0]

    def misner_sharp_mass(self, v, radius):
        """m(v, r) - q^2/(2 r) (vaidya.py:271-278), on the device."""
        return self._masses(v, radius)[1]

    def _masses(self, v, radius):
        vv, host = to_device_f64(numpy.atleast_1d(v) if not isinstance(v, torch.Tensor) else v,
                                 "v")
        rr, _ = to_device_f64(numpy.atleast_1d(radius) if not isinstance(radius, torch.Tensor)
                              else radius, "radius")
        vv, rr = torch.broadcast_tensors(vv, rr)
        vv, rr = vv.contiguous(), rr.contiguous()
        n = vv.numel()
        m = torch.empty(n, dtype=torch.float64, device=vv.device)
        ms = torch.empty(n, dtype=torch.float64, device=vv.device)
        _lib.check(_lib.load().bh_vaidya_mass(self.device_struct(vv.device), ptr(vv), ptr(rr), n,
                                              ptr(m), ptr(ms), stream_handle()), "mass_function")
        if host is not None:
            return m.cpu().numpy(), ms.cpu().numpy()
        return m, ms

    def geometry_t(self, t, x, y, z) -> VaidyaGeometry:
        """H, l, dH/dx_i = h_spatial_scale l_i, dH/dt and r at (t, x, y, z)
        (vaidya.py:285-325), on the device."""
        ts, host = to_device_f64(t, "t")
        xs, _ = to_device_f64(x, "x")
        ys, _ = to_device_f64(y, "y")
        zs, _ = to_device_f64(z, "z")
        n = xs.shape[0]
        dev = xs.device
        out = [torch.empty(n, dtype=torch.float64, device=dev) for _ in range(4)]
        l = torch.empty((n, 3), dtype=torch.float64, device=dev)
        _lib.check(_lib.load().bh_vaidya_geometry(
            self.device_struct(dev), ptr(ts), ptr(xs), ptr(ys), ptr(zs), n, ptr(out[0]), ptr(l),
            ptr(out[1]), ptr(out[2]), ptr(out[3]), stream_handle()), "geometry_t")
        conv = (lambda a: a.cpu().numpy()) if host is not None else (lambda a: a)  # noqa: E731
        return VaidyaGeometry(h=conv(out[0]), l=conv(l), h_spatial_scale=conv(out[1]),
                              h_t=conv(out[2]), radius=conv(out[3]))

    def frozen(self, time: float) -> "FrozenVaidyaSlice":
        """The constant-time view used by the tetrad machinery."""
        return FrozenVaidyaSlice(self, float(time))


class FrozenVaidyaSlice:
    """Stationary-style geometry(x, y, z) view at a fixed time (vaidya.py:334-353)."""

    def __init__(self, spacetime: ChargedVaidyaSpacetime, time: float) -> None:
        self.spacetime = spacetime
        self.time = time
        self.inner_horizon_radius = spacetime.inner_horizon_radius
        self.outer_horizon_radius = spacetime.outer_horizon_radius

    def kerr_schild_radius(self, x, y, z):
        return self.spacetime.kerr_schild_radius(x, y, z)

    def geometry(self, x, y, z) -> VaidyaGeometry:
        t = numpy.full(numpy.shape(x), self.time) if not isinstance(x, torch.Tensor) else \
            torch.full_like(x, self.time, dtype=torch.float64)
        return self.spacetime.geometry_t(t, x, y, z)


def vaidya_geodesic_rhs(spacetime: ChargedVaidyaSpacetime, states: Array) -> Array:
    """The extended Hamiltonian flow of the time-dependent surrogate
    (vaidya.py:356-394), on the device."""
    s, host = to_device_f64(states, "states")
    out = torch.empty_like(s)
    _lib.check(_lib.load().bh_vaidya_rhs(spacetime.device_struct(s.device), ptr(s), ptr(out),
                                         s.shape[0], stream_handle()), "vaidya_geodesic_rhs")
    return out.cpu().numpy() if host is not None else out


def vaidya_rk4(spacetime: ChargedVaidyaSpacetime, states: Array, h, n_steps: int = 1) -> Array:
    """n_steps of rk4_step (integrators.py:57-73) with the surrogate's RHS."""
    s, host = to_device_f64(states, "states")
    n = s.shape[0]
    hs = torch.as_tensor(numpy.broadcast_to(numpy.asarray(h, dtype=float), (n,)).copy()
                         if not isinstance(h, torch.Tensor) else h,
                         dtype=torch.float64, device=s.device).contiguous()
    out = torch.empty_like(s)
    _lib.check(_lib.load().bh_vaidya_rk4(spacetime.device_struct(s.device), ptr(s), ptr(hs),
                                         ptr(out), n, int(n_steps), stream_handle()),
               "vaidya_rk4")
    return out.cpu().numpy() if host is not None else out


def trace_vaidya_tile(spacetime: ChargedVaidyaSpacetime, state0: Array, escape_radius: float,
                      stop_radius: float, max_steps: int = 900):
    """Past-directed rays through the surrogate (offline/inflation.py:165-240):
    (status 0 escaped / 1 terminal surface / 2 budget, escape directions
    (n, 3), Misner-Sharp mass at the terminal point, v = t + r at the end)."""
    s, host = to_device_f64(state0, "state0")
    n = s.shape[0]
    dev = s.device
    lib = _lib.load()
    states = torch.empty_like(s)
    status = torch.empty(n, dtype=torch.int32, device=dev)
    edir = torch.empty((n, 3), dtype=torch.float64, device=dev)
    mass = torch.empty(n, dtype=torch.float64, device=dev)
    v_end = torch.empty(n, dtype=torch.float64, device=dev)
    ws = torch.empty(lib.bh_trace_workspace_bytes(), dtype=torch.uint8, device=dev)
    _lib.check(lib.bh_vaidya_trace(spacetime.device_struct(dev), ptr(s), n, float(escape_radius),
                                   float(stop_radius), int(max_steps), ptr(states), ptr(status),
                                   ptr(edir), ptr(mass), ptr(v_end), ptr(ws), stream_handle()),
               "trace_vaidya_tile")
    out = (status, edir, mass, v_end)
    if host is not None:
        return tuple(a.cpu().numpy() for a in out)
    return out


def rain_state(spacetime: ChargedVaidyaSpacetime, position, time: float) -> numpy.ndarray:
    """Ingoing free-fall camera state (1, 8) on the frozen slice: covariant
    p = (-1, w l), w = -sqrt(2H) / (1 + sqrt(2H)) (offline/inflation.py:39-63)."""
    pos = numpy.asarray(position, dtype=float)
    geo = spacetime.frozen(time).geometry(pos[None, 0], pos[None, 1], pos[None, 2])
    root = math.sqrt(max(2.0 * float(geo.h[0]), 0.0))
    w = -root / (1.0 + root)
    state = numpy.empty((1, 8))
    state[0, 0] = time
    state[0, 1:4] = pos
    state[0, 4:8] = [-1.0, w * geo.l[0, 0], w * geo.l[0, 1], w * geo.l[0, 2]]
    return state


def camera_four_velocity(spacetime: ChargedVaidyaSpacetime, state) -> numpy.ndarray:
    """Contravariant camera 4-velocity from a covariant state
    (offline/inflation.py:66-74)."""
    from .frames import raise_index

    s = numpy.asarray(state, dtype=float)
    return raise_index(spacetime.frozen(float(s[0, 0])), s[:, 1:4], s[:, 4:8])[0]


# ------------------------------------------------------ mass-inflation frame


def _layer_tetrad(spacetime: ChargedVaidyaSpacetime, state: numpy.ndarray, look: str):
    """The camera tetrad of a flythrough frame on the frozen slice
    (offline/inflation.py:252-289): the worldline's 4-velocity, or the rain
    observer where the worldline sample has diverged; forward along the
    outward radial direction, its opposite, or sideways."""
    from .frames import build_tetrad, raise_index

    position = state[1:4]
    slice_geo = spacetime.frozen(float(state[0]))
    outward = position / max(numpy.linalg.norm(position), 1e-12)
    up_seed = numpy.array([0.0, 0.0, 1.0])
    if abs(float(numpy.dot(outward, up_seed))) > 0.98:
        up_seed = numpy.array([0.0, 1.0, 0.0])
    if look == "inward":
        forward = -outward
    elif look == "side":
        forward = numpy.cross(up_seed, outward)
        forward = forward / max(numpy.linalg.norm(forward), 1e-12)
    else:
        forward = outward
    try:
        velocity = camera_four_velocity(spacetime, state[None, :])
        if not numpy.isfinite(velocity).all() or float(numpy.linalg.norm(velocity)) > 1e4:
            raise ValueError("diverged worldline sample")
        return slice_geo, build_tetrad(slice_geo, position, velocity, forward, up_seed)
    except ValueError:
        geo = slice_geo.geometry(position[None, 0], position[None, 1], position[None, 2])
        h = float(numpy.asarray(geo.h)[0])
        l = numpy.asarray(geo.l)[0]
        root = math.sqrt(max(2.0 * h, 0.0))
        w = -root / (1.0 + root)
        rain = raise_index(slice_geo, position[None, :],
                           numpy.array([[-1.0, w * l[0], w * l[1], w * l[2]]]))[0]
        return slice_geo, build_tetrad(slice_geo, position, rain, forward, up_seed)


def layer_frame_states(spacetime: ChargedVaidyaSpacetime, state, width: int, height: int,
                       fov_degrees: float, supersample: int, look: str = "outward"):
    """(width height supersample^2, 8) tetrad rays of a flythrough frame
    (offline/inflation.py:291-318): the supersampled pinhole grid in the
    camera's frame, momenta -g(e0 - n.e) lowered on the frozen slice, t the
    worldline's time.  Host NumPy for the grid, slice geometry from the
    device."""
    from .frames import lower_index

    state = numpy.asarray(state, dtype=float)
    slice_geo, tetrad = _layer_tetrad(spacetime, state, look)
    tan_half = math.tan(math.radians(fov_degrees) / 2.0)
    ss = supersample
    ray = numpy.arange(width * height * ss * ss)
    pixel, sub = numpy.divmod(ray, ss * ss)
    row, col = numpy.divmod(pixel, width)
    sub_row, sub_col = numpy.divmod(sub, ss)
    u = (col + (sub_col + 0.5) / ss) / width * 2.0 - 1.0
    v = 1.0 - (row + (sub_row + 0.5) / ss) / height * 2.0
    right = u * tan_half
    up = v * tan_half / (width / height)
    norm = numpy.sqrt(1.0 + right * right + up * up)
    local = numpy.stack([1.0 / norm, right / norm, up / norm], axis=-1)
    spatial = sum(local[:, k:k + 1] * tetrad[k + 1] for k in range(3))
    physical = tetrad[0][None, :] - spatial
    positions = numpy.tile(state[1:4][None, :], (local.shape[0], 1))
    momenta = numpy.asarray(lower_index(slice_geo, positions, -physical))
    out = numpy.empty((local.shape[0], 8))
    out[:, 0] = state[0]
    out[:, 1:4] = positions
    out[:, 4:8] = momenta
    return out


def render_layer_frame_device(spacetime: ChargedVaidyaSpacetime, state, width: int,
                              height: int, settings, look: str = "outward", *,
                              return_rays: bool = False):
    """One frame of the mass-inflation flythrough as a float32 (height,
    width, 3) device tensor (offline/inflation.py:243-346): tetrad rays from
    the worldline state, traced through the surrogate to max(12, 2.5 r) or
    the terminal surface at 1.001 r_minus (``trace_vaidya_tile``), then
    shaded and averaged on the device (``bh_inflation_radiance``).
    ``settings`` supplies fov_degrees and supersample (OfflineSettings)."""
    state = numpy.asarray(state, dtype=float)
    ss = int(settings.supersample)
    s0 = layer_frame_states(spacetime, state, width, height, settings.fov_degrees, ss, look)
    dev = torch.device("cuda", torch.cuda.current_device())
    escape_radius = max(12.0, 2.5 * float(numpy.linalg.norm(state[1:4])))
    status, edir, mass, v_end = trace_vaidya_tile(
        spacetime, torch.as_tensor(s0, device=dev), escape_radius,
        spacetime.inner_horizon_radius * 1.001)
    hdr = torch.empty((height, width, 3), dtype=torch.float32, device=dev)
    _lib.check(_lib.load().bh_inflation_radiance(
        float(spacetime.mass), ptr(status), ptr(edir.contiguous()), ptr(mass.contiguous()),
        width, height, ss, ptr(hdr), stream_handle()), "inflation radiance")
    if return_rays:
        return hdr, {"state0": s0, "status": status, "escape_directions": edir,
                     "end_mass": mass, "v_end": v_end}
    return hdr


def render_layer_frame(spacetime: ChargedVaidyaSpacetime, state, width: int, height: int,
                       settings, look: str = "outward") -> numpy.ndarray:
    """render_layer_frame (offline/inflation.py:243-346): the frame as a
    (height, width, 3) float32 NumPy array."""
    return render_layer_frame_device(spacetime, state, width, height, settings,
                                     look).cpu().numpy()


def build_worldline(spacetime: ChargedVaidyaSpacetime, start_radius: float, start_time: float,
                    stop_radius: float, step: float = 2e-3, mass_threshold: float = 1e4):
    """(taus (k,), states (k, 8)): the flythrough camera's worldline
    (offline/inflation.py:77-135), a rain observer from (start_radius, 0, 0)
    at start_time, RK4 in proper time with the step min(step, max(0.05 (r -
    r_minus floored at 5e-3), 2e-3)), sampled every 8 steps and at the end,
    stopped at r <= stop_radius, where the Misner-Sharp mass reaches
    mass_threshold, on a non-finite state or after 120000 steps.  The steps
    run on the device (``vaidya_rk4``, ``misner_sharp_mass``), the loop on
    the host: the worldline is one sequential trajectory."""
    state = rain_state(spacetime, numpy.array([float(start_radius), 0.0, 0.0]),
                       float(start_time))
    r_minus = spacetime.inner_horizon_radius
    tau = 0.0
    taus = [0.0]
    states = [state[0].copy()]
    for iteration in range(120000):
        radius = float(numpy.sqrt(numpy.sum(state[0, 1:4] ** 2)))
        proximity = max(radius - r_minus, 5e-3)
        step_now = float(min(step, max(0.05 * proximity, 2e-3)))
        state = vaidya_rk4(spacetime, state, numpy.array([step_now]), 1)
        if not numpy.isfinite(state).all():
            break
        tau += step_now
        radius = float(numpy.sqrt(numpy.sum(state[0, 1:4] ** 2)))
        v_here = float(state[0, 0]) + radius
        mass_here = float(numpy.asarray(spacetime.misner_sharp_mass(
            numpy.array([v_here]), numpy.array([radius])))[0])
        reached = radius <= stop_radius or mass_here >= mass_threshold
        if iteration % 8 == 0 or reached:
            taus.append(tau)
            states.append(state[0].copy())
        if reached:
            break
    return numpy.asarray(taus), numpy.stack(states)
