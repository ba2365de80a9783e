"""ctypes front end of the CPU oracle (``oracle/bh_oracle.c``).

TEST INFRASTRUCTURE ONLY.  The parity tests, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py`` check the CUDA library's results against
this oracle; the product package ``blackhorizon_b200`` never imports it.

Each wrapper names the reference function (MegaKruk/BlackHorizon, path within
that project) whose behaviour the C restatement follows.
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libbh_oracle.so")
_lib = None

_D = ctypes.c_double
_I64 = ctypes.c_int64
_P = ctypes.c_void_p


class TraceParams(ctypes.Structure):
    """Keyword arguments of blackhorizon/tracer.py:50-61 plus mass and spin."""

    _fields_ = [
        ("mass", _D), ("spin", _D), ("escape_radius", _D), ("max_steps", _I64),
        ("rtol", _D), ("atol", _D), ("initial_step", _D), ("max_step", _D),
        ("min_step", _D), ("capture_margin", _D),
    ]


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (gcc, no FMA contraction)."""
    src = os.path.join(_HERE, "bh_oracle.c")
    if force or not os.path.exists(_LIB_PATH) or (
        os.path.getmtime(_LIB_PATH) < os.path.getmtime(src)
    ):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = ctypes.CDLL(_LIB_PATH)
        _lib.bho_trace_batch.restype = _I64
        _lib.bho_error_ratio.restype = _D
        _lib.bho_step_factor.restype = _D
        _lib.bho_hamiltonian.restype = _D
        _lib.bho_step_factor.argtypes = [_D]
        _lib.bho_num_threads.restype = ctypes.c_int
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_P)


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def num_threads() -> int:
    return int(lib().bho_num_threads())


def geometry(mass: float, spin: float, xyz):
    """kerr.py:118-193 with gradients: returns r, h, l, grad_h, grad_l."""
    xyz = _f64(xyz)
    n = xyz.shape[0]
    r = np.empty(n); h = np.empty(n)
    l = np.empty((n, 3)); gh = np.empty((n, 3)); gl = np.empty((n, 3, 3))
    lib().bho_geometry_batch(_D(mass), _D(spin), _ptr(xyz), _I64(n), _ptr(r),
                             _ptr(h), _ptr(l), _ptr(gh), _ptr(gl))
    return r, h, l, gh, gl


def rhs(mass: float, spin: float, states):
    """geodesics.py:42-74."""
    s = _f64(states)
    out = np.empty_like(s)
    lib().bho_rhs_batch(_D(mass), _D(spin), _ptr(s), _I64(s.shape[0]), _ptr(out))
    return out


def hamiltonian(mass: float, spin: float, states):
    """geodesics.py:77-85."""
    s = _f64(states)
    out = np.empty(s.shape[0])
    f = lib().bho_hamiltonian
    f.argtypes = [_D, _D, _P]
    for i in range(s.shape[0]):
        out[i] = f(mass, spin, s[i].ctypes.data_as(_P))
    return out


def coordinate_velocity(mass: float, spin: float, states):
    """geodesics.py:95-106."""
    s = _f64(states)
    out = np.empty((s.shape[0], 4))
    f = lib().bho_coordinate_velocity
    for i in range(s.shape[0]):
        f(_D(mass), _D(spin), s[i].ctypes.data_as(_P), out[i].ctypes.data_as(_P))
    return out


def null_momentum(mass: float, spin: float, positions, directions,
                  past: bool = True, normalize: bool = True):
    """geodesics.py:109-170."""
    pos = _f64(positions); d = _f64(directions)
    out = np.empty((pos.shape[0], 4))
    lib().bho_null_momentum_batch(_D(mass), _D(spin), _ptr(pos), _ptr(d),
                                  _I64(pos.shape[0]), ctypes.c_int(int(past)),
                                  ctypes.c_int(int(normalize)), _ptr(out))
    return out


def dp5_step(mass: float, spin: float, states, h, rtol: float = 1e-9,
             atol: float = 1e-12):
    """integrators.py:76-117: returns (new_state, error, error_ratio)."""
    s = _f64(states)
    hh = _f64(np.broadcast_to(np.asarray(h, dtype=np.float64), (s.shape[0],)))
    y_new = np.empty_like(s); err = np.empty_like(s); ratio = np.empty(s.shape[0])
    lib().bho_dp5_batch(_D(mass), _D(spin), _ptr(s), _ptr(hh), _I64(s.shape[0]),
                        _ptr(y_new), _ptr(err), _ptr(ratio), _D(rtol), _D(atol))
    return y_new, err, ratio


def step_factor(ratio):
    """integrators.py:120-124."""
    f = lib().bho_step_factor
    return np.array([f(float(r)) for r in np.ravel(ratio)])


def rk4(mass: float, spin: float, states, h: float, n_steps: int,
        nthreads: int = 0):
    """n_steps of integrators.py:57-73 per ray."""
    s = _f64(states).copy()
    lib().bho_rk4_batch(_D(mass), _D(spin), _ptr(s), _I64(s.shape[0]),
                        _I64(n_steps), _D(h), ctypes.c_int(nthreads))
    return s


def pinhole_directions(forward, right, up, fov_degrees: float, width: int,
                       height: int):
    """camera.py:96-113 given the camera basis."""
    out = np.empty((height * width, 3))
    f = _f64(forward); r = _f64(right); u = _f64(up)
    lib().bho_pinhole_directions(_ptr(f), _ptr(r), _ptr(u), _D(fov_degrees),
                                 _I64(width), _I64(height), _ptr(out))
    return out


def trace(mass: float, spin: float, state0, escape_radius: float,
          max_steps: int = 20000, rtol: float = 1e-9, atol: float = 1e-12,
          initial_step: float = 0.1, max_step: float = 2.0,
          min_step: float = 1e-10, capture_margin: float = 1e-3,
          nthreads: int = 0):
    """tracer.py:50-157: returns (states, status, steps, iterations)."""
    s = _f64(state0).copy()
    n = s.shape[0]
    status = np.empty(n, dtype=np.int32)
    steps = np.empty(n, dtype=np.int64)
    p = TraceParams(mass, spin, escape_radius, max_steps, rtol, atol,
                    initial_step, max_step, min_step, capture_margin)
    it = lib().bho_trace_batch(ctypes.byref(p), _ptr(s), _ptr(status),
                               _ptr(steps), _I64(n), ctypes.c_int(nthreads))
    if it < 0:
        raise ValueError("escape_radius must exceed all initial radii")
    return s, status, steps, int(it)


def propagate(mass: float, spins, state0, n_steps: int, rtol: float,
              atol: float, initial_step: float = 0.1, max_step: float = 2.0,
              nthreads: int = 0):
    """n_steps attempted DP5(4) steps per ray with the tracer's accept/reject
    and step update (tracer.py:111-120) and no termination; spins is a scalar
    or a per-ray array.  Returns (states, h, accepted)."""
    s = _f64(state0).copy()
    n = s.shape[0]
    h = np.full(n, float(initial_step))
    acc = np.empty(n, dtype=np.int64)
    spins_arr = None
    spin = 0.0
    if np.ndim(spins) == 0:
        spin = float(spins)
    else:
        spins_arr = _f64(spins)
    lib().bho_propagate_batch(_D(mass), _D(spin),
                              _ptr(spins_arr) if spins_arr is not None else None,
                              _ptr(s), _ptr(h), _ptr(acc), _I64(n), _I64(n_steps),
                              _D(rtol), _D(atol), _D(max_step),
                              ctypes.c_int(nthreads))
    return s, h, acc


def propagate_to(mass: float, spins, state0, lam_target, rtol: float = 1e-12,
                 atol: float = 1e-14, initial_step: float = 0.1,
                 max_step: float = 2.0, max_attempts: int = 1_000_000,
                 nthreads: int = 0):
    """States at affine parameter lam_target (per ray), integrated with the
    reference's DP5(4) and controller and the last step cut to land on the
    target (integrators.py:127-174 per ray).  Returns (states, attempts)."""
    s = _f64(state0).copy()
    n = s.shape[0]
    lam = _f64(np.broadcast_to(np.asarray(lam_target, dtype=np.float64), (n,)))
    att = np.empty(n, dtype=np.int64)
    spins_arr = None
    spin = 0.0
    if np.ndim(spins) == 0:
        spin = float(spins)
    else:
        spins_arr = _f64(spins)
    lib().bho_propagate_to(_D(mass), _D(spin),
                           _ptr(spins_arr) if spins_arr is not None else None,
                           _ptr(s), _ptr(lam), _ptr(att), _I64(n), _D(rtol), _D(atol),
                           _D(initial_step), _D(max_step), _I64(max_attempts),
                           ctypes.c_int(nthreads))
    return s, att


def trace_tile(mass: float, spin: float, state0, escape_radius: float,
               disk_radii=None, rtol: float = 1e-9, max_steps: int = 12000,
               max_step: float = 2.0, capture_margin: float = 1e-3, nthreads: int = 0,
               interior_stop: float | None = None):
    """offline/render.py:184-349 (_trace_tile with _refine_crossings);
    ``interior_stop`` selects the interior-camera termination of
    render.py:203-248.  Returns a dict of per-ray arrays."""
    s = _f64(state0).copy()
    n = s.shape[0]
    out = {"status": np.empty(n, dtype=np.int32), "steps": np.empty(n, dtype=np.int64),
           "hit_positions": np.empty((n, 3)), "hit_momenta": np.empty((n, 3)),
           "escape_directions": np.empty((n, 3)), "saturated": np.empty(n, dtype=np.int32)}
    p = TraceParams(mass, spin, escape_radius, max_steps, rtol, rtol * 1e-3, 0.1, max_step,
                    0.0, capture_margin)
    r_in, r_out = (0.0, 0.0) if disk_radii is None else disk_radii
    stop = 0.0 if interior_stop is None else float(interior_stop)
    if interior_stop is not None and not stop > 0.0:
        raise ValueError("interior_stop must be > 0")
    lib().bho_trace_tile(ctypes.byref(p), _D(r_in), _D(r_out), _D(stop), _ptr(s),
                         _ptr(out["status"]),
                         _ptr(out["steps"]), _ptr(out["hit_positions"]),
                         _ptr(out["hit_momenta"]), _ptr(out["escape_directions"]),
                         _ptr(out["saturated"]), _I64(n), ctypes.c_int(nthreads))
    out["states"] = s
    return out


def celestial_checkerboard(directions, cells: int = 12):
    """imaging.py:27-50."""
    d = _f64(directions)
    out = np.empty((d.shape[0], 3), dtype=np.uint8)
    lib().bho_celestial_checkerboard(_ptr(d), _I64(d.shape[0]), ctypes.c_int(cells), _ptr(out))
    return out


def render_image(mass: float, spin: float, states, status, width: int, height: int,
                 cells: int = 12):
    """imaging.py:53-91: (height, width, 3) uint8."""
    s = _f64(states)
    st = np.ascontiguousarray(status, dtype=np.int32)
    n = width * height
    if s.shape[0] != n or st.shape[0] != n:
        raise ValueError("result size does not match image dimensions")
    out = np.empty((n, 3), dtype=np.uint8)
    lib().bho_render_image(_D(mass), _D(spin), _ptr(s), _ptr(st), _I64(n), ctypes.c_int(cells),
                           _ptr(out))
    return out.reshape(height, width, 3)


class RealtimeParams(ctypes.Structure):
    """bho_realtime_params_t: realtime/settings.py controls of one trace."""
    _fields_ = [("mass", _D), ("spin", _D), ("escape_radius", _D), ("max_steps", _I64),
                ("step_scale", _D), ("min_step", _D), ("max_step", _D),
                ("capture_margin", _D), ("momentum_bailout", _D), ("disk_inner", _D),
                ("disk_outer", _D), ("interior_stop", _D)]


def trace_realtime(mass: float, spin: float, state0, escape_radius: float, max_steps: int,
                   step_scale: float, min_step: float = 1e-4, max_step: float = 4.0,
                   capture_margin: float = 2e-2, momentum_bailout: float = 1e3,
                   disk_radii=None, interior_stop=None, nthreads: int = 0):
    """realtime/reference.py:41-188 (trace_like_shader)."""
    s = _f64(state0).copy()
    n = s.shape[0]
    r_in, r_out = (0.0, 0.0) if disk_radii is None else disk_radii
    p = RealtimeParams(mass, spin, escape_radius, max_steps, step_scale, min_step, max_step,
                       capture_margin, momentum_bailout, r_in, r_out,
                       0.0 if interior_stop is None else interior_stop)
    out = {"status": np.empty(n, dtype=np.int32), "hit_radii": np.empty(n),
           "hit_positions": np.empty((n, 3)), "hit_momenta": np.empty((n, 4))}
    lib().bho_trace_realtime(ctypes.byref(p), _ptr(s), _ptr(out["status"]),
                             _ptr(out["hit_radii"]), _ptr(out["hit_positions"]),
                             _ptr(out["hit_momenta"]), _I64(n), ctypes.c_int(nthreads))
    out["states"] = s
    out["positions"] = s[:, 1:4].copy()
    out["momenta"] = s[:, 4:8].copy()
    return out


class VaidyaParams(ctypes.Structure):
    """bho_vaidya_t: ChargedVaidyaSpacetime fields and its shell table."""
    _fields_ = [("mass", _D), ("charge", _D), ("tail_mass", _D), ("tail_start", _D),
                ("tail_power", _D), ("shell_energy", _D), ("shell_start_v", _D),
                ("shell_start_radius", _D), ("shell_width", _D), ("mass_cap", _D),
                ("shell_v", _P), ("shell_r", _P), ("shell_m2", _P), ("n_shell", _I64)]


class Vaidya:
    """The charged-Vaidya/Ori surrogate (vaidya.py:87-330) with its shell
    table integrated by the C restatement."""

    def __init__(self, mass=1.0, charge=0.9, tail_mass=0.01, tail_start=12.0, tail_power=12.0,
                 shell_energy=1e-3, shell_start_v=14.0, shell_start_radius=1.0,
                 shell_width=0.02, mass_cap=1e7):
        self.p = VaidyaParams(mass, charge, tail_mass, tail_start, tail_power, shell_energy,
                              shell_start_v, shell_start_radius, shell_width, mass_cap,
                              None, None, None, 0)
        cap = 4000002
        v, r, m2 = np.empty(cap), np.empty(cap), np.empty(cap)
        k = lib().bho_vaidya_shell(ctypes.byref(self.p), _ptr(v), _ptr(r), _ptr(m2), _I64(cap))
        self.shell_v, self.shell_r, self.shell_m2 = v[:k].copy(), r[:k].copy(), m2[:k].copy()
        self.p.shell_v, self.p.shell_r = _ptr(self.shell_v), _ptr(self.shell_r)
        self.p.shell_m2, self.p.n_shell = _ptr(self.shell_m2), k

    def geometry_t(self, states):
        s = _f64(states)
        n = s.shape[0]
        out = {k: np.empty(n) for k in ("h", "hs", "ht", "radius")}
        out["l"] = np.empty((n, 3))
        f = lib().bho_vaidya_geometry
        for i in range(n):
            h, hs, ht, r = _D(), _D(), _D(), _D()
            l3 = (_D * 3)()
            f(ctypes.byref(self.p), _D(s[i, 0]), _D(s[i, 1]), _D(s[i, 2]), _D(s[i, 3]),
              ctypes.byref(h), l3, ctypes.byref(hs), ctypes.byref(ht), ctypes.byref(r))
            out["h"][i], out["hs"][i], out["ht"][i], out["radius"][i] = h.value, hs.value, \
                ht.value, r.value
            out["l"][i] = list(l3)
        return out

    def mass(self, v, r):
        f = lib().bho_vaidya_mass
        f.restype = _D
        g = lib().bho_vaidya_misner_sharp
        g.restype = _D
        m = np.array([f(ctypes.byref(self.p), _D(a), _D(b)) for a, b in zip(v, r)])
        ms = np.array([g(ctypes.byref(self.p), _D(a), _D(b)) for a, b in zip(v, r)])
        return m, ms

    def rhs(self, states):
        s = _f64(states)
        out = np.empty_like(s)
        for i in range(s.shape[0]):
            lib().bho_vaidya_rhs(ctypes.byref(self.p), s[i].ctypes.data_as(_P),
                                 out[i].ctypes.data_as(_P))
        return out

    def rk4(self, states, n_steps, h):
        s = _f64(states).copy()
        lib().bho_vaidya_rk4(ctypes.byref(self.p), _ptr(s), _I64(s.shape[0]), _I64(n_steps),
                             _D(h))
        return s

    def trace(self, state0, escape_radius, stop_radius, max_steps=900, nthreads=0):
        """offline/inflation.py:165-240: (status, escape_dir, end_mass, v_end)."""
        s = _f64(state0).copy()
        n = s.shape[0]
        status = np.empty(n, dtype=np.int32)
        edir, mass, v_end = np.empty((n, 3)), np.empty(n), np.empty(n)
        lib().bho_vaidya_trace(ctypes.byref(self.p), _ptr(s), _I64(n), _D(escape_radius),
                               _D(stop_radius), _I64(max_steps), _ptr(status), _ptr(edir),
                               _ptr(mass), _ptr(v_end), ctypes.c_int(nthreads))
        return status, edir, mass, v_end


class EmissionParams(ctypes.Structure):
    _fields_ = [("mass", _D), ("spin", _D), ("disk_inner", _D), ("disk_temperature", _D),
                ("disk_detail", _D), ("observer_lapse", _D), ("bb_log_min", _D),
                ("bb_log_max", _D), ("sheet_rgb", _D * 3), ("temperature_size", ctypes.c_int32),
                ("blackbody_size", ctypes.c_int32), ("supersample", ctypes.c_int32)]


def emission_params(mass, spin, tables, disk_temperature=6500.0, disk_detail=1.0,
                    observer_lapse=1.0, sheet_rgb=(0.0, 0.0, 0.0), supersample=1):
    """``tables``: dict with temperature (float32), radii, blackbody (float32
    (B, 3)), bb_log_min, bb_log_max, disk_inner (numpy arrays)."""
    return EmissionParams(float(mass), float(spin), float(tables["disk_inner"]),
                          float(disk_temperature), float(disk_detail), float(observer_lapse),
                          float(tables["bb_log_min"]), float(tables["bb_log_max"]),
                          (_D * 3)(*(float(v) for v in sheet_rgb)),
                          int(tables["temperature"].size), int(tables["blackbody"].shape[0]),
                          int(supersample))


def starfield(directions, shift=None):
    """offline/render.py:352-419 (_starfield_hdr): (n, 3) float64."""
    d = _f64(directions)
    s = None if shift is None else _f64(shift)
    out = np.empty((d.shape[0], 3))
    lib().bho_starfield(_ptr(d), _ptr(s) if s is not None else None, _I64(d.shape[0]),
                        _ptr(out))
    return out


def disk_radiance(params: EmissionParams, positions, momenta, tables):
    """offline/render.py:422-484 (_disk_radiance): (n, 3) float64."""
    pos, mom = _f64(positions), _f64(momenta)
    t = np.ascontiguousarray(tables["temperature"], dtype=np.float32)
    r = _f64(tables["radii"])
    bb = np.ascontiguousarray(tables["blackbody"], dtype=np.float32)
    out = np.empty((pos.shape[0], 3))
    lib().bho_disk_radiance(ctypes.byref(params), _ptr(pos), _ptr(mom), _I64(pos.shape[0]),
                            _ptr(t), _ptr(r), _ptr(bb), _ptr(out))
    return out


def offline_radiance(params: EmissionParams, status, escape_dir, hit_pos, hit_mom, tables,
                     width: int, height: int, energy=None, nthreads: int = 0):
    """The shading of render_hdr (render.py:630-680): (height, width, 3)
    float32, supersample^2 consecutive rays per pixel."""
    st = np.ascontiguousarray(status, dtype=np.int32)
    ed, hp, hm = _f64(escape_dir), _f64(hit_pos), _f64(hit_mom)
    e = None if energy is None else _f64(energy)
    t = np.ascontiguousarray(tables["temperature"], dtype=np.float32)
    r = _f64(tables["radii"])
    bb = np.ascontiguousarray(tables["blackbody"], dtype=np.float32)
    out = np.empty((height, width, 3), dtype=np.float32)
    lib().bho_offline_radiance(ctypes.byref(params), _ptr(st), _ptr(ed), _ptr(hp), _ptr(hm),
                               _ptr(e) if e is not None else None, _I64(width * height),
                               _ptr(t), _ptr(r), _ptr(bb), _ptr(out), ctypes.c_int(nthreads))
    return out


def develop(hdr, weights, exposure=1.0, bloom_threshold=1.0, bloom_strength=0.35):
    """offline/post.py:88-106 (develop); weights = gaussian_kernel(sigma)."""
    img = np.ascontiguousarray(hdr, dtype=np.float32)
    w = _f64(weights)
    out = np.empty(img.shape, dtype=np.uint8)
    lib().bho_develop(_ptr(img), _I64(img.shape[1]), _I64(img.shape[0]), _D(exposure),
                      _D(bloom_threshold), _D(bloom_strength), _ptr(w),
                      ctypes.c_int(w.size // 2), _ptr(out))
    return out


class RealtimeShading(ctypes.Structure):
    _fields_ = [(k, ctypes.c_float) for k in (
        "mass", "spin", "disk_inner", "disk_outer", "disk_temperature", "disk_detail",
        "exposure", "observer_lapse", "bb_log_min", "bb_log_max", "sky_amplification",
        "sheet_radiance", "whiteout")] + [(k, ctypes.c_int32) for k in (
            "background", "temperature_size", "blackbody_size")]


def realtime_shade(params: RealtimeShading, status, states, hit_pos, hit_mom, temperature,
                   blackbody):
    """realtime/shaders/kerr_tracer.frag:205-420: (n, 3) uint8."""
    st = np.ascontiguousarray(status, dtype=np.int32)
    s, hp, hm = _f64(states), _f64(hit_pos), _f64(hit_mom)
    t = np.ascontiguousarray(temperature, dtype=np.float32)
    bb = np.ascontiguousarray(blackbody, dtype=np.float32)
    out = np.empty((st.size, 3), dtype=np.uint8)
    lib().bho_realtime_shade(ctypes.byref(params), _ptr(st), _ptr(s), _ptr(hp), _ptr(hm),
                             _I64(st.size), _ptr(t), _ptr(bb), _ptr(out))
    return out


def inflation_radiance(mass: float, status, escape_dir, end_mass, width: int, height: int,
                       supersample: int = 1):
    """offline/inflation.py:138-162, 322-346: (height, width, 3) float32."""
    st = np.ascontiguousarray(status, dtype=np.int32)
    ed, em = _f64(escape_dir), _f64(end_mass)
    out = np.empty((height, width, 3), dtype=np.float32)
    lib().bho_inflation_radiance(_D(mass), _ptr(st), _ptr(ed), _ptr(em),
                                 _I64(width * height), ctypes.c_int(supersample), _ptr(out))
    return out
