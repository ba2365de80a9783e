"""The charged-Vaidya/Ori surrogate on the GPU (vaidya.py, offline/inflation.py).

Parity with the reference's outputs (tests/golden/vaidya.npz): shell tables,
geometry_t, the mass functions and the time-dependent RHS at 2001 points,
3000-step RK4 trajectories and two flythrough camera tiles traced by the
mass-inflation renderer's loop.  The reference's m2 column carries NumPy's
vectorised power, which differs from libm's pow in the last ulp on ~5 % of
inputs and is amplified by the exponential inflation to <= 6e-10 relative;
the bounds are therefore 1e-9 relative (1e-8 after thousands of steps).
Then the reference's own physics anchors (tests/test_vaidya.py).
"""

import numpy as np
import pytest
import torch

from conftest import golden

pytestmark = pytest.mark.gpu

FIELDS = ("mass", "charge", "tail_mass", "tail_start", "tail_power", "shell_energy",
          "shell_start_v", "shell_start_radius", "shell_width", "mass_cap")


def _rel(a, b):
    a = a.cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)
    return float((np.abs(a - b) / np.maximum(np.abs(b), 1.0)).max())


def _spacetimes(g):
    from blackhorizon_b200.vaidya import ChargedVaidyaSpacetime

    return {t: ChargedVaidyaSpacetime(**dict(zip(FIELDS, (float(x) for x in g[f"{t}_params"]))))
            for t in ("default", "fly", "static")}


def test_against_reference_outputs(cuda):
    from blackhorizon_b200.vaidya import trace_vaidya_tile, vaidya_geodesic_rhs, vaidya_rk4

    g = golden("vaidya.npz")
    sp = _spacetimes(g)
    for t in ("default", "fly"):
        np.testing.assert_array_equal(sp[t]._shell_v, g[f"{t}_shell_v"])
        np.testing.assert_array_equal(sp[t]._shell_r, g[f"{t}_shell_r"])
        assert _rel(sp[t]._shell_m2, g[f"{t}_shell_m2"]) < 1e-9
    assert sp["static"]._shell_v.size == int(g["static_shell_size"])
    s = torch.as_tensor(g["sample_states"], device="cuda")
    r = torch.linalg.norm(s[:, 1:4], dim=-1)
    v = s[:, 0] + r
    for t, st in sp.items():
        geo = st.geometry_t(s[:, 0].contiguous(), s[:, 1].contiguous(), s[:, 2].contiguous(),
                            s[:, 3].contiguous())
        errs = {"h": _rel(geo.h, g[f"{t}_geo_h"]), "l": _rel(geo.l, g[f"{t}_geo_l"]),
                "hs": _rel(geo.h_spatial_scale, g[f"{t}_geo_hs"]),
                "ht": _rel(geo.h_t, g[f"{t}_geo_ht"]),
                "mass": _rel(st.mass_function(v, r), g[f"{t}_mass"]),
                "misner_sharp": _rel(st.misner_sharp_mass(v, r), g[f"{t}_misner_sharp"]),
                "rhs": _rel(vaidya_geodesic_rhs(st, s), g[f"{t}_rhs"])}
        print(t, {k: f"{e:.2g}" for k, e in errs.items()})
        assert max(errs.values()) < 1e-9, t
    for t in ("static", "default"):
        y = vaidya_rk4(sp[t], g[f"{t}_rk4_state0"], 0.002, 3000)
        print(t, "rk4", _rel(y, g[f"{t}_rk4_final"]))
        assert _rel(y, g[f"{t}_rk4_final"]) < 1e-8
    for t in ("tile_out", "tile_in"):
        esc, stop = g[f"{t}_radii"]
        status, edir, mass, v_end = trace_vaidya_tile(sp["fly"], g[f"{t}_state0"], esc, stop)
        np.testing.assert_array_equal(status, g[f"{t}_status"])
        errs = (_rel(edir, g[f"{t}_escape_dir"]), _rel(mass, g[f"{t}_end_mass"]),
                _rel(v_end, g[f"{t}_v_end"]))
        print(t, "tile", errs)
        assert max(errs) < 1e-8


def _hamiltonian(st, s):
    geo = st.geometry_t(s[:, 0].copy(), s[:, 1].copy(), s[:, 2].copy(), s[:, 3].copy())
    p_t, p_s = s[:, 4], s[:, 5:8]
    lp = -p_t + np.sum(geo.l * p_s, axis=-1)
    return 0.5 * (-p_t ** 2 + np.sum(p_s * p_s, axis=-1)) - geo.h * lp ** 2


def test_mass_function_exact_branches(cuda):
    """m(v, r) (vaidya.py:153-269) where the device skips work:
    - before the tail (v <= v_tail, v_tail itself included) the power's base is
      v_tail / v_tail and pow(1, y) = 1, so m1 = M - dm exactly, as the
      reference's float64 gives;
    - where the shell blend's clip saturates (|R(v) - r| >= w), m is m1 (outside
      the shell) or m1 + the clipped excess (inside) with no division.
    Checked against a NumPy restatement on the library's own shell table:
    exact where no power runs, within 1 ulp where one does (libm and CUDA may
    round pow differently) and inside the shell (the sum m1 + 1.0 x excess may
    be fused)."""
    from blackhorizon_b200.vaidya import ChargedVaidyaSpacetime

    rng = np.random.default_rng(7)
    st = ChargedVaidyaSpacetime(charge=0.9)  # shell launched at v = 14, after the tail start
    v = np.concatenate([rng.uniform(0.0, st.tail_start, 500), [st.tail_start, 0.0]])
    r = rng.uniform(0.3, 30.0, v.size)
    np.testing.assert_array_equal(st.mass_function(v, r), st.mass - st.tail_mass)
    v_tail = rng.uniform(st.tail_start, 14.0, 500)
    m1 = st.mass - st.tail_mass * (st.tail_start / v_tail) ** (st.tail_power - 1.0)
    np.testing.assert_array_max_ulp(st.mass_function(v_tail, np.full(500, 5.0)), m1, maxulp=1)

    fly = ChargedVaidyaSpacetime(charge=0.9, shell_start_v=6.0, shell_start_radius=1.2)
    vs = rng.uniform(6.0, 11.0, 400)
    shell_r = np.interp(vs, fly._shell_v, fly._shell_r)
    m2 = np.interp(vs, fly._shell_v, fly._shell_m2)
    inc = np.minimum(np.maximum(m2 - (fly.mass - fly.tail_mass), 0.0), fly.mass_cap)
    gap = fly.shell_width * rng.uniform(1.5, 3.0, vs.size)
    outside = fly.mass_function(vs, shell_r + gap)
    np.testing.assert_array_equal(outside, fly.mass - fly.tail_mass)
    inside_r = shell_r - gap
    ok = inside_r > 0.05
    inside = fly.mass_function(vs[ok], inside_r[ok])
    np.testing.assert_array_max_ulp(inside, (fly.mass - fly.tail_mass) + inc[ok], maxulp=1)
    assert (inc[ok] > 0).any()


def test_reference_physics_anchors(cuda):
    """tests/test_vaidya.py:32-172 through the b200 surrogate."""
    from blackhorizon_b200.vaidya import ChargedVaidyaSpacetime, vaidya_geodesic_rhs, vaidya_rk4

    st = ChargedVaidyaSpacetime(charge=0.9)
    assert abs(st.outer_horizon_radius - 1.435889) < 1e-5
    assert abs(st.inner_horizon_radius - 0.564110) < 1e-5
    assert abs(st._shell_r[-1] - st.inner_horizon_radius) < 1e-3
    assert st._shell_r[0] > st.inner_horizon_radius
    # The RHS is Hamilton's equations of the extended Hamiltonian.
    state = np.array([[20.0, 0.9, 0.3, 0.2, -1.1, 0.4, -0.7, 0.5]])
    rhs = vaidya_geodesic_rhs(st, state)
    eps = 1e-6
    for k in range(4):
        plus, minus = state.copy(), state.copy()
        plus[0, k] += eps
        minus[0, k] -= eps
        dp = -(_hamiltonian(st, plus) - _hamiltonian(st, minus))[0] / (2 * eps)
        assert abs(dp - rhs[0, 4 + k]) < 1e-6
        plus, minus = state.copy(), state.copy()
        plus[0, 4 + k] += eps
        minus[0, 4 + k] -= eps
        dx = (_hamiltonian(st, plus) - _hamiltonian(st, minus))[0] / (2 * eps)
        assert abs(dx - rhs[0, k]) < 1e-6
    # Static limit: p_t and H conserved over 20000 RK4 steps.
    static = ChargedVaidyaSpacetime(charge=0.9, tail_mass=0.0, shell_energy=0.0)
    y0 = np.array([[0.0, 5.0, 0.0, 0.0, 1.0, 0.0, 0.55, 0.0]])
    y = vaidya_rk4(static, y0, 0.002, 20000)
    assert abs(y[0, 4] - y0[0, 4]) < 1e-9
    assert abs(_hamiltonian(static, y)[0] - _hamiltonian(static, y0)[0]) < 1e-9
    # With the tail on, photon energy changes.
    y0 = np.array([[13.0, 3.0, 0.0, 0.5, 1.0, -0.9, 0.2, 0.1]])
    assert abs(vaidya_rk4(st, y0, 0.002, 3000)[0, 4] - y0[0, 4]) > 1e-4
    # Mass inflation: e-folding rate = inner-horizon surface gravity.
    wide = ChargedVaidyaSpacetime(charge=0.9, mass_cap=1e12)
    vv = wide._shell_v
    inc = wide._shell_m2 - wide.ingoing_mass(vv)
    mask = inc > 1e3
    design = np.vstack([np.ones(int(mask.sum())), vv[mask]]).T
    target = np.log(inc[mask]) + wide.tail_power * np.log(vv[mask])
    coef, *_ = np.linalg.lstsq(design, target, rcond=None)
    assert abs(coef[1] - wide.inner_surface_gravity) / wide.inner_surface_gravity < 0.05
    inc = st._shell_m2 - st.ingoing_mass(st._shell_v)
    assert float(inc[-1]) > 1e5 and float(inc[0]) < 1.0
    # The Misner-Sharp mass jumps across the shell.
    i = int(np.searchsorted(inc, 1e4))
    v, sr = float(st._shell_v[i]), float(st._shell_r[i])
    outside = float(st.misner_sharp_mass(np.array([v]), np.array([sr + 0.05]))[0])
    inside = float(st.misner_sharp_mass(np.array([v]), np.array([sr - 0.002]))[0])
    assert inside > 100.0 * outside


def test_flythrough_camera_tile(cuda):
    """The renderer's camera set-up (rain state, frozen-slice tetrad) and one
    tile traced on the device, against the reference's tile."""
    from blackhorizon_b200.frames import build_tetrad, tetrad_ray_momenta
    from blackhorizon_b200.vaidya import camera_four_velocity, rain_state, trace_vaidya_tile

    g = golden("vaidya.npz")
    st = _spacetimes(g)["fly"]
    state = rain_state(st, np.array([1.3, 0.0, 0.0]), 6.0)
    u = camera_four_velocity(st, state)
    sl = st.frozen(6.0)
    pos = state[0, 1:4]
    tet = build_tetrad(sl, pos, u, pos / np.linalg.norm(pos), np.array([0.0, 0.0, 1.0]))
    s0 = g["tile_out_state0"]
    n = s0.shape[0]
    i = np.arange(n) + 0.5
    polar = np.arccos(1.0 - 2.0 * i / n)
    az = np.pi * (1.0 + 5.0 ** 0.5) * i
    dirs = np.stack([np.cos(az) * np.sin(polar), np.sin(az) * np.sin(polar), np.cos(polar)], -1)
    mom = tetrad_ray_momenta(sl, pos, tet, dirs)
    assert _rel(mom, s0[:, 4:8]) < 1e-9
    esc, stop = g["tile_out_radii"]
    status, _, _, _ = trace_vaidya_tile(st, torch.as_tensor(s0, device="cuda"), esc, stop)
    assert status.is_cuda
    np.testing.assert_array_equal(status.cpu().numpy(), g["tile_out_status"])


def test_inflation_frame_matches_reference(cuda):
    """render_layer_frame (offline/inflation.py:243-346): the flythrough
    camera's tetrad rays on the frozen slice, the device shading of the
    reference's traced rays, and whole frames traced and shaded on the
    device, against the reference's frames (tests/golden/inflation_frame.npz)."""
    from blackhorizon_b200 import _lib
    from blackhorizon_b200.backend import ptr
    from blackhorizon_b200.offline import OfflineSettings
    from blackhorizon_b200.vaidya import (ChargedVaidyaSpacetime, layer_frame_states,
                                          render_layer_frame, render_layer_frame_device)

    g = golden("inflation_frame.npz")
    st = ChargedVaidyaSpacetime(**dict(zip(FIELDS, (float(x) for x in g["params"]))))
    w, h, ss, fov = g["frame"]
    w, h, ss = int(w), int(h), int(ss)
    settings = OfflineSettings(supersample=ss, fov_degrees=float(fov))
    for tag in ("out13", "in13", "out08"):
        look = str(g[f"{tag}_look"])
        s0 = layer_frame_states(st, g[f"{tag}_state"], w, h, float(fov), ss, look)
        assert _rel(s0, g[f"{tag}_state0"]) < 1e-12
        # The device shading of the reference's own trace outputs.
        hdr = torch.empty((h, w, 3), dtype=torch.float32, device="cuda")
        dev = lambda k: torch.as_tensor(g[f"{tag}_{k}"], device="cuda")  # noqa: E731
        status = dev("status").to(torch.int32)
        edir, mass = dev("escape_dir"), dev("end_mass")
        _lib.check(_lib.load().bh_inflation_radiance(
            float(st.mass), ptr(status), ptr(edir), ptr(mass), w, h, ss, ptr(hdr), None))
        torch.cuda.synchronize()
        ref = g[f"{tag}_hdr"]
        np.testing.assert_allclose(hdr.cpu().numpy(), ref, rtol=1e-6, atol=1e-12)
        # The whole frame on the device.
        out, rays = render_layer_frame_device(st, g[f"{tag}_state"], w, h, settings, look,
                                              return_rays=True)
        got_status = rays["status"].cpu().numpy()
        agree = float(np.mean(got_status == g[f"{tag}_status"]))
        same_px = (got_status == g[f"{tag}_status"]).reshape(h, w, ss * ss).all(axis=2)
        rel = (np.abs(out.cpu().numpy() - ref) / np.maximum(np.abs(ref), 1e-6)).max(axis=2)
        print(tag, "status agreement", agree, "max rel on equal pixels", float(rel[same_px].max()))
        assert agree >= 0.99
        assert float(np.mean(rel[same_px] < 1e-5)) >= 0.99
    host = render_layer_frame(st, g["out13_state"], w, h, settings)
    assert isinstance(host, np.ndarray) and host.dtype == np.float32 and host.shape == (h, w, 3)


def test_flythrough_worldline_matches_reference(cuda):
    """build_worldline (offline/inflation.py:77-135): the camera's worldline
    with the flythrough's defaults, against the reference's samples."""
    from blackhorizon_b200.vaidya import ChargedVaidyaSpacetime, build_worldline

    g = golden("inflation_frame.npz")
    st = ChargedVaidyaSpacetime(**dict(zip(FIELDS, (float(x) for x in g["params"]))))
    taus, states = build_worldline(st, 1.3, 6.0, st.inner_horizon_radius * 1.001)
    assert taus.size == g["worldline_taus"].size
    np.testing.assert_allclose(taus, g["worldline_taus"], rtol=1e-13)
    print("worldline: max state difference", _rel(states, g["worldline_states"]))
    assert _rel(states, g["worldline_states"]) < 1e-9
