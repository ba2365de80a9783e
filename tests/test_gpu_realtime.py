"""The real-time shader algorithm (realtime/reference.py:41-188) on the GPU.

Against the reference's own outputs (tests/golden/realtime.npz, made by
trace_like_shader): equatorial fans at every quality preset, a disk frame and
interior rain-observer views.  The float64 kernel fuses multiply-adds, so
final states agree to a tolerance rather than bit for bit; statuses must be
equal.  Then the reference's accuracy properties
(tests/test_realtime_reference.py): every preset shades an a = 0.9 fan
exactly like the adaptive tracer, the MEDIUM preset puts the Schwarzschild
shadow edge at 3 sqrt(3) M within 0.5 %, HIGH is exact at a = 0.998, and deep
plungers end captured with finite states.
"""

import numpy as np
import pytest
import torch

from conftest import golden

pytestmark = pytest.mark.gpu


def _cases(g):
    tags = sorted({k.rsplit("_", 1)[0] for k in g.files
                   if k.endswith("_status") and not k.endswith("truth_status")})
    for t in tags:
        yield t


def _settings(g, t):
    from blackhorizon_b200.realtime import RenderSettings

    ms, sc, mn, mx, cm, bo, esc = g[f"{t}_settings"]
    return RenderSettings(spin=float(g[f"{t}_spin"]), max_steps=int(ms), step_scale=float(sc),
                          min_step=float(mn), max_step=float(mx), capture_margin=float(cm),
                          momentum_bailout=float(bo)), float(esc)


def _run(g, t, precision):
    from blackhorizon_b200.kerr import KerrSpacetime
    from blackhorizon_b200.realtime import trace_like_shader

    settings, esc = _settings(g, t)
    disk = tuple(g[f"{t}_disk"]) if f"{t}_disk" in g.files else None
    interior = 0.02 if t.startswith("in") else None
    s0 = torch.as_tensor(g[f"{t}_state0"], device="cuda")
    return trace_like_shader(KerrSpacetime(1.0, float(g[f"{t}_spin"])), s0, settings, esc,
                             disk_radii=disk, interior_stop=interior, precision=precision)


def test_matches_reference_fp64(cuda):
    g = golden("realtime.npz")
    for t in _cases(g):
        r = _run(g, t, "fp64")
        status = r.status.cpu().numpy()
        np.testing.assert_array_equal(status, g[f"{t}_status"], err_msg=t)
        ok = np.isin(status, (2, 5))  # escaped and disk rays: finite, comparable states
        for k in ("positions", "momenta"):
            d = np.abs(getattr(r, k).cpu().numpy() - g[f"{t}_{k}"])[ok]
            scale = np.maximum(np.abs(g[f"{t}_{k}"][ok]), 1.0)
            err = float((d / scale).max()) if d.size else 0.0
            print(f"{t}: max relative {k} difference {err:.3g}")
            assert err < 1e-6, (t, k)
        if f"{t}_disk" in g.files:
            hit = status == 5
            dr = np.abs(r.hit_radii.cpu().numpy()[hit] - g[f"{t}_hit_radii"][hit]).max()
            assert dr < 1e-8
            assert np.isnan(r.hit_radii.cpu().numpy()[~hit]).all()


def test_mixed_policy_classification(cuda):
    g = golden("realtime.npz")
    for t in _cases(g):
        r = _run(g, t, "mixed")
        agree = float(np.mean(r.status.cpu().numpy() == g[f"{t}_status"]))
        print(f"{t}: mixed status agreement {agree:.4f}")
        assert agree >= 0.98, t


def _shaded_black(status):
    return (status == 1) | (status == 3)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_presets_shade_like_the_adaptive_tracer(cuda, precision):
    """tests/test_realtime_reference.py:56-76 and 95-113: every preset at
    a = 0.9 and HIGH at a = 0.998 colour the fan black exactly where the
    adaptive tracer (rtol 1e-10) captures."""
    g = golden("realtime.npz")
    for t in [c for c in _cases(g) if c.startswith("fan_a09_") or c == "fan_a0998_high"]:
        r = _run(g, t, precision)
        agree = np.mean(_shaded_black(r.status.cpu().numpy()) ==
                        _shaded_black(g[f"{t}_truth_status"]))
        print(f"{precision} {t}: agreement with the adaptive tracer {agree:.4f}")
        assert agree == 1.0, t


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_schwarzschild_edge_and_plungers(cuda, precision):
    """tests/test_realtime_reference.py:78-93 and 115-124."""
    from blackhorizon_b200 import conserved_quantities

    g = golden("realtime.npz")
    r = _run(g, "fan_a0_medium", precision)
    s0 = g["fan_a0_medium_state0"]
    e, lz = conserved_quantities(s0)
    impact = np.abs(lz / e)
    black = _shaded_black(r.status.cpu().numpy())
    b = 0.5 * (impact[black].max() + impact[~black].min())
    b_exact = 3.0 * np.sqrt(3.0)
    print(f"{precision}: Schwarzschild edge {b:.6f} vs {b_exact:.6f}")
    assert abs(b - b_exact) / b_exact < 5e-3
    p = _run(g, "fan_plunge_low", precision)
    assert bool(torch.isfinite(p.positions).all())
    assert bool((p.status == 1).all())


def test_interior_frames_match_reference(cuda):
    """frames.py mirror: rain 4-velocity, tetrad and tetrad ray momenta of the
    interior cameras equal the reference's (float64, 1e-12)."""
    from blackhorizon_b200.frames import build_tetrad, rain_four_velocity, tetrad_ray_momenta
    from blackhorizon_b200.kerr import KerrSpacetime

    g = golden("realtime.npz")
    for t in ("in19", "in05", "in_a06"):
        st = KerrSpacetime(1.0, float(g[f"{t}_spin"]))
        p = g[f"{t}_position"]
        u = rain_four_velocity(st, p[None, :])[0]
        np.testing.assert_allclose(u, g[f"{t}_four_velocity"], rtol=1e-12, atol=1e-14)
        tet = build_tetrad(st, p, u, -p / np.linalg.norm(p), np.array([0.0, 0.0, 1.0]))
        np.testing.assert_allclose(tet, g[f"{t}_tetrad"], rtol=1e-12, atol=1e-13)
        mom = tetrad_ray_momenta(st, p, tet, g[f"{t}_directions"])
        np.testing.assert_allclose(mom, g[f"{t}_state0"][:, 4:8], rtol=1e-12, atol=1e-13)


def test_host_arrays_and_budget_validation(cuda):
    from blackhorizon_b200.kerr import KerrSpacetime
    from blackhorizon_b200.realtime import RenderSettings, trace_like_shader

    g = golden("realtime.npz")
    settings, esc = _settings(g, "fan_a09_medium")
    r = trace_like_shader(KerrSpacetime(1.0, 0.9), g["fan_a09_medium_state0"], settings, esc)
    assert isinstance(r.status, np.ndarray) and r.hit_radii is None and r.steps > 0
    np.testing.assert_array_equal(r.status, g["fan_a09_medium_status"])
    with pytest.raises(ValueError):
        trace_like_shader(KerrSpacetime(1.0, 0.9), g["fan_a09_medium_state0"],
                          RenderSettings(max_steps=5000), esc)
