"""The persistent tracer (bh_trace) against the reference's golden traces and
its tracer behaviour tests.

Parity bar, float64 policy: per-ray status and accepted-step counts equal to
the reference's except for rays whose step sequence an ulp-level difference
can flip (at most 0.5% of rays, all of them at the shadow edge: the captured
and escaped sets differ only where a neighbouring pixel has the other
status), final states within 1e-7 relative to max(|y|, 1) where the step
counts agree.  Mixed policy: classification agrees with the reference except
at the shadow edge (<= 1% of rays, each with a neighbour of the other status).
"""

import numpy as np
import pytest
import torch

from conftest import golden

pytestmark = pytest.mark.gpu


def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a), device="cuda")


def edge_mask(status, w, h):
    """Pixels with a 4-neighbour of a different status (the shadow edge)."""
    s = status.reshape(h, w)
    e = np.zeros_like(s, dtype=bool)
    e[1:, :] |= s[1:, :] != s[:-1, :]
    e[:-1, :] |= s[:-1, :] != s[1:, :]
    e[:, 1:] |= s[:, 1:] != s[:, :-1]
    e[:, :-1] |= s[:, :-1] != s[:, 1:]
    return e.reshape(-1)


def trace_frame(C, precision, **kw):
    from blackhorizon_b200 import trace_rays
    from blackhorizon_b200.camera import PinholeCamera
    from blackhorizon_b200.kerr import KerrSpacetime

    st = KerrSpacetime(1.0, C.spin)
    cam = PinholeCamera.from_orbit(C.distance, C.inclination, fov_degrees=C.fov,
                                   width=C.width, height=C.height)
    s0 = cam.initial_states(st)
    return trace_rays(st, s0, C.escape_radius, max_steps=C.max_steps, rtol=C.rtol,
                      atol=C.atol, capture_margin=C.capture_margin,
                      precision=precision, **kw)


def test_small_frame_fp64_matches_reference(cuda):
    from blackhorizon_b200 import trace_rays
    from blackhorizon_b200.kerr import KerrSpacetime

    g = golden("trace_c1_40x30.npz")
    res = trace_rays(KerrSpacetime(1.0, 0.9), dev(g["state0"]), 100.0, max_steps=5000,
                     rtol=1e-8, atol=1e-10, capture_margin=0.01)
    status = res.status.cpu().numpy()
    steps = res.steps.cpu().numpy()
    assert np.mean(status == g["status"]) >= 0.995
    same = steps == g["steps"]
    assert np.mean(same) >= 0.99
    ref = g["states"]
    rel = np.abs(res.states.cpu().numpy() - ref) / np.maximum(np.abs(ref), 1.0)
    assert np.max(rel[same]) < 1e-7
    assert abs(res.iterations - int(g["iterations"])) <= 5
    assert res.attempts >= int(steps.sum())


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_small_config_full_frame_classification(cuda, precision):
    from blackhorizon_b200.workloads import SHADOW_SMALL as C

    g = golden("trace_c1_160x120.npz")
    res = trace_frame(C, precision)
    status = res.status.cpu().numpy()
    ref = g["status"].astype(np.int32)
    diff = status != ref
    assert set(np.unique(status)) <= {1, 2}
    frac = 0.005 if precision == "fp64" else 0.01
    assert diff.mean() <= frac
    assert np.all(edge_mask(ref, C.width, C.height)[diff])
    if precision == "fp64":
        sub = g["sub_index"]
        same = (res.steps.cpu().numpy() == g["steps"])[sub]
        got = res.states.cpu().numpy()[sub]
        rel = np.abs(got - g["sub_states"]) / np.maximum(np.abs(g["sub_states"]), 1.0)
        # Equal step counts, step sizes equal to a few ulps: end points agree
        # to the local truncation error.
        assert np.max(rel[same]) < 1e-6


def test_full_hd_frame_mixed_classification(cuda):
    """1920x1080, a=0.9, 80 deg, fov 25, rtol 1e-9, mixed policy, against the
    reference's full-frame statuses."""
    from blackhorizon_b200.workloads import SHADOW_FULL_HD as C

    g = golden("trace_c3_status.npz")
    res = trace_frame(C, "mixed")
    status = res.status.cpu().numpy()
    ref = g["status"].astype(np.int32)
    diff = status != ref
    assert diff.mean() <= 1e-3
    assert np.all(edge_mask(ref, C.width, C.height)[diff])


def test_soa_layout_matches_aos(cuda):
    from blackhorizon_b200 import _lib
    from blackhorizon_b200.backend import ptr, stream_handle
    from blackhorizon_b200.integrators import make_config

    g = golden("trace_c1_40x30.npz")
    s0 = dev(g["state0"])
    n = s0.shape[0]
    lib = _lib.load()
    outs = []
    for layout in ("aos", "soa"):
        src = s0 if layout == "aos" else s0.t().contiguous()
        states = torch.empty_like(src)
        status = torch.empty(n, dtype=torch.int32, device="cuda")
        steps = torch.empty(n, dtype=torch.int64, device="cuda")
        ws = torch.empty(256, dtype=torch.uint8, device="cuda")
        cfg = make_config(5000, 1e-8, 1e-10, 0.1, 2.0, 1e-10, "fp64", layout, 60.0)
        scene = _lib.Scene(1.0, 0.9, (1.0 + (1 - 0.81) ** 0.5) * 1.01, 100.0)
        _lib.check(lib.bh_trace(cfg, scene, ptr(src), ptr(states), ptr(status), ptr(steps),
                                n, ptr(ws), stream_handle()))
        st = _lib.TraceStats()
        _lib.check(lib.bh_trace_stats_read(ptr(ws), st, stream_handle()))
        outs.append((states if layout == "aos" else states.t(), status, steps))
    assert torch.equal(outs[0][1], outs[1][1])
    assert torch.equal(outs[0][2], outs[1][2])
    assert torch.equal(outs[0][0], outs[1][0].contiguous())


def test_radial_infall_and_escape(cuda):
    """Reference tests/test_shadow.py:136-147."""
    from blackhorizon_b200 import build_state, null_momentum_from_velocity, trace_rays
    from blackhorizon_b200.kerr import KerrSpacetime
    from blackhorizon_b200.tracer import RayStatus

    st = KerrSpacetime(spin=0.9)
    pos = np.array([[20.0, 0.0, 0.0], [20.0, 0.0, 0.0]])
    d = np.array([[-1.0, 0.0, 0.0], [1.0, 0.0, 0.0]])
    mom = null_momentum_from_velocity(st, pos, d, time_orientation="future")
    s0 = build_state(pos, mom)
    res = trace_rays(st, s0, escape_radius=30.0)
    assert isinstance(res.status, np.ndarray)
    assert int(res.status[0]) == int(RayStatus.CAPTURED)
    assert int(res.status[1]) == int(RayStatus.ESCAPED)


def test_escape_radius_validation(cuda):
    """Reference tests/test_shadow.py:149-158: ValueError."""
    from blackhorizon_b200 import build_state, null_momentum_from_velocity, trace_rays
    from blackhorizon_b200.kerr import KerrSpacetime

    st = KerrSpacetime()
    pos = np.array([[50.0, 0.0, 0.0]])
    mom = null_momentum_from_velocity(st, pos, np.array([[-1.0, 0.0, 0.0]]))
    with pytest.raises(ValueError):
        trace_rays(st, build_state(pos, mom), escape_radius=40.0)


def test_input_not_mutated_and_empty(cuda):
    from blackhorizon_b200 import trace_rays
    from blackhorizon_b200.kerr import KerrSpacetime

    g = golden("trace_c1_40x30.npz")
    s0 = dev(g["state0"][:64])
    before = s0.clone()
    trace_rays(KerrSpacetime(1.0, 0.9), s0, 100.0)
    assert torch.equal(s0, before)
    res = trace_rays(KerrSpacetime(1.0, 0.9), s0[:0], 100.0)
    assert res.states.shape == (0, 8) and res.iterations == 0


def test_budgets_and_failures(cuda):
    """MAX_STEPS from the step budget, FAILED from min_step and from
    non-finite input (tracer.py:123-149); the oracle gives the same codes."""
    from blackhorizon_b200 import trace_rays
    from blackhorizon_b200.kerr import KerrSpacetime
    from oracle import oracle

    g = golden("trace_c1_40x30.npz")
    s0 = g["state0"][:128].copy()
    s0[5, 2] = np.nan
    st = KerrSpacetime(1.0, 0.9)
    for kw in (dict(max_steps=7), dict(min_step=0.5), dict(max_steps=40, max_step=0.3)):
        res = trace_rays(st, dev(s0), 100.0, rtol=1e-8, atol=1e-10, capture_margin=0.01, **kw)
        ostates, ostatus, osteps, oit = oracle.trace(1.0, 0.9, s0, 100.0, rtol=1e-8,
                                                     atol=1e-10, capture_margin=0.01, **kw)
        status = res.status.cpu().numpy()
        assert np.mean(status == ostatus) >= 0.99
        assert status[5] == 4
        assert abs(res.iterations - oit) <= 2


def test_deadline_returns_error_and_context_survives(cuda):
    """A deadline that has already passed ends the launch with BH_ERR_TIMEOUT;
    the next call on the same context succeeds."""
    from blackhorizon_b200 import _lib, trace_rays
    from blackhorizon_b200.kerr import KerrSpacetime

    g = golden("trace_c1_40x30.npz")
    st = KerrSpacetime(1.0, 0.9)
    with pytest.raises(_lib.BHError) as info:
        trace_rays(st, dev(g["state0"]), 100.0, max_steps=5000, timeout_s=1e-9)
    assert info.value.status == _lib.BH_ERR_TIMEOUT
    res = trace_rays(st, dev(g["state0"]), 100.0, max_steps=5000, rtol=1e-8, atol=1e-10,
                     capture_margin=0.01)
    assert np.mean(res.status.cpu().numpy() == g["status"]) >= 0.995


@pytest.mark.parametrize("variant,precision", [(v, "fp64") for v in range(4)] +
                         [(v, "mixed") for v in range(8)])
def test_every_variant_gives_identical_results(cuda, variant, precision):
    """Launch shape and register cap change scheduling only.  Float64 results
    are bit-identical; float32 results may differ in rounding (the code
    generator may fuse an unrounded float32 multiply and add differently
    under another register cap), so the mixed policy is held to its
    classification bar."""
    from blackhorizon_b200 import trace_rays
    from blackhorizon_b200.kerr import KerrSpacetime

    g = golden("trace_c1_40x30.npz")
    st = KerrSpacetime(1.0, 0.9)
    base = trace_rays(st, dev(g["state0"]), 100.0, max_steps=5000, rtol=1e-8, atol=1e-10,
                      capture_margin=0.01, precision=precision)
    res = trace_rays(st, dev(g["state0"]), 100.0, max_steps=5000, rtol=1e-8, atol=1e-10,
                     capture_margin=0.01, precision=precision, variant=variant,
                     blocks_per_sm=1)
    if precision == "mixed":
        assert (base.status == res.status).float().mean().item() >= 0.99
        return
    assert torch.equal(base.status, res.status)
    assert torch.equal(base.steps, res.steps)
    assert torch.equal(base.states, res.states)


def test_camera_batch_matches_single_traces(cuda):
    from blackhorizon_b200 import trace_cameras, trace_rays
    from blackhorizon_b200.camera import PinholeCamera
    from blackhorizon_b200.kerr import KerrSpacetime
    from blackhorizon_b200.tracer import CameraScene

    scenes = [
        CameraScene(KerrSpacetime(1.0, 0.9), PinholeCamera.from_orbit(
            50.0, 60.0, fov_degrees=30.0, width=40, height=30), 100.0, 0.01),
        CameraScene(KerrSpacetime(1.0, -0.5), PinholeCamera.from_orbit(
            25.0, 10.0, fov_degrees=40.0, width=17, height=9), 50.0, 0.01),
        CameraScene(KerrSpacetime(1.0, 0.998), PinholeCamera.from_orbit(
            120.0, 0.0, fov_degrees=20.0, width=31, height=23), 240.0, 0.01),
    ]
    for precision in ("fp64", "mixed"):
        batch = trace_cameras(scenes, max_steps=5000, rtol=1e-8, atol=1e-10,
                              precision=precision)
        for cs, res in zip(scenes, batch):
            s0 = cs.camera.initial_states(cs.spacetime)
            one = trace_rays(cs.spacetime, s0, cs.escape_radius, max_steps=5000, rtol=1e-8,
                             atol=1e-10, capture_margin=cs.capture_margin,
                             precision=precision)
            assert torch.equal(one.status, res.status)
            assert torch.equal(one.steps, res.steps)
            assert torch.equal(one.states, res.states)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_termination_near_the_thresholds(cuda, precision):
    """Rays that start from 1e-6 to 5e-2 outside the capture radius heading in,
    and as far inside the escape radius heading out, cross a threshold within
    a few steps: the kernels' radius test (the stage arithmetic's r^2 away
    from a threshold, float64 near one) must classify them as the oracle's
    float64 test does, in the tracer and in the tile tracer."""
    from blackhorizon_b200 import build_state, null_momentum_from_velocity, trace_rays
    from blackhorizon_b200.kerr import KerrSpacetime
    from blackhorizon_b200.offline import OfflineSettings, trace_tile
    from oracle import oracle

    a, margin, esc = 0.9, 0.01, 30.0
    st = KerrSpacetime(1.0, a)
    rcap = st.capture_radius(margin)
    f = np.geomspace(1e-6, 5e-2, 48)
    r0 = np.concatenate([rcap * (1.0 + f), esc * (1.0 - f)])
    out = np.concatenate([-np.ones(48), np.ones(48)])
    pos, d = [], []
    for k, (r, s) in enumerate(zip(r0, out)):
        # Polar angle of the start point: near the pole for the capture group,
        # which starts outside the ergosphere there (null_momentum_from_velocity
        # needs it, geodesics.py:130-131).
        th = 0.02 + 0.002 * k if s < 0 else 0.3 + 0.05 * (k - 48)
        w = np.sqrt(r * r + a * a)
        p = np.array([w * np.sin(th), 0.0, r * np.cos(th)])
        u = s * p / np.linalg.norm(p) + np.array([0.0, 0.15 * np.sin(k), 0.0])
        pos.append(p)
        d.append(u / np.linalg.norm(u))
    pos, d = np.array(pos), np.array(d)
    s0 = build_state(pos, null_momentum_from_velocity(st, pos, d, time_orientation="future"))
    # A small first step walks each ray across its threshold in 1 to 9 steps,
    # so accepted states land on both sides of the 1e-3 band around it.
    kw = dict(rtol=1e-9, atol=1e-12, capture_margin=margin, initial_step=1e-5)
    res = trace_rays(st, dev(s0), esc, precision=precision, **kw)
    _, ostatus, osteps, _ = oracle.trace(1.0, a, s0, esc, **kw)
    np.testing.assert_array_equal(res.status.cpu().numpy(), ostatus)
    assert set(ostatus[:48]) == {1} and set(ostatus[48:]) == {2}
    if precision == "fp64":
        np.testing.assert_array_equal(res.steps.cpu().numpy(), osteps)
    settings = OfflineSettings(spin=a, capture_margin=margin)
    tile = trace_tile(st, dev(s0), esc, settings, None, 1e-9, 12000, precision=precision)
    otile = oracle.trace_tile(1.0, a, s0, esc, None, rtol=1e-9, capture_margin=margin,
                              max_step=settings.max_step)
    np.testing.assert_array_equal(tile.status.cpu().numpy(), otile["status"])
