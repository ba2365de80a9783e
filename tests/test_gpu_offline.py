"""Offline tile tracer with disk crossings (render.py:184-349) on the GPU.

Parity against the reference's own outputs (tests/golden/offline_tile.npz,
made by tests/golden/make_golden.py from render._trace_tile) and against the
oracle on larger frames.  The float64 kernel fuses multiply-adds, so a few
accept decisions near ratio = 1 can differ from NumPy's; trajectories then
differ at the tolerance level and a ray at a shadow, disk or rim edge may
change class.  Bars: statuses equal on the golden tiles, hit positions and
escape directions within 1e-6 on rays of equal status; >= 99 % status
agreement on the larger frames.
"""

import numpy as np
import pytest
import torch

from conftest import golden

pytestmark = pytest.mark.gpu


def _tile(tag, precision="fp64", retrace=False):
    from blackhorizon_b200.kerr import KerrSpacetime
    from blackhorizon_b200.offline import OfflineSettings, trace_tile

    g = golden("offline_tile.npz")
    spin = float(g[f"{tag}_spin"])
    st = KerrSpacetime(1.0, spin)
    settings = OfflineSettings(spin=spin)
    s0 = torch.as_tensor(g[f"{tag}_state0"], device="cuda")
    ms = int(g[f"{tag}_max_steps"])
    disk = tuple(float(x) for x in g[f"{tag}_disk"])
    esc = float(g[f"{tag}_escape_radius"])
    if retrace:
        idx = torch.as_tensor(g[f"{tag}_retrace_index"], device="cuda")
        return g, trace_tile(st, s0[idx], esc, settings, disk, settings.refine_rtol, 4 * ms,
                             precision=precision)
    return g, trace_tile(st, s0, esc, settings, disk, settings.rtol, ms, precision=precision)


def _compare(out, g, prefix, tol):
    status = out.status.cpu().numpy()
    ref = g[f"{prefix}status"]
    same = status == ref
    for k in ("escape_directions", "hit_positions", "hit_momenta"):
        d = np.abs(getattr(out, k).cpu().numpy() - g[f"{prefix}{k}"])[same]
        err = float(d.max()) if d.size else 0.0
        print(f"{prefix}{k}: max |diff| {err:.3g}")
        assert err < tol, k
    return same


@pytest.mark.parametrize("tag", ["a09", "am07"])
def test_tile_matches_reference_fp64(cuda, tag):
    g, out = _tile(tag)
    same = _compare(out, g, f"{tag}_", 1e-6)
    assert same.all(), np.nonzero(~same)
    np.testing.assert_array_equal(out.saturated.cpu().numpy().astype(np.int8),
                                  g[f"{tag}_saturated"])
    assert out.stats["disk_hits"] == int((g[f"{tag}_status"] == 5).sum())
    assert out.stats["crossings"] >= out.stats["disk_hits"]
    # Disk hits: the state is left before the crossing step, and the hit
    # point lies on the equator (the bisection cell is 2^-40 of a step).
    hit = out.status == 5
    hp = out.hit_positions[hit]
    assert float(hp[:, 2].abs().max()) < 1e-9
    # Kerr-Schild radius on the equator: x^2 + y^2 = r^2 + a^2.
    a = float(g[f"{tag}_spin"])
    r = torch.sqrt(hp[:, 0] ** 2 + hp[:, 1] ** 2 - a * a)
    r_in, r_out = (float(x) for x in g[f"{tag}_disk"])
    assert float(r.min()) >= r_in - 1e-9 and float(r.max()) <= r_out + 1e-9


def test_photon_shell_retrace_matches_reference(cuda):
    g, out = _tile("am07", retrace=True)
    same = _compare(out, g, "am07_retrace_", 1e-6)
    assert same.all()


def test_tile_mixed_policy(cuda):
    """float32 stages, float64 state, crossing refinement and directions."""
    for tag in ("a09", "am07"):
        g, out = _tile(tag, precision="mixed")
        status = out.status.cpu().numpy()
        agree = float(np.mean(status == g[f"{tag}_status"]))
        print(f"{tag} mixed status agreement {agree:.4f}")
        assert agree >= 0.97
        _compare(out, g, f"{tag}_", 1e-3)


def _oracle_tile(oracle, spin, s0, esc, disk, rtol, ms):
    return oracle.trace_tile(1.0, spin, s0, esc, disk, rtol=rtol, max_steps=ms)


def test_frame_two_pass_against_oracle(cuda, oracle):
    """trace_frame at 64x40 (2560 rays, supersample 1) of the renderer's
    default view against the oracle's tile tracer with the same two passes."""
    from blackhorizon_b200.kerr import KerrSpacetime
    from blackhorizon_b200.offline import (FlyCamera, OfflineSettings, camera_states,
                                           disk_radii, trace_frame)

    settings = OfflineSettings(spin=0.9, supersample=1, max_steps=400)
    cam = FlyCamera.from_orbit(26.0, 82.0, 0.0)
    st = KerrSpacetime(1.0, 0.9)
    s0 = camera_states(cam, st, 64, 40, settings)
    fr = trace_frame(cam, 64, 40, settings, state0=s0)
    radii = disk_radii(st, settings)
    s0n = s0.cpu().numpy()
    o = _oracle_tile(oracle, 0.9, s0n, fr.escape_radius, radii, settings.rtol, settings.max_steps)
    retrace = (o["saturated"] != 0) & (o["status"] != 5)
    np.testing.assert_array_equal(fr.retraced.cpu().numpy(), retrace)
    assert retrace.sum() > 0
    idx = np.nonzero(retrace)[0]
    o2 = _oracle_tile(oracle, 0.9, s0n[idx], fr.escape_radius, radii, settings.refine_rtol,
                      4 * settings.max_steps)
    for k in ("status", "escape_directions", "hit_positions", "hit_momenta"):
        o[k][idx] = o2[k]
    status = fr.status.cpu().numpy()
    agree = float(np.mean(status == o["status"]))
    print("frame status agreement", agree, np.bincount(status, minlength=6))
    assert agree >= 0.99
    same = status == o["status"]
    for k in ("escape_directions", "hit_positions"):
        d = np.abs(getattr(fr, k).cpu().numpy() - o[k])[same]
        assert float(d.max()) < 1e-6, k


def test_no_disk_and_empty_tile(cuda, oracle):
    from blackhorizon_b200.kerr import KerrSpacetime
    from blackhorizon_b200.offline import OfflineSettings, trace_tile

    g = golden("offline_tile.npz")
    st = KerrSpacetime(1.0, 0.9)
    settings = OfflineSettings(spin=0.9)
    s0 = g["a09_state0"]
    esc = float(g["a09_escape_radius"])
    out = trace_tile(st, s0, esc, settings, None, 1e-9, 12000)
    assert isinstance(out.status, np.ndarray)  # host in, host out
    o = _oracle_tile(oracle, 0.9, s0, esc, None, 1e-9, 12000)
    assert (out.status == 5).sum() == 0
    assert np.mean(out.status == o["status"]) >= 0.99
    assert out.stats["crossings"] == 0
    empty = trace_tile(st, torch.zeros((0, 8), dtype=torch.float64, device="cuda"), esc,
                       settings, (2.3, 18.0), 1e-9, 100)
    assert empty.status.shape == (0,)


def test_deadline_leaves_rays_in_flight(cuda):
    """A deadline that has already passed: every ray is written as IN_FLIGHT
    (its initial state) and the call reports BH_ERR_TIMEOUT."""
    from blackhorizon_b200._lib import BHError
    from blackhorizon_b200.kerr import KerrSpacetime
    from blackhorizon_b200.offline import OfflineSettings, trace_tile

    g = golden("offline_tile.npz")
    st = KerrSpacetime(1.0, 0.9)
    s0 = torch.as_tensor(g["a09_state0"], device="cuda")
    with pytest.raises(BHError):
        trace_tile(st, s0, float(g["a09_escape_radius"]), OfflineSettings(), (2.3, 18.0), 1e-9,
                   12000, timeout_s=1e-9)
    # The context is still usable.
    out = trace_tile(st, s0[:8], float(g["a09_escape_radius"]), OfflineSettings(), (2.3, 18.0),
                     1e-9, 12000)
    assert (out.status.cpu().numpy() > 0).all()


INTERIOR_TAGS = ["sheet", "ideal", "disk", "schw"]


def _interior(tag, precision="fp64"):
    from blackhorizon_b200.kerr import KerrSpacetime
    from blackhorizon_b200.offline import OfflineSettings, trace_tile

    g = golden("offline_interior.npz")
    spin = float(g[f"{tag}_spin"])
    disk = tuple(float(x) for x in g[f"{tag}_disk"]) if g[f"{tag}_disk"][1] > 0 else None
    settings = OfflineSettings(spin=spin, supersample=1, fov_degrees=80.0,
                               disk_enabled=disk is not None)
    s0 = torch.as_tensor(g[f"{tag}_state0"], device="cuda")
    out = trace_tile(KerrSpacetime(1.0, spin), s0, float(g[f"{tag}_escape_radius"]), settings,
                     disk, settings.rtol, settings.max_steps, float(g[f"{tag}_stop"]),
                     precision=precision)
    return g, out


@pytest.mark.parametrize("tag", INTERIOR_TAGS)
def test_interior_tile_matches_reference(cuda, tag):
    """Interior cameras (render.py:203-248): tetrad rays from inside the
    horizon cross it backwards in time, end TERMINATED at the stop radius or
    on diverging momentum, escape, or hit the disk; statuses equal the
    reference's, escape directions (with each ray's own energy) and hits
    within 1e-6."""
    g, out = _interior(tag)
    same = _compare(out, g, f"{tag}_", 1e-6)
    assert same.all(), np.nonzero(~same)
    np.testing.assert_array_equal(out.saturated.cpu().numpy().astype(np.int8),
                                  g[f"{tag}_saturated"])
    status = out.status.cpu().numpy()
    assert (status == 1).sum() == 0  # interior rays are never CAPTURED
    if tag != "disk":
        assert (status == 6).sum() > 400
    # A TERMINATED ray ends at the stop or with a large spatial momentum.
    st = out.states[out.status == 6]
    if st.shape[0]:
        from blackhorizon_b200.kerr import KerrSpacetime

        r = KerrSpacetime(1.0, float(g[f"{tag}_spin"])).kerr_schild_radius(
            st[:, 1].contiguous(), st[:, 2].contiguous(), st[:, 3].contiguous())
        pn = torch.linalg.norm(st[:, 5:8], dim=-1)
        stop = float(g[f"{tag}_stop"])
        assert bool(((r <= stop * 1.002) | (pn > 1e3)).all())


def test_interior_tile_mixed_policy(cuda):
    for tag in INTERIOR_TAGS:
        g, out = _interior(tag, precision="mixed")
        agree = float(np.mean(out.status.cpu().numpy() == g[f"{tag}_status"]))
        print(f"{tag} mixed status agreement {agree:.4f}")
        assert agree >= 0.97


def test_tetrad_frame_matches_reference(cuda):
    """trace_frame with a camera tetrad (render.py:520-630): the rain
    observer's tetrad and the tetrad ray momenta built by the b200 frames
    module equal the reference's, and the frame's statuses equal its tile."""
    from blackhorizon_b200.frames import build_tetrad, rain_four_velocity
    from blackhorizon_b200.kerr import KerrSpacetime
    from blackhorizon_b200.offline import (FlyCamera, OfflineSettings, tetrad_camera_states,
                                           trace_frame)

    g = golden("offline_interior.npz")
    for tag in ("disk", "sheet"):
        spin = float(g[f"{tag}_spin"])
        st = KerrSpacetime(1.0, spin)
        pos = g[f"{tag}_position"]
        vel = rain_four_velocity(st, pos[None, :])[0]
        np.testing.assert_allclose(vel, g[f"{tag}_velocity"], rtol=1e-13, atol=1e-13)
        tet = build_tetrad(st, pos, vel, g[f"{tag}_forward"], g[f"{tag}_up"])
        np.testing.assert_allclose(tet, g[f"{tag}_tetrad"], rtol=1e-12, atol=1e-12)
        settings = OfflineSettings(spin=spin, supersample=1, fov_degrees=80.0,
                                   disk_enabled=bool(g[f"{tag}_disk"][1] > 0))
        cam = FlyCamera(position=pos.copy(), yaw=0.0, pitch=0.0)
        s0 = tetrad_camera_states(cam, st, tet, 32, 24, settings)
        np.testing.assert_allclose(s0.cpu().numpy(), g[f"{tag}_state0"], rtol=1e-12,
                                   atol=1e-12)
        fr = trace_frame(cam, 32, 24, settings, camera_tetrad=tet,
                         interior_stop=float(g[f"{tag}_stop"]))
        assert fr.escape_radius == float(g[f"{tag}_escape_radius"])
        agree = float(np.mean(fr.status.cpu().numpy() == g[f"{tag}_status"]))
        print(f"{tag} tetrad frame status agreement {agree:.4f}")
        assert agree >= 0.99


def test_device_camera_rays_match_reference(cuda):
    """bh_offline_camera_rays builds render_hdr's initial states on the device
    (render.py:103-161, 555-599): the reference's states for its 32x20 tiles
    and the 48x30 supersample-2 frame; tetrad states are covered by
    test_tetrad_frame_matches_reference."""
    from blackhorizon_b200.kerr import KerrSpacetime
    from blackhorizon_b200.offline import FlyCamera, OfflineSettings, camera_states

    g = golden("offline_tile.npz")
    cases = [(g[f"{t}_state0"], float(g[f"{t}_spin"]), inc, az, 32, 20, 1)
             for t, inc, az in (("a09", 82.0, 0.0), ("am07", 75.0, 40.0))]
    e = golden("emission.npz")
    cases.append((e["ext_state0"], 0.9, 82.0, 0.0, 48, 30, 2))
    for ref, spin, inc, az, w, h, ss in cases:
        cam = FlyCamera.from_orbit(26.0, inc, az)
        s0 = camera_states(cam, KerrSpacetime(1.0, spin), w, h,
                           OfflineSettings(spin=spin, supersample=ss))
        assert s0.shape == ref.shape
        got = s0.cpu().numpy()
        np.testing.assert_array_equal(got[:, :4], ref[:, :4])
        rel = np.abs(got - ref) / np.maximum(np.abs(ref), 1e-300)
        print("camera rays: max relative difference", float(rel.max()))
        assert float(rel.max()) < 1e-14


def test_plunge_tetrads_and_frame(cuda):
    """offline/infall.py:156-262: the camera tetrads at worldline samples
    equal the reference's, and a plunge frame rendered on the device (tetrad
    rays, interior stop at the Cauchy horizon, disk) matches the reference's
    render_hdr frame."""
    from blackhorizon_b200.infall import plunge_frame, plunge_tetrad
    from blackhorizon_b200.kerr import KerrSpacetime
    from blackhorizon_b200.offline import OfflineSettings

    g = golden("plunge.npz")
    spin, start, energy, stop = (float(x) for x in g["rain06_args"])
    st = KerrSpacetime(1.0, spin)
    for look in ("inward", "outward", "side"):
        _, tet = plunge_tetrad(st, g[f"tetrad_{look}_sample"], look)
        np.testing.assert_allclose(tet, g[f"tetrad_{look}"], rtol=1e-12, atol=1e-12)
    settings = OfflineSettings(spin=spin, supersample=1, fov_degrees=80.0)
    hdr = plunge_frame(st, g["frame_sample"], 32, 20, settings, "inward", stop)
    ref = g["frame_hdr"]
    rel = (np.abs(hdr.cpu().numpy() - ref) / np.maximum(np.abs(ref), 1e-6)).max(axis=2)
    print("plunge frame: pixels within 1e-5:", float(np.mean(rel < 1e-5)), "max", float(rel.max()))
    assert float(np.mean(rel < 1e-5)) >= 0.99
