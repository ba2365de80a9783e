"""Host-side logic of the b200 backend that needs no GPU: backend dispatch,
the Kerr radii and argument checks, the camera basis, the RHS recognition of
the integrators and the synthetic workloads."""

import functools
import math

import numpy as np
import pytest

from conftest import golden


def test_get_xp_errors_follow_reference():
    from blackhorizon_b200 import backend

    assert backend.get_xp("cpu") is np
    with pytest.raises(ValueError):
        backend.get_xp("tpu")
    if not backend.b200_available():
        with pytest.raises(RuntimeError):
            backend.get_xp("b200")


def test_kerr_radii_match_reference_tests():
    """The analytic values pinned by the reference's tests/test_kerr.py:21-49."""
    from blackhorizon_b200.kerr import KerrSpacetime

    assert KerrSpacetime(spin=0.0).outer_horizon_radius == pytest.approx(2.0)
    assert KerrSpacetime(spin=1.0).outer_horizon_radius == pytest.approx(1.0)
    st = KerrSpacetime(spin=0.6)
    assert st.outer_horizon_radius == pytest.approx(1.8)
    assert st.inner_horizon_radius == pytest.approx(0.2)
    assert KerrSpacetime(spin=0.0).isco_radius() == pytest.approx(6.0)
    assert KerrSpacetime(spin=1.0).isco_radius(True) == pytest.approx(1.0)
    assert KerrSpacetime(spin=1.0).isco_radius(False) == pytest.approx(9.0)
    assert KerrSpacetime(spin=0.0).photon_orbit_radius() == pytest.approx(3.0)
    assert KerrSpacetime(spin=1.0).photon_orbit_radius(True) == pytest.approx(1.0)
    assert KerrSpacetime(spin=1.0).photon_orbit_radius(False) == pytest.approx(4.0)
    st = KerrSpacetime(spin=0.9)
    assert st.ergosphere_radius(0.0) == pytest.approx(st.outer_horizon_radius)
    assert st.ergosphere_radius(math.pi / 2.0) == pytest.approx(2.0)
    with pytest.raises(ValueError):
        KerrSpacetime(spin=1.01)
    with pytest.raises(ValueError):
        KerrSpacetime(mass=-1.0)
    assert KerrSpacetime(1.0, 0.9).capture_radius(0.01) == pytest.approx(
        (1.0 + math.sqrt(1 - 0.81)) * 1.01)


def test_camera_basis_matches_reference():
    from blackhorizon_b200.camera import PinholeCamera

    g = golden("camera.npz")
    for k in ("c1", "c3", "pole", "free"):
        w, h = (int(v) for v in g[f"{k}_wh"])
        cam = PinholeCamera(position=tuple(g[f"{k}_position"]), target=tuple(g[f"{k}_target"]),
                            up_hint=tuple(g[f"{k}_up_hint"]), fov_degrees=float(g[f"{k}_fov"]),
                            width=w, height=h)
        np.testing.assert_array_equal(np.stack([cam.forward, cam.right, cam.up]), g[f"{k}_basis"])
        np.testing.assert_array_equal(cam.ray_directions(), g[f"{k}_dirs"])


def test_camera_argument_errors():
    from blackhorizon_b200.camera import PinholeCamera

    with pytest.raises(ValueError):
        PinholeCamera(position=(1, 0, 0), width=0)
    with pytest.raises(ValueError):
        PinholeCamera(position=(1, 0, 0), fov_degrees=180.0)
    with pytest.raises(ValueError):
        PinholeCamera.from_orbit(0.0, 30.0)
    with pytest.raises(ValueError):
        PinholeCamera(position=(0, 0, 0))


def test_integrators_reject_unknown_rhs():
    from blackhorizon_b200 import geodesics
    from blackhorizon_b200.kerr import KerrSpacetime

    st = KerrSpacetime(1.0, 0.5)
    assert geodesics.spacetime_of_rhs(geodesics.GeodesicRhs(st)) is st
    assert geodesics.spacetime_of_rhs(functools.partial(geodesics.geodesic_rhs, st)) is st
    with pytest.raises(TypeError):
        geodesics.spacetime_of_rhs(lambda b: b)


def test_raw_workload_prefix_and_radius():
    from blackhorizon_b200.workloads import RAW_RADIUS, raw_throughput_inputs

    pos, d, spin = raw_throughput_inputs(4096)
    p2, d2, s2 = raw_throughput_inputs(1000)
    np.testing.assert_array_equal(pos[:1000], p2)
    np.testing.assert_array_equal(d[:1000], d2)
    np.testing.assert_array_equal(spin[:1000], s2)
    p3, d3, s3 = raw_throughput_inputs(100, offset=500)
    np.testing.assert_array_equal(pos[500:600], p3)
    assert np.all(np.abs(spin) <= 0.95)
    # Kerr-Schild radius of every point is exactly RAW_RADIUS (up to rounding).
    a2 = spin ** 2
    q = (pos ** 2).sum(-1) - a2
    r2 = 0.5 * (q + np.sqrt(q * q + 4 * a2 * pos[:, 2] ** 2))
    np.testing.assert_allclose(np.sqrt(r2), RAW_RADIUS, rtol=1e-13)
    np.testing.assert_allclose(np.linalg.norm(d, axis=-1), 1.0, rtol=1e-14)


def test_uneven_cameras_are_deterministic():
    from blackhorizon_b200.workloads import uneven_cameras

    a = uneven_cameras()
    b = uneven_cameras()
    assert a == b and len(a) == 64
    for c in a:
        assert 64 <= c.width <= 1024 and 48 <= c.height <= 768
        assert abs(c.spin) <= 0.998 and 0.0 <= c.inclination <= 90.0
        assert 20.0 <= c.distance <= 200.0


def test_save_png_roundtrip(tmp_path):
    """imaging.save_png writes the RGB array (imaging.py:94-96)."""
    import numpy as np
    from PIL import Image

    from blackhorizon_b200.imaging import save_png

    img = (np.arange(4 * 5 * 3) % 251).astype(np.uint8).reshape(4, 5, 3)
    path = tmp_path / "frame.png"
    save_png(img, str(path))
    np.testing.assert_array_equal(np.asarray(Image.open(path).convert("RGB")), img)


def test_offline_pixel_grid_matches_reference(oracle):
    """pinhole_grid / subpixel_directions (render.py:103-161) equal the
    reference's directions on its tiles, and with supersample 2 give the
    reference's initial states through the oracle's null momenta."""
    import numpy as np

    from blackhorizon_b200.offline import FlyCamera, subpixel_directions
    from conftest import golden

    g = golden("offline_tile.npz")
    for tag, inc, az in (("a09", 82.0, 0.0), ("am07", 75.0, 40.0)):
        cam = FlyCamera.from_orbit(26.0, inc, az)
        np.testing.assert_array_equal(cam.position, g[f"{tag}_position"])
        np.testing.assert_array_equal(subpixel_directions(cam, 32, 20, 70.0, 1),
                                      g[f"{tag}_directions"])
    e = golden("emission.npz")
    spin, w, h, ss = (e["ext_params"][k] for k in range(4))
    cam = FlyCamera.from_orbit(26.0, 82.0, 0.0)
    d = subpixel_directions(cam, int(w), int(h), 70.0, int(ss))
    pos = np.tile(cam.position[None, :], (d.shape[0], 1))
    p = oracle.null_momentum(1.0, float(spin), pos, d, True, True)
    np.testing.assert_array_equal(p, e["ext_state0"][:, 4:8])


def test_plunge_worldline_matches_reference():
    """offline/infall.py:38-153 (radial_momentum, build_plunge), integrated
    by the library on the host: the reference's momenta, step counts, proper
    times and sampled states for the rain, fast and maximal presets."""
    import numpy as np

    from blackhorizon_b200.infall import build_plunge, radial_momentum
    from blackhorizon_b200.kerr import KerrSpacetime
    from conftest import golden

    g = golden("plunge.npz")
    for tag in ("rain06", "fast0", "max09"):
        spin, start, energy, stop = (float(x) for x in g[f"{tag}_args"])
        st = KerrSpacetime(1.0, spin)
        np.testing.assert_allclose(radial_momentum(st, [start, 0.0, 0.0], energy),
                                   g[f"{tag}_momentum"], rtol=1e-14, atol=1e-15)
        taus, states = build_plunge(st, start, energy, stop)
        assert taus.size == int(g[f"{tag}_count"]), tag
        idx = g[f"{tag}_index"]
        np.testing.assert_allclose(taus[idx], g[f"{tag}_taus"], rtol=1e-12)
        ref = g[f"{tag}_states"]
        rel = np.abs(states[idx] - ref) / np.maximum(np.abs(ref), 1.0)
        print(tag, "max state difference", float(rel.max()))
        assert float(rel.max()) < 1e-8
    import pytest

    with pytest.raises(ValueError):
        radial_momentum(KerrSpacetime(1.0, 0.5), [4.0, 0.0, 0.0], 0.0)  # E = 0 outside


def test_camera_paths_match_reference():
    """offline/camera_path.py: eased keyframe poses, clamping at the ends,
    orbit sweeps and the cameras they give, against the reference's."""
    import numpy as np
    import pytest

    from blackhorizon_b200.video import CameraKeyframe, CameraPath, orbit_path
    from conftest import golden

    g = golden("video.npz")
    keys = [CameraKeyframe(*row) for row in g["keys"]]
    for tag, path in (("path", CameraPath(keys)), ("orbit", orbit_path(4.0, 25.0, 70.0, 1.5))):
        for i, t in enumerate(g["times"]):
            p = path.pose_at(float(t))
            np.testing.assert_array_equal([p.time, p.distance, p.inclination_degrees,
                                           p.azimuth_degrees, p.fov_degrees], g[f"{tag}_poses"][i])
            cam = path.camera_at(float(t))
            np.testing.assert_allclose(cam.position, g[f"{tag}_positions"][i], rtol=1e-14,
                                       atol=1e-14)
            np.testing.assert_allclose(np.stack(cam.basis()), g[f"{tag}_bases"][i], atol=1e-14)
    with pytest.raises(ValueError):
        CameraPath([])
    with pytest.raises(ValueError):
        CameraPath([keys[1], keys[0]])


def test_streamed_pieces_cover_the_batch_at_aligned_starts():
    """The streamed propagate's pieces: contiguous, covering [0, n), each
    starting at a multiple of the alignment (64 rays, or the ray order's
    16,384-ray segment); with three or more pieces the first and the last hold
    about n/16 rays."""
    from blackhorizon_b200.integrators import ORDER_SEGMENT, _pieces

    for n in (1, 63, 64, 1000, 50_000, 1 << 20, 3 * ORDER_SEGMENT + 5):
        for k in (1, 2, 3, 4, 7):
            for align in (64, ORDER_SEGMENT):
                b = _pieces(n, k, align)
                assert b[0][0] == 0 and b[-1][1] == n
                assert all(x[1] == y[0] for x, y in zip(b, b[1:]))
                assert all(a < e for a, e in b)
                assert all(a % align == 0 for a, _ in b)
                assert len(b) <= k
    b = _pieces(1 << 20, 3, ORDER_SEGMENT)
    assert [e - a for a, e in b] == [65536, 917504, 65536]
