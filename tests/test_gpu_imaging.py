"""Shading on the device (imaging.py:27-91) against the reference's pixels.

Golden images were rendered by the reference itself (tests/golden/images.npz):
the traced 40x30 and 160x120 frames of the small config, the checkerboard of
random, cell-boundary and pole directions, and a frame with every status
code.  The device's acos/atan2 (within 2 ulp) may round differently from
NumPy's (correctly rounded) where a direction lies exactly on a cell
boundary: such directions may differ, and the test checks that every
differing one is on a boundary; every other pixel must be identical.
"""

import numpy as np
import pytest
import torch

from conftest import golden

pytestmark = pytest.mark.gpu


def test_checkerboard_matches_reference(cuda):
    from blackhorizon_b200.imaging import celestial_checkerboard

    g = golden("images.npz")
    d = g["checker_directions"]
    n_random = 4000
    for cells in (12, 7):
        got = celestial_checkerboard(torch.as_tensor(d, device="cuda"), cells).cpu().numpy()
        ref = g[f"checker_colors_{cells}"]
        bad = np.nonzero((got != ref).any(axis=1))[0]
        # A differing direction must sit on a cell boundary: one of the two
        # cell coordinates the reference floors is an integer to 1e-9.
        u = np.arccos(np.clip(d[bad, 2], -1, 1)) / np.pi * cells
        v = (np.arctan2(d[bad, 1], d[bad, 0]) + np.pi) / (2 * np.pi) * 2 * cells
        on_edge = (np.abs(u - np.round(u)) < 1e-9) | (np.abs(v - np.round(v)) < 1e-9)
        print(f"cells={cells}: {bad.size} differing directions, all on cell boundaries: "
              f"{bool(on_edge.all())}")
        assert (bad >= n_random).all()
        assert on_edge.all()
    # NumPy in, NumPy out.
    assert isinstance(celestial_checkerboard(d[:10]), np.ndarray)


def test_render_image_matches_reference_pixels(cuda):
    from blackhorizon_b200.imaging import render_image
    from blackhorizon_b200.kerr import KerrSpacetime
    from blackhorizon_b200.tracer import TraceResult

    g = golden("images.npz")
    st = KerrSpacetime(1.0, 0.9)
    for states, status, (w, h), ref in (
            (g["states_40x30"], g["status_40x30"], (40, 30), g["image_40x30"]),
            (g["mixed_states"], g["mixed_status"], (30, 20), g["mixed_image"])):
        res = TraceResult(states=torch.as_tensor(states, device="cuda"),
                          status=torch.as_tensor(status, device="cuda"),
                          steps=None, iterations=0)
        img = render_image(st, res, w, h)
        assert img.shape == (h, w, 3) and img.dtype == np.uint8
        np.testing.assert_array_equal(img, ref)
    with pytest.raises(ValueError):
        render_image(st, res, w + 1, h)


def test_traced_frame_image_against_reference_and_oracle(cuda, oracle):
    """Trace the 160x120 frame on the device (fp64 and mixed), shade it there,
    and compare with the reference's image of its own trace (>= 99.5 % of
    pixels equal; rays at the shadow edge may change class) and with the
    oracle's shading of the same device states (identical)."""
    from blackhorizon_b200 import trace_rays
    from blackhorizon_b200.camera import PinholeCamera
    from blackhorizon_b200.imaging import render_image, render_image_device
    from blackhorizon_b200.kerr import KerrSpacetime
    from blackhorizon_b200.workloads import SHADOW_SMALL as C

    g = golden("images.npz")
    st = KerrSpacetime(1.0, C.spin)
    cam = PinholeCamera.from_orbit(C.distance, C.inclination, fov_degrees=C.fov,
                                   width=C.width, height=C.height)
    s0 = cam.initial_states(st)
    for prec in ("fp64", "mixed"):
        res = trace_rays(st, s0, C.escape_radius, max_steps=C.max_steps, rtol=C.rtol,
                         atol=C.atol, capture_margin=C.capture_margin, precision=prec)
        img = render_image(st, res, C.width, C.height)
        agree = float(np.mean((img == g["image_160x120"]).all(axis=2)))
        print(f"{prec}: pixels equal to the reference's image {agree:.5f}")
        assert agree >= 0.995
        o = oracle.render_image(1.0, C.spin, res.states.cpu().numpy(),
                                res.status.cpu().numpy(), C.width, C.height)
        np.testing.assert_array_equal(img, o)
        dev = render_image_device(st, res, C.width, C.height)
        assert dev.is_cuda and torch.equal(dev.cpu(), torch.as_tensor(img))


def test_camera_batch_images(cuda):
    """CameraBatch.images() shades every camera of a batched launch on the
    device; each equals render_image of that camera's TraceResult."""
    from blackhorizon_b200 import CameraBatch
    from blackhorizon_b200.camera import PinholeCamera
    from blackhorizon_b200.imaging import render_image_device
    from blackhorizon_b200.kerr import KerrSpacetime
    from blackhorizon_b200.tracer import CameraScene

    scenes = [CameraScene(KerrSpacetime(1.0, 0.9), PinholeCamera.from_orbit(
                  50.0, 60.0, fov_degrees=30.0, width=40, height=30), 100.0, 0.01),
              CameraScene(KerrSpacetime(1.0, -0.5), PinholeCamera.from_orbit(
                  30.0, 85.0, fov_degrees=35.0, width=24, height=18), 60.0, 0.01)]
    batch = CameraBatch(scenes, max_steps=5000, rtol=1e-8, atol=1e-10)
    batch.run()
    imgs = batch.images()
    for cs, res, img in zip(scenes, batch.results(), imgs):
        w, h = cs.camera.width, cs.camera.height
        assert img.shape == (h, w, 3)
        assert torch.equal(img, render_image_device(cs.spacetime, res, w, h))
        assert int((img.sum(dim=2) == 0).sum()) > 0  # the shadow is there
    batch.close()
