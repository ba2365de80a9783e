"""The real-time viewer's frames on the GPU: the shader algorithm's trace shaded
as realtime/shaders/kerr_tracer.frag:205-420 shades it (headless.py:32-48).

No OpenGL context exists here, so the shader cannot run; the shading is
restated from its source in the device kernel and, independently, in the C
oracle (both float32, like the shader).  Checks:
- in checkerboard mode the sky equals the imaging module's colours, which
  are pinned to the reference's own images;
- the device equals the oracle's restatement on the same trace, except
  where float32 functions (sinf, powf, atan2f, acosf) of the two libraries
  differ by an ulp at a cell, star or rounding boundary;
- interior frames carry the blue-sheet glow and whiteout of the engine's
  uniforms.
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _settings(**kw):
    from blackhorizon_b200.realtime import QualityPreset, RenderSettings

    return RenderSettings(**kw).apply_preset(QualityPreset.MEDIUM)


def _oracle_params(oracle, sh):
    p = oracle.RealtimeShading()
    for name, _ in oracle.RealtimeShading._fields_:
        setattr(p, name, sh[name])
    return p


def test_checkerboard_sky_matches_imaging(cuda):
    """Escaped pixels take the reference's checker colours (104, 128, 178) /
    (24, 30, 52); captured pixels are black."""
    from blackhorizon_b200.imaging import render_image_device
    from blackhorizon_b200.kerr import KerrSpacetime
    from blackhorizon_b200.offline import FlyCamera
    from blackhorizon_b200.realtime import BackgroundMode, render_frame_device
    from blackhorizon_b200.tracer import TraceResult

    settings = _settings(spin=0.9, disk_enabled=False, background=BackgroundMode.CHECKERBOARD)
    cam = FlyCamera.from_orbit(30.0, 85.0, 0.0)
    w, h = 192, 108
    rgb, res, sh = render_frame_device(settings, cam, w, h, return_rays=True)
    assert rgb.shape == (h, w, 3) and rgb.dtype == torch.uint8
    status = res.status.cpu().numpy()
    ref = render_image_device(KerrSpacetime(1.0, 0.9),
                              TraceResult(states=sh["states"], status=res.status, steps=None,
                                          iterations=0), w, h).cpu().numpy().reshape(-1, 3)
    got = rgb.cpu().numpy().reshape(-1, 3)
    esc = status == 2
    same = np.all(got[esc] == ref[esc], axis=1)
    print("escaped", int(esc.sum()), "equal", float(same.mean()))
    assert esc.sum() > 0.5 * status.size and same.mean() > 0.995
    assert np.all(got[status == 1] == 0)


@pytest.mark.parametrize("background", [0, 1])
def test_frame_matches_oracle_shading(cuda, oracle, background):
    """Disk, starfield or checkerboard, the 8-bit colours of the device against
    the oracle's restatement of the shader on the same trace."""
    from blackhorizon_b200.offline import FlyCamera
    from blackhorizon_b200.realtime import BackgroundMode, render_frame_device

    settings = _settings(spin=0.9, background=BackgroundMode(background), exposure=1.5)
    cam = FlyCamera.from_orbit(30.0, 82.0, 20.0)
    w, h = 256, 144
    rgb, res, sh = render_frame_device(settings, cam, w, h, return_rays=True)
    status = res.status.cpu().numpy()
    assert (status == 5).sum() > 1000 and (status == 2).sum() > 1000
    o = oracle.realtime_shade(_oracle_params(oracle, sh), status, sh["states"].cpu().numpy(),
                              sh["hit_positions"].cpu().numpy(),
                              sh["hit_momenta"].cpu().numpy(), sh["temperature"],
                              sh["blackbody"])
    got = rgb.cpu().numpy().reshape(-1, 3).astype(int)
    diff = np.abs(got - o.astype(int)).max(axis=1)
    esc = status == 2
    print("pixels off by > 1 level:", int((diff > 1).sum()), "of", diff.size,
          "escaped:", int((diff[esc] > 1).sum()), "disk pixels max off:",
          int(diff[status == 5].max()))
    assert diff[status == 5].max() <= 2
    if background == 0:
        assert (diff > 1).mean() < 2e-3
    else:
        # The starfield hashes floor(220 d) and raises the hash to the 60th
        # power: where a direction's float32 rounding differs by an ulp
        # between the two libraries at a cell edge, a star moves.  Only sky
        # pixels may differ, and few of them.
        assert np.all(diff[~esc] <= 2)
        assert (diff[esc] > 1).mean() < 1e-2
    # Reinhard keeps disk colours below white.
    assert got[status == 5].max() <= 255


def test_interior_frame_sheet_and_whiteout(cuda, oracle):
    """A realistic interior camera close to the inner horizon: rays ending on
    the terminal surface glow, and the frame washes toward white by the
    engine's whiteout fraction."""
    from blackhorizon_b200.emission import blueshift_amplification, whiteout_fraction
    from blackhorizon_b200.kerr import KerrSpacetime
    from blackhorizon_b200.offline import FlyCamera
    from blackhorizon_b200.realtime import render_frame, render_frame_device

    settings = _settings(spin=0.9, interior_mode=True, interior_journey="realistic",
                         disk_enabled=False)
    cam = FlyCamera(position=np.array([0.03, 0.03, 0.58]), yaw=0.0, pitch=-1.2)
    w, h = 96, 64
    rgb, res, sh = render_frame_device(settings, cam, w, h, return_rays=True)
    st = KerrSpacetime(1.0, 0.9)
    b = float(blueshift_amplification(st, np.array([float(np.asarray(st.kerr_schild_radius(
        np.array([0.03]), np.array([0.03]), np.array([0.58])))[0])]))[0])
    white = float(whiteout_fraction(np.array([b]))[0])
    assert abs(sh["whiteout"] - white) < 1e-6 and white > 0.0 and sh["sheet_radiance"] > 0.0
    status = res.status.cpu().numpy()
    print("statuses", np.bincount(status, minlength=7), "B", b, "white", white)
    assert (status == 6).sum() > 0
    got = rgb.cpu().numpy().reshape(-1, 3).astype(int)
    floor = np.floor(np.array([0.90, 0.95, 1.0]) * white * 255.0) - 1
    assert np.all(got >= floor)
    o = oracle.realtime_shade(_oracle_params(oracle, sh), status, sh["states"].cpu().numpy(),
                              sh["hit_positions"].cpu().numpy(),
                              sh["hit_momenta"].cpu().numpy(), sh["temperature"],
                              sh["blackbody"])
    assert np.abs(got - o.astype(int)).max() <= 1
    host = render_frame(settings, cam, w, h)
    assert isinstance(host, np.ndarray) and host.shape == (h, w, 3)
    with pytest.raises(ValueError):
        render_frame(settings, cam, w, h, ctx=object())
