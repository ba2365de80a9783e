"""Batched multi-camera launches, their CUDA graph, and the autotuner.

The uneven 64-camera workload (resolutions log-uniform from 64x64 to
1024x768, spin in [-0.998, 0.998], inclination in [0, 90] deg, distance in
[20, 200] M, escape at twice the distance) runs as one persistent launch,
captured into a CUDA graph; 4096 strided pixels of every camera are checked
against the oracle in both precision policies, disagreements allowed only at
the shadow edge."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def small_scenes():
    from blackhorizon_b200.camera import PinholeCamera
    from blackhorizon_b200.kerr import KerrSpacetime
    from blackhorizon_b200.tracer import CameraScene

    return [
        CameraScene(KerrSpacetime(1.0, 0.9), PinholeCamera.from_orbit(
            50.0, 60.0, fov_degrees=30.0, width=40, height=30), 100.0, 0.01),
        CameraScene(KerrSpacetime(1.0, -0.7), PinholeCamera.from_orbit(
            30.0, 85.0, fov_degrees=35.0, width=24, height=18), 60.0, 0.01),
    ]


def uneven_scenes():
    from blackhorizon_b200.camera import PinholeCamera
    from blackhorizon_b200.kerr import KerrSpacetime
    from blackhorizon_b200.tracer import CameraScene
    from blackhorizon_b200.workloads import uneven_cameras

    out = []
    for c in uneven_cameras():
        cam = PinholeCamera.from_orbit(c.distance, c.inclination, fov_degrees=c.fov,
                                       width=c.width, height=c.height)
        out.append(CameraScene(KerrSpacetime(1.0, c.spin), cam, c.escape_radius, 0.01))
    return out


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_graph_replay_matches_direct_launch(cuda, precision):
    from blackhorizon_b200 import CameraBatch, trace_cameras

    sc = small_scenes()
    ref = trace_cameras(sc, max_steps=5000, rtol=1e-8, atol=1e-10, precision=precision)
    batch = CameraBatch(sc, max_steps=5000, rtol=1e-8, atol=1e-10, precision=precision)
    for _ in range(2):
        batch.run()
        got = batch.results()
        for a, b in zip(ref, got):
            assert torch.equal(a.status, b.status)
            assert torch.equal(a.steps, b.steps)
            assert torch.equal(a.states, b.states)
            assert a.attempts == b.attempts
    batch.close()


def oracle_status(cs, idx):
    """Statuses of pixels idx of a camera scene traced by the oracle from
    initial states it builds itself (pinhole directions, null momenta)."""
    from oracle import oracle

    cam, st = cs.camera, cs.spacetime
    d = oracle.pinhole_directions(cam.forward, cam.right, cam.up, cam.fov_degrees,
                                  cam.width, cam.height)[idx]
    pos = cam.ray_origins()[idx]
    p = oracle.null_momentum(1.0, st.spin, pos, d, True, True)
    s0 = np.zeros((idx.size, 8))
    s0[:, 1:4] = pos
    s0[:, 4:8] = p
    _, status, _, _ = oracle.trace(1.0, st.spin, s0, cs.escape_radius, max_steps=10000,
                                   rtol=1e-8, atol=1e-10, capture_margin=0.01)
    return status


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_uneven_64_cameras_against_oracle(cuda, precision):
    """One graph-captured launch of all 64 cameras.  4096 strided pixels of
    every camera (all pixels of the 64x48 ones) are traced by the oracle; the
    statuses agree except at the shadow edge: every pixel that disagrees has
    a 4-neighbour of another status in the oracle's own frame, and such
    pixels are at most 0.5 % (float64) or 1 % (mixed) of the sample."""
    from blackhorizon_b200 import CameraBatch

    sc = uneven_scenes()
    assert len(sc) == 64
    batch = CameraBatch(sc, max_steps=10000, rtol=1e-8, atol=1e-10, precision=precision)
    batch.run()
    res = batch.results()
    batch.close()
    total = differ = off_edge = 0
    for cs, r in zip(sc, res):
        w, h = cs.camera.width, cs.camera.height
        n = w * h
        idx = np.arange(n) if n <= 4096 else np.unique(
            np.round(np.linspace(0, n - 1, 4096)).astype(np.int64))
        assert idx.size >= min(n, 4096) - 1
        own = oracle_status(cs, idx)
        got = r.status.cpu().numpy()[idx]
        bad = idx[got != own]
        total += idx.size
        differ += bad.size
        if bad.size:
            rows, cols = np.divmod(bad, w)
            nbrs = np.stack([np.stack([rows - 1, cols], -1), np.stack([rows + 1, cols], -1),
                             np.stack([rows, cols - 1], -1), np.stack([rows, cols + 1], -1)],
                            axis=1)  # (bad, 4, 2)
            inside = ((nbrs[..., 0] >= 0) & (nbrs[..., 0] < h) & (nbrs[..., 1] >= 0)
                      & (nbrs[..., 1] < w))
            flat = np.where(inside, nbrs[..., 0] * w + nbrs[..., 1], 0)
            nb_status = oracle_status(cs, flat.reshape(-1)).reshape(flat.shape)
            centre = own[got != own][:, None]
            at_edge = np.any(inside & (nb_status != centre), axis=1)
            off_edge += int((~at_edge).sum())
    print("%s: %d of %d sampled pixels differ from the oracle, %d off the shadow edge"
          % (precision, differ, total, off_edge))
    assert total >= 64 * 3072
    assert off_edge == 0
    assert differ / total <= (0.005 if precision == "fp64" else 0.01)


def test_autotuner_picks_and_caches(cuda, tmp_path, monkeypatch):
    from blackhorizon_b200 import autotune, trace_rays
    from blackhorizon_b200.camera import PinholeCamera
    from blackhorizon_b200.kerr import KerrSpacetime

    monkeypatch.setenv("BH_AUTOTUNE_CACHE", str(tmp_path / "tune.json"))
    autotune._MEM.clear()
    st = KerrSpacetime(1.0, 0.9)
    cam = PinholeCamera.from_orbit(50.0, 60.0, fov_degrees=30.0, width=64, height=48)
    s0 = cam.initial_states(st)
    tuned = autotune.tune_trace(st, s0, 100.0, "fp64", 5000, 1e-8, 1e-10, 0.01)
    assert 0 <= tuned["variant"] < len(autotune.variants("fp64"))
    assert len(tuned["table"]) == len(autotune.variants("fp64"))
    assert (tmp_path / "tune.json").exists()
    assert autotune.lookup("trace", "fp64", s0.shape[0], "rtol=1.0e-08") == tuned
    # Launch shapes change scheduling only: float64 results are bit-identical.
    a = trace_rays(st, s0, 100.0, max_steps=5000, rtol=1e-8, atol=1e-10, capture_margin=0.01)
    b = trace_rays(st, s0, 100.0, max_steps=5000, rtol=1e-8, atol=1e-10, capture_margin=0.01,
                   variant="auto")
    assert torch.equal(a.states, b.states) and torch.equal(a.status, b.status)
    mixed = autotune.variants("mixed")
    assert {v["rays_per_thread"] for v in mixed} == {1, 2}
