"""bh_trace_cameras_noalloc -- the multi-camera trace for callers that cannot
allocate device memory (an application that owns all GPU memory through its
own fixed pool and lends this library only its output buffers, or code under
a hard memory budget).  Its scratch (launch counters, work-queue head, camera
table) lives in a static device array of the library instead of a
caller-owned workspace.

Checked through the C ABI against bh_trace_cameras with a caller-owned
workspace: both run the same kernel, so status, step counts and states must
be identical (the same bar as the camera-batch tests), on two calls in a row
(the second call must start from cleared counters, not the first call's).
This file is collected last so a failure here cannot stop the other tests."""

import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def scenes():
    from blackhorizon_b200.camera import PinholeCamera
    from blackhorizon_b200.kerr import KerrSpacetime
    from blackhorizon_b200.tracer import CameraScene

    return [
        CameraScene(KerrSpacetime(1.0, 0.9), PinholeCamera.from_orbit(
            50.0, 60.0, fov_degrees=30.0, width=40, height=30), 100.0, 0.01),
        CameraScene(KerrSpacetime(1.0, -0.5), PinholeCamera.from_orbit(
            25.0, 10.0, fov_degrees=40.0, width=17, height=9), 50.0, 0.01),
        CameraScene(KerrSpacetime(1.0, 0.998), PinholeCamera.from_orbit(
            120.0, 0.0, fov_degrees=20.0, width=31, height=23), 240.0, 0.01),
    ]


def outputs(n):
    return (torch.empty((n, 8), dtype=torch.float64, device="cuda"),
            torch.empty(n, dtype=torch.int32, device="cuda"),
            torch.empty(n, dtype=torch.int64, device="cuda"))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_noalloc_matches_workspace_trace_twice(cuda, precision):
    from blackhorizon_b200 import _lib
    from blackhorizon_b200.backend import ptr, stream_handle
    from blackhorizon_b200.integrators import make_config
    from blackhorizon_b200.tracer import camera_table

    lib = _lib.load()
    sc = scenes()
    table = camera_table(sc)
    nc = len(sc)
    n = sum(c.camera.width * c.camera.height for c in sc)
    cfg = make_config(5000, 1e-8, 1e-10, 0.1, 2.0, 1e-10, precision, "aos", 60.0)
    stream = stream_handle()

    # Existing entry point with a caller-owned workspace.
    wsb = lib.bh_trace_cameras_workspace_bytes(nc)
    ws = torch.empty(wsb, dtype=torch.uint8, device="cuda")
    n_rays = ctypes.c_int64(0)
    _lib.check(lib.bh_camera_table_upload(table, nc, ptr(ws), wsb, n_rays, stream))
    assert n_rays.value == n
    ref_states, ref_status, ref_steps = outputs(n)
    _lib.check(lib.bh_trace_cameras(cfg, nc, n, ptr(ref_states), ptr(ref_status),
                                    ptr(ref_steps), ptr(ws), wsb, stream))
    ref_stats = _lib.TraceStats()
    _lib.check(lib.bh_trace_stats_read(ptr(ws), ref_stats, stream))

    for _ in range(2):
        states, status, steps = outputs(n)
        stats = _lib.TraceStats()
        _lib.check(lib.bh_trace_cameras_noalloc(cfg, table, nc, ptr(states), ptr(status),
                                                ptr(steps), stats, stream))
        assert torch.equal(status, ref_status)
        assert torch.equal(steps, ref_steps)
        assert torch.equal(states, ref_states)
        assert (stats.iterations, stats.attempts, stats.accepted) == (
            ref_stats.iterations, ref_stats.attempts, ref_stats.accepted)
        assert stats.timed_out == 0 and stats.bad_rays == 0
    assert set(np.unique(ref_status.cpu().numpy())) <= {1, 2}


def test_noalloc_rejects_more_cameras_than_its_scratch_holds(cuda):
    from blackhorizon_b200 import _lib
    from blackhorizon_b200.backend import stream_handle
    from blackhorizon_b200.integrators import make_config
    from blackhorizon_b200.tracer import camera_table

    lib = _lib.load()
    sc = scenes()[:1] * 257
    table = camera_table(sc)
    cfg = make_config(5000, 1e-8, 1e-10, 0.1, 2.0, 1e-10, "fp64", "aos", 60.0)
    states, status, steps = outputs(8)
    rc = lib.bh_trace_cameras_noalloc(cfg, table, len(sc), states.data_ptr(),
                                      status.data_ptr(), steps.data_ptr(), None,
                                      stream_handle())
    assert rc == _lib.BH_ERR_INVALID_ARGUMENT
    assert b"at most 256 cameras" in lib.bh_last_error()
