"""Batched geodesic ray tracing with adaptive stepping, b200 backend.

``trace_rays`` keeps the signature of blackhorizon/tracer.py:50-61 and
returns the same ``TraceResult``; the whole active-set loop runs in one
persistent CUDA kernel (libbh_b200 ``bh_trace``).  Extra keyword-only
arguments choose the precision policy ('fp64' reproduces the reference's
arithmetic, 'mixed' runs the stage arithmetic in float32), the launch-shape
variant and a device deadline.

``trace_cameras`` traces many pinhole cameras (each with its own spin and
escape radius) in one launch with the ray generation fused into the kernel.
"""

from __future__ import annotations

from dataclasses import dataclass
from enum import IntEnum

import torch

from . import _lib
from .backend import Array, out_like, ptr, stream_handle, to_device_f64
from .integrators import make_config
from .kerr import KerrSpacetime


class RayStatus(IntEnum):
    """Terminal state of a traced geodesic (tracer.py:21-30)."""

    IN_FLIGHT = 0
    CAPTURED = 1
    ESCAPED = 2
    MAX_STEPS = 3
    FAILED = 4
    DISK = 5
    TERMINATED = 6


@dataclass(frozen=True)
class TraceResult:
    """Outcome of tracing a batch (tracer.py:33-47).

    Attributes:
        states: final states, shape (n, 8).
        status: per-ray RayStatus value, shape (n,), int32.
        steps: accepted integration steps per ray, shape (n,), int64.
        iterations: controller iterations of the batch; equals the largest
            per-ray attempt count, as in the reference's batch loop.
        attempts / accepted: attempted and accepted ray-steps summed over rays.
    """

    states: Array
    status: Array
    steps: Array
    iterations: int
    attempts: int = 0
    accepted: int = 0


DEFAULT_TIMEOUT_S = 120.0


def _stats(lib, ws, stream, what):
    stats = _lib.TraceStats()
    _lib.check(lib.bh_trace_stats_read(ptr(ws), stats, stream), what)
    return stats


def trace_rays(
    spacetime: KerrSpacetime,
    state0: Array,
    escape_radius: float,
    max_steps: int = 20000,
    rtol: float = 1e-9,
    atol: float = 1e-12,
    initial_step: float = 0.1,
    max_step: float = 2.0,
    min_step: float = 1e-10,
    capture_margin: float = 1e-3,
    *,
    precision: str = "fp64",
    variant: int | str = -1,
    blocks_per_sm: int = 0,
    timeout_s: float = DEFAULT_TIMEOUT_S,
    workspace=None,
    project_every: int = 0,
) -> TraceResult:
    """Trace a batch of geodesics to termination (tracer.py:50-157).

    The input is copied, never mutated.  Raises ValueError when an initial
    radius is at or beyond ``escape_radius`` (tracer.py:95-99) and
    RuntimeError when the device deadline passes.  ``variant="auto"`` picks
    the launch shape with the autotuner (cached per GPU, policy and size);
    ``precision="auto"`` picks the policy too, by timing both on a probe.
    ``project_every`` K > 0 projects every ray in flight onto the null
    constraint H = 0 in float64 every K controller iterations (one Newton
    step on the spatial momentum, p_t kept); the reference never projects,
    so it is off by default and runs on the default launch shape."""
    s, host = to_device_f64(state0, "state0")
    if s.dim() != 2 or s.shape[1] != 8:
        raise ValueError("state0 must have shape (n, 8)")
    n = s.shape[0]
    lib = _lib.load()
    if precision == "auto":
        from .autotune import tune_trace_policy

        if n:
            pick = tune_trace_policy(spacetime, s, escape_radius, max_steps, rtol, atol,
                                     capture_margin, max_step)
            precision, variant = pick["precision"], pick["variant"]
        else:
            precision = "fp64"
    if variant == "auto":
        from .autotune import tune_trace

        variant = tune_trace(spacetime, s, escape_radius, precision, max_steps, rtol, atol,
                             capture_margin, max_step)["variant"] if n else -1
    states = torch.empty_like(s)
    status = torch.empty(n, dtype=torch.int32, device=s.device)
    steps = torch.empty(n, dtype=torch.int64, device=s.device)
    ws = workspace if workspace is not None else torch.empty(
        lib.bh_trace_workspace_bytes(), dtype=torch.uint8, device=s.device)
    scene = _lib.Scene(spacetime.mass, spacetime.spin,
                       spacetime.capture_radius(capture_margin), float(escape_radius))
    cfg = make_config(max_steps, rtol, atol, initial_step, max_step, min_step,
                      precision, "aos", timeout_s, variant, blocks_per_sm, project_every)
    stream = stream_handle()
    _lib.check(lib.bh_trace(cfg, scene, ptr(s), ptr(states), ptr(status), ptr(steps),
                            n, ptr(ws), stream), "trace_rays")
    st = _stats(lib, ws, stream, "trace_rays")
    if host is not None:
        return TraceResult(states=out_like(states, host, state0),
                           status=status.cpu().numpy(), steps=steps.cpu().numpy(),
                           iterations=int(st.iterations), attempts=int(st.attempts),
                           accepted=int(st.accepted))
    return TraceResult(states=out_like(states, None, state0), status=status,
                       steps=steps, iterations=int(st.iterations),
                       attempts=int(st.attempts), accepted=int(st.accepted))


@dataclass(frozen=True)
class CameraScene:
    """One camera of a batched launch: the spacetime it looks at, the camera
    and the tracer's escape radius and capture margin for it."""

    spacetime: KerrSpacetime
    camera: "object"
    escape_radius: float
    capture_margin: float = 1e-3


def camera_struct(cs: CameraScene) -> "_lib.Camera":
    cam = cs.camera
    st = cs.spacetime
    scene = _lib.Scene(st.mass, st.spin, st.capture_radius(cs.capture_margin),
                       float(cs.escape_radius))
    c = _lib.Camera()
    for name, vec in (("position", cam.position), ("forward", cam.forward),
                      ("right", cam.right), ("up", cam.up)):
        arr = getattr(c, name)
        for i in range(3):
            arr[i] = float(vec[i])
    c.fov_degrees = float(cam.fov_degrees)
    c.width = int(cam.width)
    c.height = int(cam.height)
    c.scene = scene
    return c


def camera_table(scenes):
    arr = (_lib.Camera * len(scenes))()
    for i, cs in enumerate(scenes):
        arr[i] = camera_struct(cs)
    return arr


def trace_cameras(
    scenes,
    max_steps: int = 20000,
    rtol: float = 1e-9,
    atol: float = 1e-12,
    initial_step: float = 0.1,
    max_step: float = 2.0,
    min_step: float = 1e-10,
    *,
    precision: str = "fp64",
    variant: int = -1,
    blocks_per_sm: int = 0,
    timeout_s: float = DEFAULT_TIMEOUT_S,
    project_every: int = 0,
):
    """Trace every pixel of every camera in one persistent launch.

    ``scenes`` is a sequence of CameraScene.  Returns one TraceResult per
    camera (device tensors; views into one concatenated buffer), each as if
    trace_rays had run on that camera's initial states."""
    if not scenes:
        raise ValueError("need at least one camera")
    lib = _lib.load()
    table = camera_table(scenes)
    nc = len(scenes)
    dev = torch.device("cuda", torch.cuda.current_device())
    wsb = lib.bh_trace_cameras_workspace_bytes(nc)
    ws = torch.empty(wsb, dtype=torch.uint8, device=dev)
    stream = stream_handle()
    n_rays = _lib._I64(0)
    _lib.check(lib.bh_camera_table_upload(table, nc, ptr(ws), wsb, n_rays, stream),
               "trace_cameras")
    n = int(n_rays.value)
    states = torch.empty((n, 8), dtype=torch.float64, device=dev)
    status = torch.empty(n, dtype=torch.int32, device=dev)
    steps = torch.empty(n, dtype=torch.int64, device=dev)
    cfg = make_config(max_steps, rtol, atol, initial_step, max_step, min_step,
                      precision, "aos", timeout_s, variant, blocks_per_sm, project_every)
    _lib.check(lib.bh_trace_cameras(cfg, nc, n, ptr(states), ptr(status), ptr(steps),
                                    ptr(ws), wsb, stream), "trace_cameras")
    st = _stats(lib, ws, stream, "trace_cameras")
    out = []
    off = 0
    for cs in scenes:
        k = int(cs.camera.width) * int(cs.camera.height)
        out.append(TraceResult(states=states[off:off + k], status=status[off:off + k],
                               steps=steps[off:off + k], iterations=int(st.iterations),
                               attempts=int(st.attempts), accepted=int(st.accepted)))
        off += k
    return out



class CameraBatch:
    """Many pinhole cameras traced in one persistent launch, captured once
    into a CUDA graph and replayed per frame.

    The camera table is uploaded once into the batch's workspace and the
    outputs are allocated once; ``run()`` replays the graph (counter reset +
    launch) on the current stream and ``results()`` reads the counters and
    returns one TraceResult per camera (views into the batch's buffers, which
    the next ``run()`` overwrites)."""

    def __init__(self, scenes, max_steps: int = 20000, rtol: float = 1e-9,
                 atol: float = 1e-12, initial_step: float = 0.1, max_step: float = 2.0,
                 min_step: float = 1e-10, *, precision: str = "fp64", variant: int = -1,
                 blocks_per_sm: int = 0, timeout_s: float = DEFAULT_TIMEOUT_S,
                 graph: bool = True, project_every: int = 0):
        if not scenes:
            raise ValueError("need at least one camera")
        self.lib = _lib.load()
        self.scenes = list(scenes)
        self.table = camera_table(self.scenes)
        self.nc = len(self.scenes)
        dev = torch.device("cuda", torch.cuda.current_device())
        self.wsb = self.lib.bh_trace_cameras_workspace_bytes(self.nc)
        self.ws = torch.empty(self.wsb, dtype=torch.uint8, device=dev)
        n_rays = _lib._I64(0)
        _lib.check(self.lib.bh_camera_table_upload(self.table, self.nc, ptr(self.ws), self.wsb,
                                                   n_rays, stream_handle()), "CameraBatch")
        self.n = int(n_rays.value)
        self.states = torch.empty((self.n, 8), dtype=torch.float64, device=dev)
        self.status = torch.empty(self.n, dtype=torch.int32, device=dev)
        self.steps = torch.empty(self.n, dtype=torch.int64, device=dev)
        self.cfg = make_config(max_steps, rtol, atol, initial_step, max_step, min_step,
                               precision, "aos", timeout_s, variant, blocks_per_sm,
                               project_every)
        self.graph = None
        if graph:
            torch.cuda.current_stream().synchronize()
            g = _lib._P()
            _lib.check(self.lib.bh_graph_trace_cameras(
                self.cfg, self.nc, self.n, ptr(self.states), ptr(self.status), ptr(self.steps),
                ptr(self.ws), self.wsb, g), "CameraBatch capture")
            self.graph = g

    def run(self) -> None:
        """Trace every camera's rays (asynchronous on the current stream)."""
        if self.graph is not None:
            _lib.check(self.lib.bh_graph_launch(self.graph, stream_handle()), "CameraBatch")
        else:
            _lib.check(self.lib.bh_trace_cameras(
                self.cfg, self.nc, self.n, ptr(self.states), ptr(self.status), ptr(self.steps),
                ptr(self.ws), self.wsb, stream_handle()), "CameraBatch")

    def results(self):
        st = _stats(self.lib, self.ws, stream_handle(), "CameraBatch")
        out, off = [], 0
        for cs in self.scenes:
            k = int(cs.camera.width) * int(cs.camera.height)
            out.append(TraceResult(states=self.states[off:off + k], status=self.status[off:off + k],
                                   steps=self.steps[off:off + k], iterations=int(st.iterations),
                                   attempts=int(st.attempts), accepted=int(st.accepted)))
            off += k
        return out

    def images(self, cells: int = 12):
        """One (height, width, 3) uint8 device image per camera, shaded on the
        device from the last run (imaging.py:53-91); only these pixels need
        to cross to the host."""
        from .imaging import render_image_device

        out, off = [], 0
        for cs in self.scenes:
            w, h = int(cs.camera.width), int(cs.camera.height)
            k = w * h
            res = TraceResult(states=self.states[off:off + k], status=self.status[off:off + k],
                              steps=self.steps[off:off + k], iterations=0)
            out.append(render_image_device(cs.spacetime, res, w, h, cells))
            off += k
        return out

    def close(self) -> None:
        if self.graph is not None:
            torch.cuda.current_stream().synchronize()
            _lib.check(self.lib.bh_graph_destroy(self.graph), "CameraBatch")
            self.graph = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
