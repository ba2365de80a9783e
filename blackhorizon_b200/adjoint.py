"""Differentiable ray tracing: the discrete adjoint of the accepted DP5(4)
step sequence behind ``torch.autograd.Function``.

``trace_rays_differentiable(spacetime_spin, state0, ...)`` traces like
``trace_rays`` (tracer.py:50-157) and records the tape: every accepted step
size and a float64 checkpoint every K accepted steps.  Its backward pass
runs the hand-written adjoint kernel (``bh_adjoint``): each segment of K
steps is replayed from its checkpoint and swept backward, the stages of each
step recomputed inside the vector-Jacobian product.  Gradients flow to the
initial states (and so to camera pose and pixel coordinates, through the
differentiable ray generation below) and to the spin.  The step sequence is
frozen: the gradient is that of the map the trace actually applied, and
finite differences must replay the same sequence (``replay``).

Ray generation and the loss are small per-ray formulas evaluated with
PyTorch operations on the device so autograd can chain them:
``fly_camera_rays`` builds past-directed null initial states from a
FlyCamera-style yaw/pitch basis (blackhorizon/realtime/fly_camera.py:37-88)
and the pinhole grid of blackhorizon/camera.py:96-113;
``celestial_angles`` is the escape direction of blackhorizon/imaging.py:77-81
as (theta, phi) = (arccos z, atan2(y, x)).
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import torch

from . import _lib
from .backend import ptr, stream_handle
from .integrators import make_config
from .kerr import KerrSpacetime


@dataclass
class Tape:
    """The accepted-step sequence of a traced batch."""

    h: torch.Tensor            # (n, capacity) accepted step sizes
    checkpoints: torch.Tensor  # (n, ceil(capacity / every), 8) states
    steps: torch.Tensor        # (n,) accepted steps
    capacity: int
    every: int
    mass: float
    spin: float
    precision: str


# Tape entries per ray of a first attempt when the caller gives no capacity:
# a ray with more accepted steps than this makes the call trace again with
# room for max_steps.  (A tape sized for max_steps from the start holds
# n x max_steps step sizes, 5 GB for a 256x256 frame at 10000 steps, almost
# all of it unused.)
FIRST_TAPE_CAPACITY = 1024


def trace_with_tape(spacetime: KerrSpacetime, state0: torch.Tensor, escape_radius: float,
                    max_steps: int = 20000, rtol: float = 1e-9, atol: float = 1e-12,
                    initial_step: float = 0.1, max_step: float = 2.0,
                    min_step: float = 1e-10, capture_margin: float = 1e-3, *,
                    precision: str = "fp64", checkpoint_every: int = 64,
                    capacity: int | None = None, variant: int = -1,
                    timeout_s: float = 120.0):
    """trace_rays plus the tape of every ray's accepted steps.

    ``capacity`` is the tape's length per ray.  Without one the tape starts
    at FIRST_TAPE_CAPACITY entries and the call traces once more with
    max_steps entries if a ray took more accepted steps than that.

    Returns (states, status, steps, Tape)."""
    s = state0.detach().to(torch.float64).contiguous()
    n = s.shape[0]
    cap = int(capacity) if capacity else min(int(max_steps), FIRST_TAPE_CAPACITY)
    lib = _lib.load()
    dev = s.device
    states = torch.empty_like(s)
    status = torch.empty(n, dtype=torch.int32, device=dev)
    steps = torch.empty(n, dtype=torch.int64, device=dev)
    ws = torch.empty(lib.bh_trace_workspace_bytes(), dtype=torch.uint8, device=dev)
    scene = _lib.Scene(spacetime.mass, spacetime.spin,
                       spacetime.capture_radius(capture_margin), float(escape_radius))
    cfg = make_config(max_steps, rtol, atol, initial_step, max_step, min_step, precision,
                      "aos", timeout_s, variant)
    stream = stream_handle()
    while True:
        h_tape = torch.empty((n, cap), dtype=torch.float64, device=dev)
        nck = (cap + checkpoint_every - 1) // checkpoint_every
        ckpt = torch.empty((n, nck, 8), dtype=torch.float64, device=dev)
        _lib.check(lib.bh_trace_tape(cfg, scene, ptr(s), ptr(states), ptr(status), ptr(steps),
                                     n, ptr(h_tape), ptr(ckpt), cap, int(checkpoint_every),
                                     ptr(ws), stream), "trace_with_tape")
        st = _lib.TraceStats()
        rc = lib.bh_trace_stats_read(ptr(ws), st, stream)
        if rc == _lib.BH_ERR_TAPE and not capacity and cap < int(max_steps):
            cap = int(max_steps)
            continue
        _lib.check(rc, "trace_with_tape")
        break
    tape = Tape(h_tape, ckpt, steps, cap, int(checkpoint_every), spacetime.mass,
                spacetime.spin, precision)
    return states, status, steps, tape


def adjoint(tape: Tape, grad_states: torch.Tensor, precision: str | None = None,
            sort: bool = True):
    """(dL/d state0 (n,8), dL/d spin per ray (n,)) for dL/d final states.

    With ``sort`` the threads take the rays in order of decreasing accepted
    steps, rays without a cotangent last, so that the lanes of a warp sweep
    segments of equal length together; the results do not depend on it."""
    g = grad_states.detach().to(torch.float64).contiguous()
    n = g.shape[0]
    out = torch.empty_like(g)
    gspin = torch.empty(n, dtype=torch.float64, device=g.device)
    order = None
    if sort and n:
        key = tape.steps.clamp(max=tape.capacity) * (g != 0).any(dim=1)
        order = torch.argsort(key, descending=True, stable=True).contiguous()
    _lib.check(_lib.load().bh_adjoint(
        _lib.PRECISION[precision or tape.precision], tape.mass, tape.spin, ptr(tape.h),
        ptr(tape.checkpoints), ptr(tape.steps), tape.capacity, tape.every, ptr(g), ptr(out),
        ptr(gspin), ptr(order), n, stream_handle()), "adjoint")
    return out, gspin


def replay(tape: Tape, state0: torch.Tensor, spin: float | None = None,
           precision: str | None = None) -> torch.Tensor:
    """The frozen-sequence map: each ray's taped accepted steps from state0."""
    s = state0.detach().to(torch.float64).contiguous()
    out = torch.empty_like(s)
    _lib.check(_lib.load().bh_replay(
        _lib.PRECISION[precision or tape.precision], tape.mass,
        tape.spin if spin is None else float(spin), ptr(s), ptr(tape.h), ptr(tape.steps),
        tape.capacity, ptr(out), s.shape[0], stream_handle()), "replay")
    return out


class _TraceFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, state0, spin, mass, escape_radius, kwargs):
        st = KerrSpacetime(mass, float(spin))
        states, status, steps, tape = trace_with_tape(st, state0, escape_radius, **kwargs)
        ctx.tape = tape
        ctx.mark_non_differentiable(status, steps)
        return states, status, steps

    @staticmethod
    def backward(ctx, g_states, g_status, g_steps):
        tape = ctx.tape
        if g_states is None:
            return None, None, None, None, None
        g0, gspin = adjoint(tape, g_states)
        return g0, gspin.sum().reshape(()), None, None, None


def trace_rays_differentiable(spin: torch.Tensor, state0: torch.Tensor,
                              escape_radius: float, mass: float = 1.0, **kwargs):
    """trace_rays with gradients to state0 (n,8) and the 0-d spin tensor
    through the discrete adjoint.  Returns (states, status, steps); keyword
    arguments are those of trace_with_tape (max_steps, rtol, atol,
    capture_margin, precision, checkpoint_every, ...)."""
    if not isinstance(spin, torch.Tensor):
        spin = torch.tensor(float(spin), dtype=torch.float64, device=state0.device)
    return _TraceFunction.apply(state0, spin, float(mass), float(escape_radius), kwargs)


# ------------------------------------------------------ differentiable rays
def _ks_h_l(a, x, y, z, m=1.0):
    """Kerr-Schild H and spatial l (kerr.py:135-155) as PyTorch expressions."""
    a2 = a * a
    q = x * x + y * y + z * z - a2
    s = torch.sqrt(q * q + 4.0 * a2 * z * z)
    r2 = 0.5 * (q + s)
    r = torch.sqrt(r2)
    h = m * r * r2 / (r2 * r2 + a2 * z * z)
    w = r2 + a2
    l = torch.stack([(r * x + a * y) / w, (r * y - a * x) / w, z / r], dim=-1)
    return h, l


def null_momentum_torch(a, pos, dirs, m=1.0):
    """Past-directed null covector with |p_t| = 1 (geodesics.py:141-170) as
    PyTorch expressions of the position, direction and spin."""
    h, l = _ks_h_l(a, pos[..., 0], pos[..., 1], pos[..., 2], m)
    l_dot_s = (l * dirs).sum(-1)
    s_dot_s = (dirs * dirs).sum(-1)
    g_tt = 2.0 * h - 1.0
    b = 4.0 * h * l_dot_s
    c = s_dot_s + 2.0 * h * l_dot_s * l_dot_s
    sq = torch.sqrt(torch.clamp(b * b - 4.0 * g_tt * c, min=0.0))
    ra = (-b + sq) / (2.0 * g_tt)
    rb = (-b - sq) / (2.0 * g_tt)
    k_t = torch.minimum(ra, rb)
    l_dot_k = k_t + l_dot_s
    p_t = -k_t + 2.0 * h * l_dot_k
    p_s = dirs + (2.0 * h * l_dot_k)[..., None] * l
    p = torch.cat([p_t[..., None], p_s], dim=-1)
    return p / torch.abs(p_t)[..., None]


def fly_basis(yaw, pitch):
    """(forward, right, up) of a yaw/pitch camera (fly_camera.py:76-90)."""
    cp = torch.cos(pitch)
    forward = torch.stack([cp * torch.cos(yaw), cp * torch.sin(yaw), torch.sin(pitch)])
    world_up = torch.tensor([0.0, 0.0, 1.0], dtype=forward.dtype, device=forward.device)
    right = torch.linalg.cross(forward, world_up)
    norm = torch.linalg.norm(right)
    if float(norm.detach()) < 1e-9:
        right = torch.stack([torch.sin(yaw), -torch.cos(yaw), torch.zeros_like(yaw)])
    else:
        right = right / norm
    up = torch.linalg.cross(right, forward)
    return forward, right, up


def orbit_look_at(distance: float, inclination_degrees: float):
    """Yaw and pitch (radians) of a camera on the orbit sphere looking at the
    origin (fly_camera.py:37-65, 92-105)."""
    inc = math.radians(inclination_degrees)
    pos = (distance * math.sin(inc), 0.0, distance * math.cos(inc))
    nrm = math.sqrt(sum(c * c for c in pos))
    d = [-c / nrm for c in pos]
    yaw = math.atan2(d[1], d[0])
    limit = math.radians(89.0)
    pitch = max(-limit, min(limit, math.asin(d[2])))
    return yaw, pitch


def pixel_grid(width: int, height: int, fov_degrees: float, device, dtype=torch.float64):
    """(u, v) image-plane offsets of every pixel centre, row-major from the
    top-left (camera.py:102-109)."""
    half_w = math.tan(math.radians(fov_degrees) / 2.0)
    half_h = half_w * height / width
    cols = (torch.arange(width, dtype=dtype, device=device) + 0.5) / width * 2.0 - 1.0
    rows = 1.0 - (torch.arange(height, dtype=dtype, device=device) + 0.5) / height * 2.0
    v, u = torch.meshgrid(rows * half_h, cols * half_w, indexing="ij")
    return u.reshape(-1), v.reshape(-1)


def fly_camera_rays(spin, inclination_deg, yaw, pitch, distance, u, v, m=1.0):
    """Initial (n,8) states of the pixels (u, v) of a camera on the orbit
    sphere at `inclination_deg` from +z, oriented by yaw/pitch; every input
    may be a tensor that requires grad."""
    inc = inclination_deg * (math.pi / 180.0)
    zero = torch.zeros_like(inc)
    pos = torch.stack([distance * torch.sin(inc), zero, distance * torch.cos(inc)])
    fwd, right, up = fly_basis(yaw, pitch)
    d = fwd[None, :] + u[:, None] * right[None, :] + v[:, None] * up[None, :]
    d = d / torch.linalg.norm(d, dim=-1, keepdim=True)
    p0 = pos[None, :].expand(d.shape[0], 3)
    mom = null_momentum_torch(spin, p0, d, m)
    t0 = torch.zeros((d.shape[0], 1), dtype=d.dtype, device=d.device)
    return torch.cat([t0, p0, mom], dim=-1)


def celestial_angles(spin, states, m=1.0):
    """(theta, phi) of the escape direction dx^i/dlambda = p - 2 H lp l at
    each final state (geodesics.py:95-106, imaging.py:77-81)."""
    h, l = _ks_h_l(spin, states[:, 1], states[:, 2], states[:, 3], m)
    lp = -states[:, 4] + (l * states[:, 5:8]).sum(-1)
    vel = states[:, 5:8] - (2.0 * h * lp)[:, None] * l
    d = vel / torch.linalg.norm(vel, dim=-1, keepdim=True)
    theta = torch.acos(torch.clamp(d[:, 2], -1.0, 1.0))
    phi = torch.atan2(d[:, 1], d[:, 0])
    return theta, phi


def angle_loss(theta, phi, theta_t, phi_t, mask):
    """Sum over masked rays of (theta - theta*)^2 + wrap(phi - phi*)^2."""
    dphi = torch.remainder(phi - phi_t + math.pi, 2.0 * math.pi) - math.pi
    return (((theta - theta_t) ** 2 + dphi ** 2) * mask).sum()
