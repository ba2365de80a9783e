"""Discrete adjoint of the accepted DP5(4) step sequence.

The gradient is that of the map the trace applied: each ray's accepted step
sizes are frozen (recorded on the tape).  Checks:

* gradient of a linear functional of the end state with respect to all 8
  initial-state components and the spin, against central finite differences
  (h = 1e-6) of the frozen-sequence replay, float64;
* the analytic Hamiltonian gradient: H is conserved along the flow, so the
  adjoint of L = H(y_N) must return grad H(y_0) = (0, -pdot, tdot, xdot) at
  the initial state, with the derivatives from the reference's Hamilton
  equations (the oracle's geodesic_rhs, geodesics.py:42-74);
* a small version of the differentiable-tracing workload (celestial-angle
  loss against a target frame at another spin): gradients with respect to
  spin, inclination, yaw and pitch against central finite differences,
  float64, and the mixed policy against float64.
"""

import math

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def small_frame(spin=0.7, w=24, hgt=18, inc=60.0):
    from blackhorizon_b200.adjoint import fly_camera_rays, orbit_look_at, pixel_grid

    dev = torch.device("cuda", 0)
    yaw0, pitch0 = orbit_look_at(50.0, inc)
    u, v = pixel_grid(w, hgt, 30.0, dev)
    t = lambda x: torch.tensor(x, dtype=torch.float64, device=dev)  # noqa: E731
    return fly_camera_rays(t(spin), t(inc), t(yaw0), t(pitch0), 50.0, u, v), (u, v, yaw0, pitch0)


def test_linear_functional_against_finite_differences(cuda):
    from blackhorizon_b200.adjoint import adjoint, replay, trace_with_tape
    from blackhorizon_b200.kerr import KerrSpacetime

    st = KerrSpacetime(1.0, 0.7)
    s0, _ = small_frame()
    s0 = s0[::7].contiguous()  # 62 rays
    states, status, steps, tape = trace_with_tape(st, s0, 100.0, max_steps=5000, rtol=1e-9,
                                                  capture_margin=0.01, checkpoint_every=16)
    esc = (status == 2)
    assert int(esc.sum()) > 10
    rng = np.random.default_rng(1)
    wts = torch.as_tensor(rng.normal(size=(s0.shape[0], 8)), device="cuda") * esc[:, None]
    g0, gspin = adjoint(tape, wts)
    # The replay reproduces the trace.
    torch.testing.assert_close(replay(tape, s0), states, rtol=1e-12, atol=1e-12)
    eps = 1e-6
    fd = torch.zeros_like(s0)
    for c in range(8):
        d = torch.zeros_like(s0)
        d[:, c] = eps
        fp = (replay(tape, s0 + d) * wts).sum(1)
        fm = (replay(tape, s0 - d) * wts).sum(1)
        fd[:, c] = (fp - fm) / (2 * eps)
    fa = ((replay(tape, s0, spin=0.7 + eps) - replay(tape, s0, spin=0.7 - eps)) * wts).sum(1) / (2 * eps)
    scale = torch.clamp(g0.abs().amax(1, keepdim=True), min=1e-3)
    rel = ((g0 - fd).abs() / scale)[esc]
    print("adjoint vs FD: max relative %.3g, median %.3g" % (rel.max(), rel.median()))
    assert float(rel.max()) < 1e-4
    rel_a = ((gspin - fa).abs() / torch.clamp(fa.abs(), min=1e-3))[esc]
    assert float(rel_a.max()) < 1e-4


def test_adjoint_of_hamiltonian_is_its_gradient(cuda):
    """H(y_N) = H(y_0) along the flow, so d H(y_N) / d y_0 = grad H(y_0)."""
    from oracle import oracle

    from blackhorizon_b200.adjoint import adjoint, trace_with_tape
    from blackhorizon_b200.kerr import KerrSpacetime

    st = KerrSpacetime(1.0, 0.7)
    s0, _ = small_frame()
    s0 = s0[::5].contiguous()
    states, status, steps, tape = trace_with_tape(st, s0, 100.0, max_steps=5000, rtol=1e-10,
                                                  atol=1e-13, capture_margin=0.01)
    esc = (status == 2).cpu().numpy()

    def grad_h(y):
        d = oracle.rhs(1.0, 0.7, y)  # (tdot, xdot, ydot, zdot, 0, pdot)
        g = np.zeros_like(y)
        g[:, 1:4] = -d[:, 5:8]
        g[:, 4] = d[:, 0]
        g[:, 5:8] = d[:, 1:4]
        return g

    gN = torch.as_tensor(grad_h(states.cpu().numpy()), device="cuda")
    g0, _ = adjoint(tape, gN)
    expect = grad_h(s0.cpu().numpy())
    got = g0.cpu().numpy()
    rel = np.abs(got - expect).max(1) / np.abs(expect).max(1)
    print("adjoint of H vs analytic grad H: median %.3g max %.3g" % (
        np.median(rel[esc]), rel[esc].max()))
    assert np.median(rel[esc]) < 1e-5
    assert rel[esc].max() < 1e-3


def _workload_loss_and_fd(precision):
    """Gradients of the celestial-angle loss w.r.t. (spin, inclination, yaw,
    pitch) through the adjoint, and the frozen-sequence central FD."""
    from blackhorizon_b200.adjoint import (angle_loss, celestial_angles, fly_camera_rays,
                                           replay, trace_rays_differentiable, trace_with_tape)
    from blackhorizon_b200.kerr import KerrSpacetime

    dev = torch.device("cuda", 0)
    s0_target, (u, v, yaw0, pitch0) = small_frame(spin=0.9)
    tgt_states, tgt_status, _, _ = trace_with_tape(KerrSpacetime(1.0, 0.9), s0_target, 100.0,
                                                   max_steps=10000, rtol=1e-9, capture_margin=0.01)
    th_t, ph_t = celestial_angles(torch.tensor(0.9, dtype=torch.float64, device=dev), tgt_states)
    params = [torch.tensor(x, dtype=torch.float64, device=dev, requires_grad=True)
              for x in (0.7, 60.0, yaw0, pitch0)]
    spin, inc, yaw, pitch = params
    s0 = fly_camera_rays(spin, inc, yaw, pitch, 50.0, u, v)
    states, status, steps = trace_rays_differentiable(
        spin, s0, 100.0, max_steps=10000, rtol=1e-9, capture_margin=0.01, precision=precision,
        checkpoint_every=64)
    mask = ((status == 2) & (tgt_status == 2)).to(torch.float64)
    th, ph = celestial_angles(spin, states)
    loss = angle_loss(th, ph, th_t, ph_t, mask)
    loss.backward()
    grads = np.array([float(p.grad) for p in params])
    # Frozen-sequence finite differences: rebuild the tape of this trace and
    # replay it with each parameter moved by +-h.
    _, _, _, tape = trace_with_tape(KerrSpacetime(1.0, 0.7), s0.detach(), 100.0,
                                    max_steps=10000, rtol=1e-9, capture_margin=0.01,
                                    precision="fp64", checkpoint_every=64)
    base = [0.7, 60.0, yaw0, pitch0]
    eps = 1e-6
    fd = []
    for k in range(4):
        vals = []
        for sgn in (1, -1):
            p = list(base)
            p[k] += sgn * eps
            pt = [torch.tensor(x, dtype=torch.float64, device=dev) for x in p]
            y0 = fly_camera_rays(pt[0], pt[1], pt[2], pt[3], 50.0, u, v)
            yN = replay(tape, y0, spin=p[0], precision="fp64")
            t, f = celestial_angles(pt[0], yN)
            vals.append(float(angle_loss(t, f, th_t, ph_t, mask)))
        fd.append((vals[0] - vals[1]) / (2 * eps))
    return grads, np.array(fd), float(loss.detach())


def test_workload_gradients_against_finite_differences_fp64(cuda):
    grads, fd, loss = _workload_loss_and_fd("fp64")
    rel = np.abs(grads - fd) / np.maximum(np.abs(fd), 1e-8)
    print("fp64 loss %.6g grads %s fd %s rel %s" % (loss, grads, fd, rel))
    assert loss > 0
    assert np.all(rel < 1e-4)


def test_workload_gradients_mixed_policy(cuda):
    """Mixed policy (float32 stages in the forward trace and the adjoint):
    gradients agree with the float64 finite differences to 1e-2."""
    grads, fd, loss = _workload_loss_and_fd("mixed")
    rel = np.abs(grads - fd) / np.maximum(np.abs(fd), 1e-8)
    print("mixed loss %.6g grads %s fd %s rel %s" % (loss, grads, fd, rel))
    assert np.all(rel < 1e-2)


def test_ray_order_does_not_change_results(cuda):
    """The sweep's thread order (sorted by accepted steps, or identity) only
    schedules the rays: results are bit-identical."""
    from blackhorizon_b200.adjoint import adjoint, trace_with_tape
    from blackhorizon_b200.kerr import KerrSpacetime

    s0, _ = small_frame()
    _, status, _, tape = trace_with_tape(KerrSpacetime(1.0, 0.7), s0, 100.0, max_steps=5000,
                                         rtol=1e-9, capture_margin=0.01, checkpoint_every=16)
    rng = np.random.default_rng(3)
    g = torch.as_tensor(rng.normal(size=(s0.shape[0], 8)), device="cuda") * (status == 2)[:, None]
    for prec in ("fp64", "mixed"):
        a0, as0 = adjoint(tape, g, precision=prec, sort=False)
        a1, as1 = adjoint(tape, g, precision=prec, sort=True)
        assert torch.equal(a0, a1) and torch.equal(as0, as1)
