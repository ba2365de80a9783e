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


def _c5_setup(precision, pixels_require_grad=False):
    """The 256x256 differentiable-tracing workload (a = 0.7, inclination 60
    deg, r_obs = 50 M, fov 30, rtol 1e-9, checkpoint every 64 accepted
    steps): loss of the escaped rays' celestial angles against a target frame
    at a = 0.9.  Returns the adjoint's gradients, a function evaluating the
    loss through the frozen float64 step sequence at moved parameters or
    pixel coordinates, and the pixel tensors."""
    from blackhorizon_b200.adjoint import (angle_loss, celestial_angles, fly_camera_rays,
                                           orbit_look_at, pixel_grid, replay,
                                           trace_rays_differentiable, trace_with_tape)
    from blackhorizon_b200.kerr import KerrSpacetime
    from blackhorizon_b200.workloads import DIFFERENTIABLE as C

    dev = torch.device("cuda", 0)
    t = lambda x, g=False: torch.tensor(x, dtype=torch.float64, device=dev,  # noqa: E731
                                        requires_grad=g)
    yaw0, pitch0 = orbit_look_at(C.distance, C.inclination)
    u, v = pixel_grid(C.width, C.height, C.fov, dev)
    kw = dict(max_steps=C.max_steps, rtol=C.rtol, atol=C.atol, capture_margin=C.capture_margin)
    y_tgt = fly_camera_rays(t(0.9), t(C.inclination), t(yaw0), t(pitch0), C.distance, u, v)
    tgt, tgt_status, _, _ = trace_with_tape(KerrSpacetime(1.0, 0.9), y_tgt, C.escape_radius,
                                            **kw)
    th_t, ph_t = celestial_angles(t(0.9), tgt)
    params = [t(x, True) for x in (C.spin, C.inclination, yaw0, pitch0)]
    uu = u.clone().requires_grad_(pixels_require_grad)
    vv = v.clone().requires_grad_(pixels_require_grad)
    s0 = fly_camera_rays(*params, C.distance, uu, vv)
    states, status, _ = trace_rays_differentiable(params[0], s0, C.escape_radius,
                                                  precision=precision, checkpoint_every=64,
                                                  **kw)
    mask = ((status == 2) & (tgt_status == 2)).to(torch.float64)
    th, ph = celestial_angles(params[0], states)
    angle_loss(th, ph, th_t, ph_t, mask).backward()
    _, _, _, tape = trace_with_tape(KerrSpacetime(1.0, C.spin), s0.detach(), C.escape_radius,
                                    precision="fp64", checkpoint_every=64, **kw)

    def frozen_loss(p, du=None, dv=None, ray=None):
        # ray: only that ray's term of the loss (a single pixel moves the
        # total, of order 10^3, by ~1e-9: its difference would be rounding).
        pt = [t(x) for x in p]
        y0 = fly_camera_rays(*pt, C.distance, u if du is None else u + du,
                             v if dv is None else v + dv)
        yN = replay(tape, y0, spin=p[0], precision="fp64")
        a_, b_ = celestial_angles(pt[0], yN)
        if ray is not None:
            sl = slice(ray, ray + 1)
            return float(angle_loss(a_[sl], b_[sl], th_t[sl], ph_t[sl], mask[sl]))
        return float(angle_loss(a_, b_, th_t, ph_t, mask))

    grads = np.array([float(p.grad) for p in params])
    base = [C.spin, C.inclination, yaw0, pitch0]
    return grads, base, frozen_loss, (uu, vv, mask)


def _central(f, base, k, h):
    p, m = list(base), list(base)
    p[k] += h
    m[k] -= h
    return (f(p) - f(m)) / (2.0 * h)


def test_c5_gradients_against_finite_differences(cuda):
    """fp64 adjoint gradients of the 256x256 workload with respect to spin,
    inclination, yaw and pitch against central differences of the frozen
    step sequence at h = 1e-6 and 1e-7 and their Richardson combination
    (100 D(1e-7) - D(1e-6)) / 99, which removes the h^2 truncation term.
    Per parameter: the Richardson estimate within 1e-5 relative, the plain
    differences within 1e-4 at h = 1e-7 and 1e-2 at h = 1e-6 (the loss is
    steep near the shadow edge, where the truncation term is large).  The
    mixed policy's gradients (its own float32 trace and sweep) agree with
    the fp64 Richardson estimate within 1e-2."""
    grads, base, f, _ = _c5_setup("fp64")
    names = ("spin", "inclination", "yaw", "pitch")
    report = {}
    for k, name in enumerate(names):
        d6 = _central(f, base, k, 1e-6)
        d7 = _central(f, base, k, 1e-7)
        rich = (100.0 * d7 - d6) / 99.0
        rel = [abs(grads[k] - d) / abs(d) for d in (d6, d7, rich)]
        report[name] = (grads[k], d6, d7, rich, rel)
        assert rel[2] <= 1e-5, (name, report[name])
        assert rel[1] <= 1e-4, (name, report[name])
        assert rel[0] <= 1e-2, (name, report[name])
    print("fp64 adjoint vs FD (h=1e-6, 1e-7, Richardson):",
          {k: ["%.2e" % r for r in v[4]] for k, v in report.items()})
    mixed, _, _, _ = _c5_setup("mixed")
    rich = np.array([report[n][3] for n in names])
    rel_m = np.abs(mixed - rich) / np.abs(rich)
    print("mixed adjoint vs fp64 Richardson:", dict(zip(names, ["%.2e" % r for r in rel_m])))
    assert np.all(rel_m <= 1e-2)


def test_c5_pixel_coordinate_gradients(cuda):
    """Gradients with respect to the image-plane coordinates (u, v) of single
    pixels (the pinhole grid of camera.py:96-113, through the yaw/pitch
    camera of fly_camera.py:37-88): the adjoint's dL/du_i and dL/dv_i of 12
    escaped pixels against Richardson-combined central differences of the
    frozen sequence (h = 1e-6, 1e-7) of that pixel's own term of the loss
    (only it depends on the pixel's coordinates), within 1e-5 relative (1e-9
    absolute for pixels whose gradient is near zero)."""
    grads, base, f, (uu, vv, mask) = _c5_setup("fp64", pixels_require_grad=True)
    gu, gv = uu.grad.cpu().numpy(), vv.grad.cpu().numpy()
    esc = np.nonzero(mask.cpu().numpy() > 0)[0]
    rng = np.random.default_rng(9)
    pick = rng.choice(esc, 12, replace=False)
    n = uu.shape[0]
    checked = 0
    for i in pick:
        for g, which in ((gu, "u"), (gv, "v")):
            d = []
            for h in (1e-6, 1e-7):
                e = torch.zeros(n, dtype=torch.float64, device=uu.device)
                e[i] = h
                if which == "u":
                    d.append((f(base, du=e, ray=i) - f(base, du=-e, ray=i)) / (2 * h))
                else:
                    d.append((f(base, dv=e, ray=i) - f(base, dv=-e, ray=i)) / (2 * h))
            rich = (100.0 * d[1] - d[0]) / 99.0
            err = abs(g[i] - rich)
            assert err <= max(1e-5 * abs(rich), 1e-9), (i, which, g[i], d, rich)
            checked += 1
    assert checked == 24


def test_tape_grows_when_a_ray_outruns_it(cuda, monkeypatch):
    """Without a capacity the tape starts short and the trace runs again with
    room for max_steps when a ray overflows it: the result equals a trace
    with the full capacity from the start."""
    from blackhorizon_b200 import adjoint as adj
    from blackhorizon_b200.kerr import KerrSpacetime

    st = KerrSpacetime(1.0, 0.7)
    s0, _ = small_frame()
    kw = dict(max_steps=5000, rtol=1e-9, capture_margin=0.01, checkpoint_every=16)
    full = adj.trace_with_tape(st, s0, 100.0, capacity=5000, **kw)
    monkeypatch.setattr(adj, "FIRST_TAPE_CAPACITY", 8)
    grown = adj.trace_with_tape(st, s0, 100.0, **kw)
    assert int(full[2].max()) > 8 and grown[3].capacity == 5000
    assert torch.equal(full[0], grown[0]) and torch.equal(full[2], grown[2])
    g = torch.ones_like(s0) * (full[1] == 2)[:, None]
    a, b = adj.adjoint(full[3], g), adj.adjoint(grown[3], g)
    assert torch.equal(a[0], b[0]) and torch.equal(a[1], b[1])
