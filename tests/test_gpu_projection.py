"""Float64 projection onto the null constraint (off by default).

The reference never projects: its tracer lets the super-Hamiltonian drift
with the integration error.  With ``project_every`` K > 0 the kernels move
every ray back onto H = 0 every K controller iterations (one float64 Newton
step on the spatial momentum).  Checks: H stays at float64 rounding where
the unprojected mixed trace drifts; the energy p_t is untouched;
classification still agrees with the reference's golden frame; endpoint
errors at equal affine parameter are no worse than without projection.
"""

import numpy as np
import pytest
import torch

from conftest import golden

pytestmark = pytest.mark.gpu


def _frame():
    from blackhorizon_b200.camera import PinholeCamera
    from blackhorizon_b200.kerr import KerrSpacetime
    from blackhorizon_b200.workloads import SHADOW_SMALL as C

    st = KerrSpacetime(1.0, C.spin)
    cam = PinholeCamera.from_orbit(C.distance, C.inclination, fov_degrees=C.fov,
                                   width=C.width, height=C.height)
    return C, st, cam.initial_states(st)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_projection_holds_the_null_constraint(cuda, precision):
    from blackhorizon_b200 import hamiltonian, trace_rays

    C, st, s0 = _frame()
    kw = dict(max_steps=C.max_steps, rtol=C.rtol, atol=C.atol, capture_margin=C.capture_margin,
              precision=precision)
    plain = trace_rays(st, s0, C.escape_radius, **kw)
    proj = trace_rays(st, s0, C.escape_radius, project_every=1, **kw)
    h_plain = hamiltonian(st, plain.states).abs()
    h_proj = hamiltonian(st, proj.states).abs()
    esc = proj.status == 2
    print(f"{precision}: max |H| escaped plain {float(h_plain[plain.status == 2].max()):.3g} "
          f"projected {float(h_proj[esc].max()):.3g}")
    assert float(h_proj[esc].max()) < 1e-14
    assert float(h_proj[esc].max()) < float(h_plain[plain.status == 2].max())
    # The energy is never touched.
    assert torch.equal(proj.states[:, 4], s0[:, 4].to(proj.states.device))
    ref = golden("trace_c1_160x120.npz")["status"].astype(np.int32)
    agree = float(np.mean(proj.status.cpu().numpy() == ref))
    print(f"{precision}: projected status agreement with the reference {agree:.5f}")
    assert agree >= 0.995


def test_projection_periods(cuda):
    """Any period: returned states lie on the constraint (they are projected
    when the ray finishes) and the classification does not move."""
    from blackhorizon_b200 import hamiltonian, trace_rays

    C, st, s0 = _frame()
    kw = dict(max_steps=C.max_steps, rtol=C.rtol, atol=C.atol, capture_margin=C.capture_margin,
              precision="mixed")
    base = trace_rays(st, s0, C.escape_radius, project_every=1, **kw)
    for k in (16, 4):
        r = trace_rays(st, s0, C.escape_radius, project_every=k, **kw)
        worst = float(hamiltonian(st, r.states)[r.status == 2].abs().max())
        agree = float((r.status == base.status).double().mean())
        print(f"K={k}: max |H| {worst:.3g}, status agreement with K=1 {agree:.5f}")
        assert worst < 1e-13
        assert agree >= 0.995


def test_projected_endpoints_against_oracle(cuda, oracle):
    """Raw-throughput rays (per-ray spin), 400 attempted steps: endpoint error
    at equal affine parameter against the oracle (rtol 1e-12), with and
    without projection."""
    from blackhorizon_b200 import propagate
    from blackhorizon_b200.geodesics import build_state, null_momentum_from_velocity
    from blackhorizon_b200.kerr import KerrSpacetime
    from blackhorizon_b200.workloads import PLUNGE_RADIUS, ks_radius_np, raw_throughput_inputs

    n = 2048
    pos, d, spin = raw_throughput_inputs(n)
    st = object.__new__(KerrSpacetime)
    st.mass, st.spin = 1.0, spin
    pos_t = torch.as_tensor(pos, device="cuda")
    s0 = build_state(pos_t, null_momentum_from_velocity(
        st, pos_t, torch.as_tensor(d, device="cuda"), "past"))
    s0n = s0.cpu().numpy()
    spins = torch.as_tensor(spin, device="cuda")
    med = {}
    # Projection runs without the float64 band, so the mixed reference point
    # is the float32-stage path (f64_radius = 0).
    for name, prec, k in (("mixed", "mixed", 0), ("mixed_projected", "mixed", 1),
                          ("fp64_projected", "fp64", 1)):
        states, _, lam, _, _ = propagate(KerrSpacetime(1.0, 0.0), s0, 400, 1e-8, 1e-10,
                                         precision=prec, spins=spins, project_every=k,
                                         f64_radius=0.0)
        truth, _ = oracle.propagate_to(1.0, spin, s0n, lam.cpu().numpy(), rtol=1e-12,
                                       atol=1e-14)
        got = states.cpu().numpy()
        ok = np.all(np.isfinite(truth), axis=1) & np.all(np.isfinite(got), axis=1)
        ok &= np.nan_to_num(ks_radius_np(truth, spin), nan=0.0) >= PLUNGE_RADIUS
        rel = np.max(np.abs(got[ok] - truth[ok]) / np.maximum(np.abs(truth[ok]), 1.0), axis=1)
        med[name] = (float(np.median(rel)), float(np.quantile(rel, 0.99)))
    print("endpoint error (median, p99):", med)
    assert med["mixed_projected"][0] <= 2.0 * med["mixed"][0]
    assert med["mixed_projected"][1] <= 1e-5
    assert med["fp64_projected"][0] <= 1e-8
