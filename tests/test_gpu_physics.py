"""Physics anchors of the reference's tests run through the b200 backend.

Shadow edges: the capture/escape boundary of an equatorial fan of photons
from a distant camera (reference tests/test_shadow.py:22-132) must sit at the
critical impact parameter: 3 sqrt(3) M for a = 0 and Bardeen's equatorial
values (about 2.84 M prograde and 6.83 M retrograde) for a = 0.9, within
0.5 %, in both precision policies.

Conservation and orbits (reference tests/test_orbits.py:22-136): photon
flyby (E, L_z, H), timelike H = -1/2, the r = 3M photon sphere and the r = 6M
circular orbit, integrated by the b200 integrate_dense in float64 with the
reference's tolerances.  The tracer's own conservation on the 160x120 frame
is checked for both policies.
"""

import math

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

DISTANCE = 1000.0


def equatorial_fan(spacetime, offsets, precision, rtol):
    """Photons from (D, 0, 0) with direction (-1, offset, 0): per-ray status
    and the impact parameter b = L_z / E of the initial state."""
    from blackhorizon_b200 import build_state, conserved_quantities, null_momentum_from_velocity
    from blackhorizon_b200 import trace_rays

    n = offsets.shape[0]
    pos = np.tile(np.array([[DISTANCE, 0.0, 0.0]]), (n, 1))
    d = np.stack([-np.ones(n), offsets, np.zeros(n)], axis=-1)
    d /= np.linalg.norm(d, axis=-1, keepdims=True)
    mom = null_momentum_from_velocity(spacetime, pos, d, time_orientation="past")
    s0 = build_state(pos, mom)
    res = trace_rays(spacetime, s0, escape_radius=1.2 * DISTANCE, max_steps=60000,
                     rtol=rtol, atol=rtol * 1e-3, max_step=5.0, precision=precision)
    energy, l_z = conserved_quantities(s0)
    return np.asarray(res.status), l_z / energy


def capture_boundary(spacetime, lo, hi, precision, rtol, rounds=3, fan=48):
    """Bracket the boundary between the largest captured and the smallest
    escaped |offset| and refine; returns |b| at the boundary."""
    b = None
    for _ in range(rounds):
        offsets = np.linspace(lo, hi, fan)
        status, impact = equatorial_fan(spacetime, offsets, precision, rtol)
        captured, escaped = status == 1, status == 2
        assert captured.any() and escaped.any() and (captured | escaped).all()
        mag = np.abs(offsets)
        i_cap = int(np.argmax(np.where(captured, mag, -1.0)))
        i_esc = int(np.argmin(np.where(escaped & (mag > mag[i_cap]), mag, np.inf)))
        lo, hi = float(offsets[i_cap]), float(offsets[i_esc])
        b = 0.5 * float(abs(impact[i_cap]) + abs(impact[i_esc]))
    return b


def bardeen_equatorial(spacetime, prograde):
    """|xi| of the equatorial circular photon orbit (Bardeen 1973):
    xi = (r^2 (r - 3M) + a^2 (r + M)) / (a (M - r)) at the photon-orbit
    radius."""
    m, a = spacetime.mass, spacetime.spin
    r = spacetime.photon_orbit_radius(prograde=prograde)
    return abs((r * r * (r - 3.0 * m) + a * a * (r + m)) / (a * (m - r)))


# The reference's fan settings use rtol 1e-10; the mixed policy runs at its
# own working tolerance 1e-8 (float32 stage arithmetic cannot resolve 1e-10).
POLICIES = [("fp64", 1e-10), ("mixed", 1e-8)]


@pytest.mark.parametrize("precision,rtol", POLICIES)
def test_schwarzschild_critical_impact_parameter(cuda, precision, rtol):
    from blackhorizon_b200.kerr import KerrSpacetime

    b = capture_boundary(KerrSpacetime(spin=0.0), 4.5e-3, 6.5e-3, precision, rtol)
    err = abs(b - 3.0 * math.sqrt(3.0)) / (3.0 * math.sqrt(3.0))
    print(f"{precision}: a=0 boundary b={b:.5f}, relative error {err:.2e}")
    assert err < 5e-3


@pytest.mark.parametrize("precision,rtol", POLICIES)
def test_kerr_prograde_retrograde_edges(cuda, precision, rtol):
    from blackhorizon_b200.kerr import KerrSpacetime

    st = KerrSpacetime(spin=0.9)
    pro, ret = bardeen_equatorial(st, True), bardeen_equatorial(st, False)
    b_pro = capture_boundary(st, -4.0e-3, -2.0e-3, precision, rtol)
    b_ret = capture_boundary(st, 5.5e-3, 8.0e-3, precision, rtol)
    print(f"{precision}: a=0.9 prograde b={b_pro:.5f} (Bardeen {pro:.5f}, "
          f"{abs(b_pro - pro) / pro:.2e}), retrograde b={b_ret:.5f} (Bardeen {ret:.5f}, "
          f"{abs(b_ret - ret) / ret:.2e})")
    assert abs(b_pro - pro) / pro < 5e-3
    assert abs(b_ret - ret) / ret < 5e-3
    assert b_pro < b_ret


@pytest.mark.parametrize("precision,rtol", POLICIES)
def test_zero_spin_symmetry(cuda, precision, rtol):
    from blackhorizon_b200.kerr import KerrSpacetime

    st = KerrSpacetime(spin=0.0)
    b_plus = capture_boundary(st, 4.5e-3, 6.5e-3, precision, rtol, rounds=2)
    b_minus = capture_boundary(st, -6.5e-3, -4.5e-3, precision, rtol, rounds=2)
    assert abs(b_plus - b_minus) / b_plus < 1e-3


def _dense(st, state0, lam, rtol):
    from blackhorizon_b200 import GeodesicRhs, integrate_dense

    states = integrate_dense(GeodesicRhs(st), state0, lambda_total=lam, rtol=rtol)
    return np.concatenate([np.asarray(s) for s in states], axis=0)


def test_photon_flyby_conservation(cuda):
    """Reference tests/test_orbits.py:22-45."""
    from blackhorizon_b200 import (build_state, conserved_quantities, hamiltonian,
                                   null_momentum_from_velocity)
    from blackhorizon_b200.kerr import KerrSpacetime

    st = KerrSpacetime(spin=0.9)
    pos = np.array([[30.0, 4.0, 1.5]])
    mom = null_momentum_from_velocity(st, pos, np.array([[-1.0, 0.0, 0.0]]),
                                      time_orientation="future")
    traj = _dense(st, build_state(pos, mom), 70.0, 1e-11)
    energy, l_z = conserved_quantities(traj)
    ham = hamiltonian(st, traj)
    np.testing.assert_allclose(energy, energy[0], rtol=1e-12)
    np.testing.assert_allclose(l_z, l_z[0], rtol=1e-8)
    np.testing.assert_allclose(ham, 0.0, atol=1e-9)
    r = st.kerr_schild_radius(traj[:, 1], traj[:, 2], traj[:, 3])
    assert float(r.min()) < 6.0


def test_timelike_normalisation_and_circular_orbit(cuda):
    """Reference tests/test_orbits.py:48-64 and 108-136."""
    from blackhorizon_b200 import (build_state, conserved_quantities, hamiltonian,
                                   timelike_momentum)
    from blackhorizon_b200.kerr import KerrSpacetime

    st = KerrSpacetime(spin=0.9)
    r_orbit = 6.0
    assert r_orbit > st.isco_radius(prograde=True)
    omega = 1.0 / (r_orbit ** 1.5 + st.spin)
    pos = np.array([[r_orbit, st.spin, 0.0]])
    vel = np.array([[-omega * st.spin, omega * r_orbit, 0.0]])
    s0 = build_state(pos, timelike_momentum(st, pos, vel))
    traj = _dense(st, s0, 120.0, 1e-11)
    np.testing.assert_allclose(hamiltonian(st, traj), -0.5, rtol=1e-9)
    traj = _dense(st, s0, 170.0, 1e-11)
    r = st.kerr_schild_radius(traj[:, 1], traj[:, 2], traj[:, 3])
    np.testing.assert_allclose(r, r_orbit, rtol=1e-6)
    assert np.allclose(traj[:, 3], 0.0, atol=1e-8)
    energy, l_z = conserved_quantities(traj)
    np.testing.assert_allclose(energy, energy[0], rtol=1e-12)
    np.testing.assert_allclose(l_z, l_z[0], rtol=1e-10)


def test_photon_sphere(cuda):
    """Reference tests/test_orbits.py:68-104."""
    from blackhorizon_b200 import build_state, conserved_quantities, null_momentum_from_velocity
    from blackhorizon_b200.kerr import KerrSpacetime

    st = KerrSpacetime(spin=0.0)
    pos = np.array([[3.0, 0.0, 0.0]])
    mom = null_momentum_from_velocity(st, pos, np.array([[0.0, 1.0, 0.0]]),
                                      time_orientation="future")
    s0 = build_state(pos, mom)
    energy, l_z = conserved_quantities(s0)
    np.testing.assert_allclose(float(l_z[0] / energy[0]), 3.0 * math.sqrt(3.0), rtol=1e-12)
    traj = _dense(st, s0, 16.0, 1e-12)
    r = st.kerr_schild_radius(traj[:, 1], traj[:, 2], traj[:, 3])
    np.testing.assert_allclose(r, 3.0, atol=1e-6)
    phi = np.unwrap(np.arctan2(traj[:, 2], traj[:, 1]))
    assert abs(phi[-1] - phi[0]) > 2.5 * math.pi


@pytest.mark.parametrize("precision,h_tol,lz_tol", [("fp64", 1e-6, 1e-7), ("mixed", 1e-4, 1e-5)])
def test_tracer_conservation_small_frame(cuda, precision, h_tol, lz_tol):
    """160x120 frame (a=0.9, 60 deg, rtol 1e-8): p_t is conserved exactly, and
    escaped rays keep the null constraint and L_z (the float64 reference
    keeps |H| <= 2.3e-7 and |dL_z| <= 5.5e-8 on this frame)."""
    from blackhorizon_b200 import conserved_quantities, hamiltonian, trace_rays
    from blackhorizon_b200.camera import PinholeCamera
    from blackhorizon_b200.kerr import KerrSpacetime

    st = KerrSpacetime(1.0, 0.9)
    cam = PinholeCamera.from_orbit(50.0, 60.0, fov_degrees=30.0, width=160, height=120)
    s0 = cam.initial_states(st)
    res = trace_rays(st, s0, 100.0, max_steps=5000, rtol=1e-8, atol=1e-10,
                     capture_margin=0.01, precision=precision)
    esc = res.status == 2
    assert torch.equal(res.states[:, 4], s0[:, 4])
    ham = hamiltonian(st, res.states)[esc]
    _, lz0 = conserved_quantities(s0)
    _, lz = conserved_quantities(res.states)
    assert float(ham.abs().max()) <= h_tol
    assert float((lz - lz0)[esc].abs().max()) <= lz_tol



@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_full_hd_frame_edges_on_the_critical_curve(cuda, precision):
    """The 1920x1080 frame (a = 0.9, inclination 80 deg, fov 25, rtol 1e-9):
    along seven rows across the shadow (heights -0.85 .. 0.85 of its half
    height) and down the column through its middle, the traced capture
    boundary lies where the photons' constants cross the general critical
    curve of spherical photon orbits (Bardeen 1973): the impact parameter
    sqrt(eta + xi^2) at the traced edge (midway between the last captured and
    the first escaped pixel) is within 0.5 % of the analytic edge's, and the
    two edges are within two pixels.  The prograde and retrograde edges are
    the two ends of the middle row."""
    from blackhorizon_b200 import trace_rays
    from blackhorizon_b200.camera import PinholeCamera
    from blackhorizon_b200.kerr import KerrSpacetime
    from blackhorizon_b200.workloads import SHADOW_FULL_HD as C

    st = KerrSpacetime(1.0, C.spin)
    cam = PinholeCamera.from_orbit(C.distance, C.inclination, fov_degrees=C.fov,
                                   width=C.width, height=C.height)
    res = trace_rays(st, cam.initial_states(st), C.escape_radius, max_steps=C.max_steps,
                     rtol=C.rtol, atol=C.atol, capture_margin=C.capture_margin,
                     precision=precision)
    from oracle import bardeen

    checks = bardeen.frame_edges_against_curve(cam, C.spin, res.status.cpu().numpy())
    worst = max(c["relative"] for c in checks)
    print(f"{precision}: {len(checks)} edges, worst impact-parameter difference {worst:.2e}")
    for c in checks:
        assert abs(c["traced"] - c["analytic"]) <= 2.0, c
        assert c["relative"] <= 5e-3, c
