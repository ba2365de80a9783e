"""The analytic shadow-edge oracle (oracle/bardeen.py) on the CPU: the
critical curve is a double root of the radial potential, reproduces the
reference's equatorial critical impact parameters (tests/test_shadow.py:
96-106: 2.8444 M prograde, 6.8323 M retrograde at a = 0.9), classifies
photons as the quartic's roots do, and the photon constants of Kerr-Schild
states are conserved along oracle trajectories."""

import numpy as np
import pytest

from oracle import bardeen


def radial_potential(a, xi, eta, r, m=1.0):
    delta = r * r - 2.0 * m * r + a * a
    return (r * r + a * a - a * xi) ** 2 - delta * (eta + (xi - a) ** 2)


@pytest.mark.parametrize("a", [0.3, 0.9, -0.7, 0.998])
def test_critical_curve_is_a_double_root(a):
    r_pro, r_ret = bardeen.equatorial_photon_orbits(abs(a))
    r = np.linspace(r_pro, r_ret, 101)[1:-1]
    xi, eta = bardeen.critical_curve(a, r)
    assert np.all(eta > 0)
    scale = (r * r) ** 2
    assert np.max(np.abs(radial_potential(a, xi, eta, r)) / scale) < 1e-12
    dr = 1e-6
    deriv = (radial_potential(a, xi, eta, r + dr) - radial_potential(a, xi, eta, r - dr)) / (2 * dr)
    assert np.max(np.abs(deriv) / (r * r * r)) < 1e-7


def test_equatorial_values_of_the_reference():
    r_pro, r_ret = bardeen.equatorial_photon_orbits(0.9)
    xi_pro = bardeen.critical_curve(0.9, r_pro)[0]
    xi_ret = bardeen.critical_curve(0.9, r_ret)[0]
    assert abs(xi_pro - 2.8444) < 1e-4
    assert abs(abs(xi_ret) - 6.8323) < 1e-4
    assert abs(bardeen.critical_curve(0.9, r_pro)[1]) < 1e-9
    # Small spin: the curve shrinks to the circle xi^2 + eta = 27 M^2.
    r = np.linspace(*bardeen.equatorial_photon_orbits(1e-4), 9)[1:-1]
    xi, eta = bardeen.critical_curve(1e-4, r)
    np.testing.assert_allclose(xi * xi + eta, 27.0, rtol=1e-3)


@pytest.mark.parametrize("a", [0.9, -0.6])
def test_curve_and_quartic_classify_alike(a):
    rng = np.random.default_rng(3)
    xi = rng.uniform(-9, 9, 4000)
    eta = rng.uniform(0, 40, 4000)
    by_curve = bardeen.captured_by_curve(a, xi, eta)
    by_roots = bardeen.captured_by_potential(a, xi, eta, 1e4)
    assert 0.1 < by_curve.mean() < 0.9
    np.testing.assert_array_equal(by_curve, by_roots)


def test_photon_constants_are_conserved(oracle):
    """xi and eta of states from the oracle's null momentum stay constant
    along oracle trajectories (float64, rtol 1e-12)."""
    rng = np.random.default_rng(5)
    a = 0.9
    n = 64
    u = rng.normal(size=(n, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    pos = 20.0 * u
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    s0 = np.zeros((n, 8))
    s0[:, 1:4] = pos
    s0[:, 4:8] = oracle.null_momentum(1.0, a, pos, d, True, True)
    xi0, eta0 = bardeen.photon_constants(a, s0)
    s1, _ = oracle.propagate_to(1.0, a, s0, np.full(n, 15.0), rtol=1e-12, atol=1e-14)
    r1 = np.sqrt(np.sum(s1[:, 1:4] ** 2, axis=1))
    ok = r1 > 3.0  # not fallen through the horizon
    xi1, eta1 = bardeen.photon_constants(a, s1)
    assert ok.sum() > n // 2
    np.testing.assert_allclose(xi1[ok], xi0[ok], rtol=1e-9, atol=1e-9)
    np.testing.assert_allclose(eta1[ok], eta0[ok], rtol=1e-8, atol=1e-8)


def test_reference_full_hd_frame_edges_on_the_curve(oracle):
    """The reference's own 1920x1080 statuses (a = 0.9, inclination 80 deg,
    fov 25, rtol 1e-9; tests/golden/trace_c3_status.npz) have their capture
    boundary on the critical curve: every checked edge within two pixels and
    0.5 % in impact parameter.  This pins the analytic check that the GPU
    frames are held to."""
    from conftest import golden

    from blackhorizon_b200.camera import PinholeCamera
    from blackhorizon_b200.workloads import SHADOW_FULL_HD as C

    cam = PinholeCamera.from_orbit(C.distance, C.inclination, fov_degrees=C.fov,
                                   width=C.width, height=C.height)
    checks = bardeen.frame_edges_against_curve(cam, C.spin, golden("trace_c3_status.npz")["status"])
    assert len(checks) == 16
    for c in checks:
        assert abs(c["traced"] - c["analytic"]) <= 2.0, c
        assert c["relative"] <= 5e-3, c
    print("worst", max(c["relative"] for c in checks), max(abs(c["traced"] - c["analytic"]) for c in checks))
