"""Analytic shadow edge of a Kerr black hole: test infrastructure only.

The capture/escape boundary of photons is the set of spherical photon orbits
(Bardeen 1973, "Timelike and null geodesics in the Kerr metric", in Black
Holes, Les Houches).  The reference implements only the equatorial critical
impact parameter (tests/test_shadow.py:96-106); this module restates the
general curve, derived here from the photon's radial potential in
Boyer-Lindquist form (units of the photon energy E, M the mass, a the spin):

    R(r) = (r^2 + a^2 - a xi)^2 - Delta (eta + (xi - a)^2),
    Delta = r^2 - 2 M r + a^2,  xi = L_z / E,  eta = Q / E^2.

A spherical orbit at radius r is a double root, R(r) = R'(r) = 0, which
solved for (xi, eta) gives

    xi_c(r)  = (r^2 (3M - r) - a^2 (r + M)) / (a (r - M)),
    eta_c(r) = r^3 (4 a^2 M - r (r - 3M)^2) / (a^2 (r - M)^2),

for r between the prograde and retrograde equatorial photon orbits, where
eta_c = 0 (r (r - 3M)^2 = 4 a^2 M).  A photon arriving from outside is
captured when its xi lies in the curve's range and eta < eta_c(r*) with
xi_c(r*) = xi; otherwise it has a radial turning point and escapes.  The
same classification follows from the real roots of the quartic R(r) (no
root between the horizon and the photon's radius: captured), which the
tests use to check the curve.

The constants of a Kerr-Schild Cartesian state (t, x, y, z, p_t, p_x, p_y,
p_z): E = -p_t, L_z = x p_y - y p_x (the axial Killing vector is the same
in both charts), and Carter's Q = p_theta^2 + cos^2 theta (L_z^2 / sin^2 theta
- a^2 E^2) with p_theta = cot theta (x p_x + y p_y) - r sin theta p_z, from
x + i y = (r + i a) e^{i phi} sin theta, z = r cos theta (theta and p_theta
coincide in the two charts, whose t and phi differ by functions of r only).
Past-directed states give the same xi and eta (both L_z and E change sign).
"""

from __future__ import annotations

import numpy as np


def critical_curve(a: float, r, mass: float = 1.0):
    """(xi_c, eta_c) of the spherical photon orbit at Boyer-Lindquist radius
    r (array), spin a != 0."""
    r = np.asarray(r, dtype=np.float64)
    m = mass
    xi = (r * r * (3.0 * m - r) - a * a * (r + m)) / (a * (r - m))
    eta = r ** 3 * (4.0 * a * a * m - r * (r - 3.0 * m) ** 2) / (a * a * (r - m) ** 2)
    return xi, eta


def equatorial_photon_orbits(a: float, mass: float = 1.0):
    """(prograde, retrograde) equatorial circular photon orbit radii: the
    roots of r (r - 3M)^2 = 4 a^2 M in [M, 4M] (eta_c = 0)."""
    m = mass

    def g(r):
        return r * (r - 3.0 * m) ** 2 - 4.0 * a * a * m

    def root(lo, hi):
        for _ in range(200):
            mid = 0.5 * (lo + hi)
            if (g(lo) > 0) == (g(mid) > 0):
                lo = mid
            else:
                hi = mid
        return 0.5 * (lo + hi)

    # g(M) = 4M^3 - 4a^2 M >= 0, g(3M) = -4 a^2 M < 0, g(4M) = 4M^3 - 4a^2 M >= 0.
    return root(m, 3.0 * m), root(3.0 * m, 4.0 * m)


def photon_constants(a: float, states):
    """(xi, eta) of (n, 8) Kerr-Schild Cartesian photon states."""
    s = np.asarray(states, dtype=np.float64)
    x, y, z = s[:, 1], s[:, 2], s[:, 3]
    pt, px, py, pz = s[:, 4], s[:, 5], s[:, 6], s[:, 7]
    a2 = a * a
    q = x * x + y * y + z * z - a2
    r2 = 0.5 * (q + np.sqrt(q * q + 4.0 * a2 * z * z))
    r = np.sqrt(r2)
    cos_t = z / r
    sin2 = 1.0 - cos_t * cos_t
    sin_t = np.sqrt(sin2)
    energy = -pt
    l_z = x * py - y * px
    p_theta = (cos_t / sin_t) * (x * px + y * py) - r * sin_t * pz
    carter = p_theta ** 2 + cos_t ** 2 * (l_z ** 2 / sin2 - a2 * energy ** 2)
    return l_z / energy, carter / energy ** 2


def captured_by_curve(a: float, xi, eta, mass: float = 1.0):
    """Capture of photons arriving from outside the photon region, from the
    critical curve: xi inside the curve's range and eta below eta_c there."""
    xi = np.atleast_1d(np.asarray(xi, dtype=np.float64))
    eta = np.atleast_1d(np.asarray(eta, dtype=np.float64))
    r_pro, r_ret = equatorial_photon_orbits(a, mass)
    # xi_c decreases monotonically from xi_c(r_pro) to xi_c(r_ret) (a > 0;
    # for a < 0 the curve mirrors, xi -> -xi).
    sgn = 1.0 if a > 0 else -1.0
    aa = abs(a)
    xs = sgn * xi
    lo, hi = np.full(xs.shape, r_pro), np.full(xs.shape, r_ret)
    xi_hi = critical_curve(aa, r_pro, mass)[0]
    xi_lo = critical_curve(aa, r_ret, mass)[0]
    inside = (xs <= xi_hi) & (xs >= xi_lo)
    for _ in range(80):
        mid = 0.5 * (lo + hi)
        above = critical_curve(aa, mid, mass)[0] > xs
        lo = np.where(above, mid, lo)
        hi = np.where(above, hi, mid)
    eta_c = critical_curve(aa, 0.5 * (lo + hi), mass)[1]
    return inside & (eta < eta_c)


def captured_by_potential(a: float, xi, eta, r_from, mass: float = 1.0):
    """Capture of inward photons starting at radius r_from: no real root of
    the quartic R(r) between the outer horizon and r_from."""
    m = mass
    r_plus = m + np.sqrt(m * m - a * a)
    out = []
    for x, e, r0 in zip(np.atleast_1d(xi), np.atleast_1d(eta),
                        np.broadcast_to(r_from, np.shape(np.atleast_1d(xi)))):
        aa = a * a - a * x
        k = e + (x - a) ** 2
        roots = np.roots([1.0, 0.0, 2.0 * aa - k, 2.0 * m * k, aa * aa - a * a * k])
        real = roots[np.abs(roots.imag) <= 1e-9 * np.maximum(1.0, np.abs(roots.real))].real
        out.append(not np.any((real > r_plus) & (real < r0)))
    return np.array(out)


def pixel_photon_constants(cam, a: float, col, row):
    """(xi, eta) of the photons at fractional pixel coordinates (col, row) of
    a pinhole camera (the pixel convention of camera.py:96-113 with
    continuous indices; `cam` has forward/right/up, position, width, height
    and half_extents()), past-directed null momenta from the oracle."""
    from oracle import oracle

    col, row = np.broadcast_arrays(np.atleast_1d(col).astype(float),
                                   np.atleast_1d(row).astype(float))
    half_w, half_h = cam.half_extents()
    u = ((col + 0.5) / cam.width * 2.0 - 1.0) * half_w
    v = (1.0 - (row + 0.5) / cam.height * 2.0) * half_h
    d = cam.forward[None, :] + u[:, None] * cam.right[None, :] + v[:, None] * cam.up[None, :]
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    pos = np.tile(np.asarray(cam.position, dtype=np.float64), (d.shape[0], 1))
    s = np.zeros((d.shape[0], 8))
    s[:, 1:4] = pos
    s[:, 4:8] = oracle.null_momentum(1.0, a, pos, d, True, True)
    return photon_constants(a, s)


def analytic_edge(cam, a: float, inside, outside, fixed, along_row: bool):
    """The fractional pixel coordinate between `inside` (captured) and
    `outside` (escaped) pixels of one row (along_row) or column where the
    photons' constants cross the critical curve, and the impact parameter
    sqrt(eta + xi^2) of the photon there."""

    def constants(c):
        return (pixel_photon_constants(cam, a, c, fixed) if along_row
                else pixel_photon_constants(cam, a, fixed, c))

    def captured(c):
        xi, eta = constants(c)
        return bool(captured_by_curve(a, xi, eta)[0])

    step = 1.0 if outside > inside else -1.0
    lo, hi = float(inside), float(outside)
    for _ in range(8):  # widen the bracket until it straddles the curve
        if captured(lo) and not captured(hi):
            break
        lo -= step
        hi += step
    if not (captured(lo) and not captured(hi)):
        raise AssertionError(f"no crossing of the critical curve near pixel {inside}")
    for _ in range(60):
        mid = 0.5 * (lo + hi)
        if captured(mid):
            lo = mid
        else:
            hi = mid
    c = 0.5 * (lo + hi)
    xi, eta = constants(c)
    return c, float(np.sqrt(eta[0] + xi[0] ** 2))


def frame_edges_against_curve(cam, a: float, status,
                              heights=(-0.85, -0.6, -0.3, 0.0, 0.3, 0.6, 0.85)):
    """Compare the capture boundary of a traced frame (status 1 = captured,
    row-major) with the critical curve: along rows at the given fractions of
    the shadow's half height (both ends of each) and down the column through
    the middle of the shadow (both ends).  For every edge: the traced edge
    (midway between the last captured and the first escaped pixel), the
    analytic one, and the relative difference of the photons' impact
    parameters sqrt(eta + xi^2) there."""
    cap = (np.asarray(status) == 1).reshape(cam.height, cam.width)
    rows = np.nonzero(cap.any(axis=1))[0]
    centre, half = 0.5 * (rows.min() + rows.max()), 0.5 * (rows.max() - rows.min())
    edges = []
    for f in heights:
        r = int(round(centre + f * half))
        cols = np.nonzero(cap[r])[0]
        edges.append((True, r, cols.min(), cols.min() - 1))
        edges.append((True, r, cols.max(), cols.max() + 1))
    mid_cols = np.nonzero(cap[int(round(centre))])[0]
    col = int(round(0.5 * (mid_cols.min() + mid_cols.max())))
    rr = np.nonzero(cap[:, col])[0]
    edges.append((False, col, rr.min(), rr.min() - 1))
    edges.append((False, col, rr.max(), rr.max() + 1))
    out = []
    for along_row, fixed, c_in, c_out in edges:
        c_star, b_star = analytic_edge(cam, a, c_in, c_out, fixed, along_row)
        c_t = 0.5 * (c_in + c_out)
        xi, eta = (pixel_photon_constants(cam, a, c_t, fixed) if along_row
                   else pixel_photon_constants(cam, a, fixed, c_t))
        b_t = float(np.sqrt(eta[0] + xi[0] ** 2))
        out.append({"along_row": along_row, "line": int(fixed), "traced": c_t,
                    "analytic": c_star, "b_traced": b_t, "b_analytic": b_star,
                    "relative": abs(b_t - b_star) / b_star})
    return out
