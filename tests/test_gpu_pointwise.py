"""Point-wise kernels against the reference's golden vectors (float64).

Tolerances: the kernels evaluate the reference formulas with FMA contraction
and a regrouped gradient contraction, so results agree to a few ulps of the
largest term: rtol 1e-12 on values, an absolute floor of 1e-14 x the largest
magnitude in each array for terms that cancel.
"""

import numpy as np
import pytest
import torch

from conftest import golden

pytestmark = pytest.mark.gpu


def close(a, b, rtol=1e-12, floor=1e-14):
    a = a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)
    b = np.asarray(b)
    atol = floor * max(np.max(np.abs(b)), 1.0)
    np.testing.assert_allclose(a, b, rtol=rtol, atol=atol)


def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a), device="cuda")


def test_geometry(cuda):
    from blackhorizon_b200.kerr import KerrSpacetime

    g = golden("geometry.npz")
    for tag in ("a09", "a095", "a0", "am0998"):
        st = KerrSpacetime(1.0, float(g[f"{tag}_spin"]))
        xyz = dev(g[f"{tag}_xyz"])
        geo = st.geometry(xyz[:, 0].contiguous(), xyz[:, 1].contiguous(),
                          xyz[:, 2].contiguous(), gradients=True)
        close(geo.radius, g[f"{tag}_r"])
        close(geo.h, g[f"{tag}_h"])
        close(geo.l, g[f"{tag}_l"])
        close(geo.grad_h, g[f"{tag}_grad_h"], rtol=1e-11)
        close(geo.grad_l, g[f"{tag}_grad_l"], rtol=1e-11)


def test_geometry_numpy_in_numpy_out(cuda):
    from blackhorizon_b200.kerr import KerrSpacetime

    st = KerrSpacetime(1.0, 0.8)
    x = np.array([2.0, 5.0, 11.0])
    r = st.kerr_schild_radius(x, np.zeros(3), np.zeros(3))
    assert isinstance(r, np.ndarray)
    # Reference tests/test_kerr.py:61-66: r = sqrt(x^2 - a^2) on the equator.
    np.testing.assert_allclose(r, np.sqrt(x * x - 0.64), rtol=1e-14)
    z = np.array([1.5, 3.0, -7.0])
    np.testing.assert_allclose(st.kerr_schild_radius(np.zeros(3), np.zeros(3), z),
                               np.abs(z), rtol=1e-14)


def test_rhs_hamiltonian_velocity(cuda):
    from blackhorizon_b200 import geodesics
    from blackhorizon_b200.kerr import KerrSpacetime

    g = golden("steps.npz")
    st = KerrSpacetime(1.0, float(g["spin"]))
    s = dev(g["state"])
    close(geodesics.geodesic_rhs(st, s), g["rhs"], rtol=1e-11)
    close(geodesics.hamiltonian(st, s), g["hamiltonian"], rtol=1e-9, floor=1e-15)
    close(geodesics.coordinate_velocity(st, s), g["velocity"])


@pytest.mark.parametrize("tor", ["past", "future"])
@pytest.mark.parametrize("norm", [True, False])
def test_null_momentum(cuda, tor, norm):
    from blackhorizon_b200 import geodesics
    from blackhorizon_b200.kerr import KerrSpacetime

    g = golden("null_momentum.npz")
    st = KerrSpacetime(1.0, float(g["spin"]))
    p = geodesics.null_momentum_from_velocity(st, dev(g["pos"]), dev(g["dir"]), tor, norm)
    close(p, g[f"{tor}_{int(norm)}"])


def test_camera_states(cuda):
    from blackhorizon_b200.camera import PinholeCamera
    from blackhorizon_b200.kerr import KerrSpacetime

    g = golden("trace_c1_40x30.npz")
    cam = PinholeCamera.from_orbit(50.0, 60.0, fov_degrees=30.0, width=40, height=30)
    s = cam.initial_states(KerrSpacetime(1.0, 0.9))
    close(s, g["state0"])


def test_dp5_step_fp64(cuda):
    from blackhorizon_b200 import integrators
    from blackhorizon_b200.geodesics import GeodesicRhs
    from blackhorizon_b200.kerr import KerrSpacetime

    g = golden("steps.npz")
    rhs = GeodesicRhs(KerrSpacetime(1.0, float(g["spin"])))
    s, h = dev(g["state"]), dev(g["h"])
    new, err = integrators.dormand_prince_step(rhs, s, h)
    close(new, g["dp5_new"])
    # The embedded error is a difference of O(h^5) terms: compare against the
    # magnitude of the step it estimates.
    ref = g["dp5_err"]
    scale = np.abs(g["h"])[:, None] * np.maximum(np.abs(g["rhs"]), 1e-3)
    assert np.max(np.abs(err.cpu().numpy() - ref) / scale) < 1e-12
    # error_ratio on the reference's own step outputs: same formula and
    # NumPy's pairwise summation order.
    ratio = integrators.error_ratio(s, dev(g["dp5_new"]), dev(g["dp5_err"]),
                                    float(g["rtol"]), float(g["atol"]))
    np.testing.assert_allclose(ratio.cpu().numpy(), g["ratio"], rtol=1e-15)
    factor = integrators.step_factor(dev(g["ratio"]))
    np.testing.assert_allclose(factor.cpu().numpy(), g["factor"], rtol=1e-15)


def test_dp5_step_mixed(cuda):
    """Mixed policy: float32 stage arithmetic; the update is float64, so on
    steps the reference accepts (error ratio <= 1) the new state differs from
    the reference by ~1e-6 of the step increment."""
    from blackhorizon_b200 import integrators
    from blackhorizon_b200.geodesics import GeodesicRhs
    from blackhorizon_b200.kerr import KerrSpacetime

    g = golden("steps.npz")
    rhs = GeodesicRhs(KerrSpacetime(1.0, float(g["spin"])))
    s, h = dev(g["state"]), dev(g["h"])
    new, _ = integrators.dormand_prince_step(rhs, s, h, precision="mixed")
    ok = g["ratio"] <= 1.0
    assert ok.sum() > 100
    inc = np.max(np.abs(g["dp5_new"] - g["state"]), axis=1, keepdims=True)
    rel = np.abs(new.cpu().numpy() - g["dp5_new"])[ok] / inc[ok]
    print("mixed dp5 step: max error / increment %.3g" % np.max(rel))
    assert np.max(rel) < 1e-5


def test_rk4_benchmark(cuda):
    from blackhorizon_b200 import integrators
    from blackhorizon_b200.geodesics import GeodesicRhs
    from blackhorizon_b200.kerr import KerrSpacetime

    g = golden("rk4.npz")
    rhs = GeodesicRhs(KerrSpacetime(1.0, 0.9))
    out = integrators.rk4_step(rhs, dev(g["state0"]), float(g["h"]), n_steps=int(g["n_steps"]))
    close(out, g["final"], rtol=1e-11)
    one = integrators.rk4_step(rhs, dev(g["state0"]), float(g["h"]))
    two = integrators.rk4_step(rhs, one, float(g["h"]))
    both = integrators.rk4_step(rhs, dev(g["state0"]), float(g["h"]), n_steps=2)
    close(two, both.cpu().numpy(), rtol=1e-14)


def test_empty_batches(cuda):
    from blackhorizon_b200 import geodesics, integrators
    from blackhorizon_b200.geodesics import GeodesicRhs
    from blackhorizon_b200.kerr import KerrSpacetime

    st = KerrSpacetime(1.0, 0.9)
    empty = torch.empty((0, 8), dtype=torch.float64, device="cuda")
    assert geodesics.geodesic_rhs(st, empty).shape == (0, 8)
    new, err = integrators.dormand_prince_step(GeodesicRhs(st), empty,
                                               torch.empty(0, dtype=torch.float64, device="cuda"))
    assert new.shape == (0, 8) and err.shape == (0, 8)


def test_nan_error_is_infinite_ratio(cuda):
    """Reference tests/test_integrators.py:72-76."""
    from blackhorizon_b200 import integrators

    s = torch.zeros((1, 8), dtype=torch.float64, device="cuda")
    s[0, 1] = 1.0
    bad = s.clone()
    bad[0, 1] = float("nan")
    r = integrators.error_ratio(s, s, bad, 1e-9, 1e-12)
    assert torch.isinf(r[0])


def test_implicit_midpoint_matches_reference(cuda):
    """implicit_midpoint_step (integrators.py:177-207): one step from the
    golden states with 4 and 6 iterations, and 200 steps of the bound orbit
    of tests/test_offline.py, against the reference's outputs."""
    import numpy as np

    from blackhorizon_b200 import GeodesicRhs, implicit_midpoint_step
    from blackhorizon_b200.kerr import KerrSpacetime
    from conftest import golden

    g = golden("midpoint.npz")
    rhs = GeodesicRhs(KerrSpacetime(1.0, float(g["spin"])))
    for it in (4, 6):
        got = implicit_midpoint_step(rhs, g["state"], g["h"], iterations=it)
        ref = g[f"step_it{it}"]
        np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-13)
    orbit = GeodesicRhs(KerrSpacetime(1.0, 0.9))
    got = implicit_midpoint_step(orbit, g["orbit_state0"], np.array([0.2]), n_steps=200)
    np.testing.assert_allclose(got, g["orbit_200"], rtol=1e-10, atol=1e-11)


def test_implicit_midpoint_properties(cuda):
    """tests/test_offline.py:46-103 through the b200 steppers: second-order
    convergence on one orbit, and a bounded Hamiltonian error where RK4's
    grows secularly over 30000 steps of h = 0.6."""
    import numpy as np

    from blackhorizon_b200 import (GeodesicRhs, build_state, hamiltonian,
                                   implicit_midpoint_step, rk4_step, timelike_momentum)
    from blackhorizon_b200.kerr import KerrSpacetime

    st = KerrSpacetime(1.0, 0.9)
    pos = np.array([[14.0, 0.0, 0.0]])
    s0 = build_state(pos, timelike_momentum(st, pos, np.array([[0.0, 0.21, 0.02]])))
    rhs = GeodesicRhs(st)

    def endpoint(h, steps):
        return implicit_midpoint_step(rhs, s0, np.array([h]), iterations=6, n_steps=steps)

    ref = endpoint(0.025, 4000)
    e_coarse = np.abs(endpoint(0.2, 500)[0, 1:4] - ref[0, 1:4]).max()
    e_fine = np.abs(endpoint(0.1, 1000)[0, 1:4] - ref[0, 1:4]).max()
    assert 1.6 < np.log2(e_coarse / e_fine) < 2.6
    samples = {}
    for name, stepper in (("rk4", rk4_step), ("midpoint", implicit_midpoint_step)):
        y, errors = s0.copy(), []
        for _ in range(12):
            y = stepper(rhs, y, np.array([0.6]), n_steps=2500)
            errors.append(abs(float(hamiltonian(st, y)[0]) + 0.5))
        samples[name] = np.asarray(errors)
    assert bool(np.all(np.diff(samples["rk4"]) > 0.0)) and samples["rk4"][-1] > 5 * samples["rk4"][0]
    mid = samples["midpoint"]
    assert float(mid[-1]) < 0.05 * float(mid.max()) and float(mid.max()) < 1e-2


def _device_math(op, x):
    from blackhorizon_b200 import _lib
    from blackhorizon_b200.backend import stream_handle

    xd = torch.as_tensor(x, device="cuda")
    yd = torch.empty_like(xd)
    _lib.check(_lib.load().bh_device_math(op, xd.data_ptr(), yd.data_ptr(), xd.numel(),
                                          stream_handle()), "device_math")
    return yd.cpu().numpy()


def _ulps(got, ref):
    return np.abs(got - ref) / np.spacing(np.abs(ref))


def test_float64_reciprocals_within_two_ulp(cuda):
    """The float64 reciprocal and reciprocal square root of the stage
    arithmetic (MUFU seed and two Newton-Raphson steps) against the
    correctly rounded results, from 80-bit extended NumPy arithmetic, on 10^6
    inputs log-uniform over [1e-30, 1e30] (the range of r^2, w = r^2 + a^2
    and r^4 + a^2 z^2 on the path), plus powers of two."""
    rng = np.random.default_rng(11)
    x = 10.0 ** rng.uniform(-30, 30, 1_000_000)
    x = np.concatenate([x, 2.0 ** np.arange(-99, 100), [1.0, 3.0, 0.75]])
    xl = x.astype(np.longdouble)
    rcp_ref = (1 / xl).astype(np.float64)
    rsq_ref = (1 / np.sqrt(xl)).astype(np.float64)
    rcp = _device_math(0, x)
    rsq = _device_math(1, x)
    u_rcp, u_rsq = _ulps(rcp, rcp_ref), _ulps(rsq, rsq_ref)
    print("rcp: max %.2f ulp, %.4f%% not correctly rounded; rsqrt: max %.2f ulp, %.4f%%"
          % (u_rcp.max(), 100 * np.mean(u_rcp > 0), u_rsq.max(), 100 * np.mean(u_rsq > 0)))
    assert u_rcp.max() <= 2.0 and u_rsq.max() <= 2.0
    neg = -x[:1000]
    assert np.all(_ulps(_device_math(0, neg), (1 / neg.astype(np.longdouble)).astype(np.float64))
                  <= 2.0)


def test_mixed_step_factor_from_r2(cuda):
    """The mixed controller's float64 step factor clip(0.9 x^-0.1, 0.2, 5) of
    x = r^2 (float32 seed, one Newton-Raphson step) equals the reference's
    step_factor(sqrt(x)) (integrators.py:120-124) to 1e-11 relative, and
    clips exactly at both ends."""
    rng = np.random.default_rng(12)
    x = np.concatenate([10.0 ** rng.uniform(-12, 12, 200_000),
                        [0.0, 1e-40, 3.5e-8, 3.6e-8, 1.0, 3.4e6, 3.41e6, 1e300, np.inf]])
    got = _device_math(2, x)
    xl = x.astype(np.longdouble)
    with np.errstate(divide="ignore"):
        ref = np.clip(np.longdouble(0.9) * np.power(np.maximum(xl, np.longdouble(1e-32)),
                                                    np.longdouble(-1) / 10), 0.2, 5.0)
    rel = np.abs(got - ref.astype(np.float64)) / ref.astype(np.float64)
    print("step factor: max relative error %.3g" % rel.max())
    assert rel.max() <= 1e-11
    assert got[-1] == 0.2 and got[-2] == 0.2 and got[-9] == 5.0
