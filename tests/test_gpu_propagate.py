"""Raw-throughput workload (2000 attempted DP5(4) steps per ray, per-ray spin,
no termination) against the reference's end points for its first 512 rays.

Endpoint error of a ray = max over the 8 components of
|y - y_ref| / max(|y_ref|, 1): relative for large components, absolute for
components near zero (momenta of order 1, p_z of an equatorial ray ~ 0).
Float64 policy: median 1e-10, every ray 1e-6.  Mixed policy: median 1e-6;
the target of the raw-throughput benchmark is <= 1e-6 at the median.
"""

import numpy as np
import pytest
import torch

from conftest import golden

pytestmark = pytest.mark.gpu


def endpoint_error(got, ref):
    return np.max(np.abs(got - ref) / np.maximum(np.abs(ref), 1.0), axis=1)


def run(precision, layout="aos"):
    from blackhorizon_b200 import propagate
    from blackhorizon_b200.kerr import KerrSpacetime

    g = golden("raw_throughput.npz")
    s0 = torch.as_tensor(g["state0"], device="cuda")
    if layout == "soa":
        s0 = s0.t().contiguous()
    states, h, acc, stats = propagate(
        KerrSpacetime(1.0, 0.0), s0, int(g["n_steps"]), rtol=float(g["rtol"]),
        atol=float(g["atol"]), precision=precision, spins=g["spin"], layout=layout)
    if layout == "soa":
        states = states.t()
    return g, states.cpu().numpy(), acc.cpu().numpy(), stats


def test_fp64_endpoints(cuda):
    g, got, acc, stats = run("fp64")
    err = endpoint_error(got, g["final"])
    assert np.median(err) < 1e-10
    assert np.max(err) < 1e-6
    assert stats.attempts == 512 * 2000 and stats.iterations == 2000
    assert np.mean(acc == g["accepted"]) > 0.9
    assert stats.accepted == int(acc.sum())


def test_soa_layout(cuda):
    _, a, acc_a, _ = run("fp64")
    _, b, acc_b, _ = run("fp64", "soa")
    np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(acc_a, acc_b)


def test_mixed_endpoints(cuda):
    g, got, acc, stats = run("mixed")
    err = endpoint_error(got, g["final"])
    print("mixed endpoint error: median %.3g p90 %.3g max %.3g; accepted %.4f of ref"
          % (np.median(err), np.quantile(err, 0.9), np.max(err),
             acc.sum() / g["accepted"].sum()))
    assert np.median(err) < 1e-6
    assert np.all(np.isfinite(got))
