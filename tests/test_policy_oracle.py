"""CPU checks of the policy's fp64 oracle: its analytic gradient against central
finite differences, and its parameter layout against the engine's C ABI size."""
import numpy as np

from oracle import policy_oracle as PO
from pathfinding_gpu_b200 import policy as P
from pathfinding_gpu_b200 import _native as N


def test_layout_matches_the_engine():
    assert PO.NP == P.NP
    assert N.load().pfg_policy_param_count() == P.NP


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    X = rng.normal(size=(40, PO.IN))
    Y = rng.dirichlet(np.ones(PO.OUT), size=40)
    flat = P.init_params(3, X.mean(0), 1 / X.std(0)).astype(np.float64)
    g = PO.grad(flat, X, Y)
    idx = list(range(0, PO.NP - 2 * PO.IN, 97))
    fd = PO.finite_difference(flat, X, Y, idx)
    np.testing.assert_allclose(g[idx], fd, rtol=1e-5, atol=1e-8)
    assert np.all(g[-2 * PO.IN:] == 0)


def test_soft_targets_prefer_the_fastest_class():
    y = P.soft_targets([2.0, 1.0, 1.5, 4.0, 8.0, 9.0, 9.5, 10.0])
    assert abs(y.sum() - 1) < 1e-6 and int(np.argmax(y)) == 1
