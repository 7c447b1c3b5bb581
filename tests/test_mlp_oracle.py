"""The MLP oracle's analytic gradient against central finite differences (CPU)."""
import numpy as np

from oracle import mlp_oracle as mo


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = rng.normal(0, 0.3, mo.NPARAMS)
    X = rng.normal(0, 1, (37, mo.F))
    T = rng.normal(0, 1, 37)
    loss, g = mo.loss_and_grad(p, X, T)
    idx = rng.choice(mo.NPARAMS, 300, replace=False)
    idx = np.concatenate([idx, [mo.OFF["b3"], mo.OFF["W1"], mo.OFF["b2"]]])
    eps = 1e-6
    for k in idx:
        pp, pm = p.copy(), p.copy()
        pp[k] += eps
        pm[k] -= eps
        num = (mo.loss_and_grad(pp, X, T)[0] - mo.loss_and_grad(pm, X, T)[0]) / (2 * eps)
        assert abs(num - g[k]) <= 1e-6 + 1e-5 * abs(num), (k, num, g[k])


def test_parameter_count():
    assert mo.NPARAMS == 4609
