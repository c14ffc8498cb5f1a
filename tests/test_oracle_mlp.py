"""The float64 statement of the control-variate network and estimator (oracle/mlp.py): its
analytic gradient against central finite differences, and the estimator's unbiasedness."""
import itertools

import numpy as np

from oracle import mlp as O


def _net(seed=0, D=6, H=8, B=5):
    rs = np.random.default_rng(seed)
    n = H * D + H + H * H + H + H + 1
    p = rs.standard_normal(n) * 0.5
    X = rs.standard_normal((B, D))
    t = rs.standard_normal(B) * 2.0 + 1.0
    mean, istd = rs.standard_normal(D) * 0.1, 1.0 + rs.random(D)
    return p, X, t, D, H, mean, istd


def test_gradient_matches_finite_differences():
    p, X, t, D, H, mean, istd = _net()
    loss, g = O.loss_and_grad(p, X, t, D, H, mean, istd, 1.0, 2.0)
    h = 1e-6
    num = np.empty_like(p)
    for i in range(p.size):
        e = np.zeros_like(p)
        e[i] = h
        lp, _ = O.loss_and_grad(p + e, X, t, D, H, mean, istd, 1.0, 2.0)
        lm, _ = O.loss_and_grad(p - e, X, t, D, H, mean, istd, 1.0, 2.0)
        num[i] = (lp - lm) / (2 * h)
    assert np.max(np.abs(num - g)) < 1e-7 * max(1.0, np.max(np.abs(g)))


def test_gelu_grad():
    z = np.linspace(-4, 4, 41)
    h = 1e-6
    num = (O.gelu(z + h) - O.gelu(z - h)) / (2 * h)
    assert np.max(np.abs(num - O.gelu_grad(z))) < 1e-8


def test_multifidelity_estimator_is_unbiased():
    """The average over every subset of size k equals the exact weighted sum, for any f."""
    rs = np.random.default_rng(3)
    W, k = 7, 3
    omega = rs.random(W) + 0.1
    e = rs.standard_normal(W)
    f = rs.standard_normal(W)  # a poor predictor: unbiasedness must not depend on it
    ests = [O.multifidelity_sum(omega, f, e[list(S)], list(S))
            for S in itertools.combinations(range(W), k)]
    assert abs(np.mean(ests) - np.sum(omega * e)) < 1e-12
    # with f = e the estimator is exact for every subset
    ests = [O.multifidelity_sum(omega, e, e[list(S)], list(S))
            for S in itertools.combinations(range(W), k)]
    assert np.max(np.abs(np.array(ests) - np.sum(omega * e))) < 1e-12


def test_weighted_draw_estimator_is_unbiased():
    """Expectation over the multinomial draws (enumerated exactly for k = 2) equals the exact
    weighted sum for any f and any positive draw probabilities."""
    rs = np.random.default_rng(4)
    W = 6
    omega = rs.random(W) + 0.1
    e, f = rs.standard_normal(W), rs.standard_normal(W)
    prob = omega / omega.sum()
    exp = 0.0
    for a in range(W):
        for b in range(W):
            exp += prob[a] * prob[b] * O.multifidelity_sum_weighted(omega, f, e, [a, b], prob)
    assert abs(exp - np.sum(omega * e)) < 1e-12
