"""The surrogate's CPU oracle: BF16 rounding, the network's gradient and the feature map."""

import numpy as np

from oracle import mlp as om
from pystarc_b200.surrogate import SurrogateSpec


def test_bf16_rounding_known_values():
    x = np.array([1.0, 1.00390625, 1.005859375, 3.0e38, -2.5, 1.0 + 2 ** -8 + 2 ** -9], dtype=np.float64)
    y = om.bf16(x)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: even mantissa wins (1.0)
    assert y[0] == 1.0 and y[1] == 1.0
    assert y[2] == 1.0078125  # above the tie: rounds up
    assert y[4] == -2.5
    assert y[5] == 1.0078125
    assert np.isfinite(y[3])


def _case(seed=3, n=64, dims=(5, 16, 2, 3)):
    rng = np.random.default_rng(seed)
    in_dim, hidden, n_hidden, out_dim = dims
    d = om.layer_dims(in_dim, hidden, n_hidden, out_dim)
    n_par = sum(o * i + o for i, o in d)
    p = rng.normal(0, 0.5, n_par)
    X = rng.normal(0, 1, (n, in_dim))
    T = rng.normal(0, 1, (n, out_dim))
    return d, p, X, T


def test_oracle_gradient_matches_finite_differences():
    d, p, X, T = _case()
    loss, g = om.loss_and_grad(p, d, X, T, rounding=False)
    rng = np.random.default_rng(0)
    for k in rng.choice(p.size, 40, replace=False):
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[k] += h
        pm[k] -= h
        fd = (om.loss_and_grad(pp, d, X, T, False)[0] - om.loss_and_grad(pm, d, X, T, False)[0]) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(fd)), (k, fd, g[k])


def test_rounded_gradient_close_to_exact():
    d, p, X, T = _case()
    _, g = om.loss_and_grad(p, d, X, T, rounding=False)
    _, gr = om.loss_and_grad(p, d, X, T, rounding=True)
    assert np.linalg.norm(gr - g) <= 2e-2 * np.linalg.norm(g)


def test_adam_first_step_moves_by_lr():
    p = np.array([1.0, -2.0, 3.0])
    g = np.array([0.5, -1e-3, 0.0])
    pn, m1, m2 = om.adam(p, g, np.zeros(3), np.zeros(3), 1, 1e-3)
    # bias-corrected first step: lr * sign(g) (zero gradient: no move)
    np.testing.assert_allclose(pn - p, [-1e-3, 1e-3, 0.0], rtol=1e-4, atol=1e-12)


def test_features_identify_q_and_minus_q():
    spec = SurrogateSpec()
    c = np.array([[30.0, -4.0, 2.0]])
    q = np.array([[-0.5, 0.5, -0.5, 0.5]])
    f1, f2 = spec.features(c, q), spec.features(c, -q)
    np.testing.assert_array_equal(f1, f2)
    assert f1.shape == (1, 13) and f1.dtype == np.float32
    assert abs(f1[0, 3] - np.linalg.norm(c) / spec.r_scale) < 1e-7


def test_envelope_follows_a_radial_profile():
    rng = np.random.default_rng(4)
    r = rng.uniform(20, 60, 200000)
    size = np.exp(-r / 8.0) / r
    d = rng.normal(size=(r.size, 3))
    f = d / np.linalg.norm(d, axis=1, keepdims=True) * size[:, None]
    spec = SurrogateSpec()
    spec.fit_envelope(r, f)
    probe = np.linspace(22, 58, 50)
    ratio = spec.envelope(probe) / (np.exp(-probe / 8.0) / probe)
    assert np.all(np.abs(np.log(ratio)) < 0.05), ratio
    assert spec.envelope(np.array([5.0]))[0] == spec.envelope(np.array([spec.env_r0]))[0]  # clamped
