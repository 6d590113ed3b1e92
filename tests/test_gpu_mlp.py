"""Surrogate MLP kernels (BF16 tensor cores, FP32 accumulation) against the CPU oracle."""

import numpy as np
import pytest

from oracle import mlp as om

pytestmark = pytest.mark.gpu


def _ens(members=2, in_dim=13, hidden=256, n_hidden=4, out_dim=6, seed=7):
    from pystarc_b200.surrogate import MLPEnsemble

    return MLPEnsemble(members, in_dim, hidden, n_hidden, out_dim, seed=seed)


def _data(n, in_dim, out_dim, seed=1):
    rng = np.random.default_rng(seed)
    return rng.normal(0, 1, (n, in_dim)).astype(np.float32), rng.normal(0, 1, (n, out_dim)).astype(np.float32)


@pytest.mark.parametrize("shape", [(13, 256, 4, 6), (7, 128, 2, 3)])
def test_forward_matches_oracle(shape):
    in_dim, hidden, n_hidden, out_dim = shape
    e = _ens(2, in_dim, hidden, n_hidden, out_dim)
    X, _ = _data(1000, in_dim, out_dim)
    for m in range(2):
        p = e.get_params(m).astype(np.float64)
        Y = e.forward(m, X).cpu().numpy()
        Yo, _ = om.forward(p, e.dims, X, rounding=True)
        assert np.max(np.abs(Y - Yo)) <= 2e-2 * np.max(np.abs(Yo)) + 1e-4
    e.close()


@pytest.mark.parametrize("n", [64, 2048])
def test_gradient_matches_oracle(n):
    e = _ens(1)
    X, T = _data(n, 13, 6, seed=n)
    loss, g = e.grad(0, X, T)
    p = e.get_params(0).astype(np.float64)
    lo, go = om.loss_and_grad(p, e.dims, X, T, rounding=True)
    g = g.cpu().numpy().astype(np.float64)
    assert abs(loss - lo) <= 1e-3 * lo
    # layer by layer: relative L2 error of each weight and bias block
    k = 0
    for i, o in e.dims:
        for size in (o * i, o):
            a, b = g[k:k + size], go[k:k + size]
            assert np.linalg.norm(a - b) <= 2e-2 * np.linalg.norm(b) + 1e-9, (i, o, size)
            k += size
    e.close()


def test_adam_step_applies_oracle_update():
    e = _ens(1)
    X, T = _data(512, 13, 6, seed=5)
    p0 = e.get_params(0).astype(np.float64)
    _, g = e.grad(0, X, T)
    e.train_step(0, e._dev(X), e._dev(T), 1e-3)
    p1 = e.get_params(0).astype(np.float64)
    pn, _, _ = om.adam(p0, g.cpu().numpy().astype(np.float64), np.zeros_like(p0), np.zeros_like(p0), 1, 1e-3)
    np.testing.assert_allclose(p1, pn, rtol=0, atol=2e-6)
    e.close()


def test_training_fits_a_smooth_function():
    e = _ens(1)
    rng = np.random.default_rng(2)
    X = rng.uniform(-1, 1, (8192, 13)).astype(np.float32)
    T = np.stack([np.sin(2 * X[:, 0]) + X[:, 1] * X[:, 2], np.cos(X[:, 3]) - X[:, 4] ** 2] + [X[:, 5]] * 4,
                 axis=1).astype(np.float32)
    Xd, Td = e._dev(X), e._dev(T)
    l0, _ = e.grad(0, X, T)
    for _ in range(400):
        e.train_step(0, Xd, Td, 1e-3)
    l1, _ = e.grad(0, X, T)
    assert l1 < 0.05 * l0, (l0, l1)
    e.close()


def test_ensemble_mean_and_spread():
    e = _ens(3)
    X, _ = _data(777, 13, 6, seed=9)
    mean, spread = e.ensemble(X)
    Ys = np.stack([e.forward(m, X).cpu().numpy() for m in range(3)])
    np.testing.assert_allclose(mean.cpu().numpy(), Ys.mean(0), rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(spread.cpu().numpy(), Ys.std(0), rtol=1e-4, atol=1e-6)
    e.close()


def test_bad_batch_is_rejected():
    from pystarc_b200._lib import BdError

    e = _ens(1)
    X, T = _data(40, 13, 6)
    with pytest.raises(BdError, match="multiple of 32"):
        e.grad(0, X, T)
    e.close()


def test_device_training_loop_matches_eager_steps_in_effect():
    """bd_mlp_train (graph-replayed) lowers the loss like the eager steps do."""
    e = _ens(1)
    rng = np.random.default_rng(3)
    X = rng.uniform(-1, 1, (20000, 13)).astype(np.float32)
    T = np.stack([np.sin(2 * X[:, 0]) + X[:, 1] * X[:, 2], np.cos(X[:, 3])] + [X[:, 5]] * 4, axis=1).astype(np.float32)
    l0, _ = e.grad(0, X[:4096], T[:4096])
    tr = e.train(0, X, T, 1024, 600, 1e-3, seed=5).cpu().numpy()
    l1, _ = e.grad(0, X[:4096], T[:4096])
    assert np.all(np.isfinite(tr)) and tr[-50:].mean() < 0.1 * tr[:5].mean()
    assert l1 < 0.05 * l0, (l0, l1)
    # a second call continues from the trained weights (Adam state kept)
    tr2 = e.train(0, X, T, 1024, 50, 1e-3, seed=6).cpu().numpy()
    assert tr2.mean() < 2 * tr[-50:].mean()
    e.close()


@pytest.mark.parametrize("shape,n", [((13, 256, 4, 6), 1000), ((13, 256, 4, 6), 300_000), ((7, 128, 2, 3), 333)])
def test_tcgen05_inference_matches_mma_sync_and_oracle(shape, n):
    in_dim, hidden, n_hidden, out_dim = shape
    e = _ens(3, in_dim, hidden, n_hidden, out_dim, seed=21)
    X, _ = _data(n, in_dim, out_dim, seed=4)
    e.set_inference(1)
    Y_tc = e.forward(1, X).cpu().numpy()
    mean_tc, spread_tc = (t.cpu().numpy() for t in e.ensemble(X))
    e.set_inference(0)
    Y_mma = e.forward(1, X).cpu().numpy()
    mean_mma, spread_mma = (t.cpu().numpy() for t in e.ensemble(X))
    scale = np.max(np.abs(Y_mma))
    assert np.all(np.isfinite(Y_tc))
    assert np.max(np.abs(Y_tc - Y_mma)) <= 2e-2 * scale, np.max(np.abs(Y_tc - Y_mma))
    assert np.median(np.abs(Y_tc - Y_mma)) <= 1e-3 * scale
    np.testing.assert_allclose(mean_tc, mean_mma, atol=2e-2 * np.max(np.abs(mean_mma)))
    k = min(n, 2000)
    Yo, _ = om.forward(e.get_params(1).astype(np.float64), e.dims, X[:k], rounding=True)
    assert np.max(np.abs(Y_tc[:k] - Yo)) <= 2e-2 * np.max(np.abs(Yo)) + 1e-4
    e.close()


# 4096 rows: 64-column tiles; 12800: 128-column tiles; 40000: 256-column tiles, several row tiles per CTA
@pytest.mark.parametrize("shape,n", [((13, 256, 4, 6), 4096), ((7, 128, 2, 3), 2080), ((13, 256, 4, 6), 12800),
                                     ((13, 256, 4, 6), 40000)])
def test_tcgen05_training_gemms_match_mma_sync(shape, n):
    """The training GEMMs on tcgen05 (forward, weight and activation gradients, split-K partials) give
    the loss and the per-layer gradients of the mma.sync GEMMs to BF16-rounding accuracy."""
    in_dim, hidden, n_hidden, out_dim = shape
    e = _ens(1, in_dim, hidden, n_hidden, out_dim, seed=11)
    X, T = _data(n, in_dim, out_dim, seed=6)
    e.set_gemm(1)
    l_tc, g_tc = e.grad(0, X, T)
    Y_tc = e.forward(0, X).cpu().numpy()
    e.set_gemm(0)
    l_mma, g_mma = e.grad(0, X, T)
    Y_mma = e.forward(0, X).cpu().numpy()
    e.set_gemm(1)
    assert abs(l_tc - l_mma) <= 1e-3 * l_mma
    assert np.max(np.abs(Y_tc - Y_mma)) <= 1e-2 * np.max(np.abs(Y_mma))
    g_tc, g_mma = g_tc.cpu().numpy().astype(np.float64), g_mma.cpu().numpy().astype(np.float64)
    k = 0
    for i, o in e.dims:
        for size in (o * i, o):
            a, b = g_tc[k:k + size], g_mma[k:k + size]
            assert np.linalg.norm(a - b) <= 1e-2 * np.linalg.norm(b) + 1e-9, (i, o, size)
            k += size
    e.close()
