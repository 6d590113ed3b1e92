"""CPU oracle of the surrogate MLP (test infrastructure only).

There is no reference counterpart: the surrogate is the engine's own learned
part.  This module restates, in FP64 NumPy, the network the CUDA kernels in
``pystarc_b200/csrc/bd_mlp.cu`` compute: ``in -> hidden x n_hidden (SiLU) ->
out`` with the mean squared error over rows and outputs.  Parameters are one
flat FP32 vector per member, layer by layer W (out x in, row-major) then b.

``rounding=True`` mirrors the kernels' BF16 rounding points (inputs, weights,
hidden activations, output gradient dY and hidden gradients dZ are rounded to
BF16; everything else stays wide), so the CUDA gradients can be compared
element by element.  ``rounding=False`` is the plain FP64 network, which the
finite-difference test pins.
"""

from __future__ import annotations

import numpy as np


def bf16(x):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    f = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def layer_dims(in_dim, hidden, n_hidden, out_dim):
    dims = [in_dim] + [hidden] * n_hidden + [out_dim]
    return list(zip(dims[:-1], dims[1:]))


def unpack(params, dims):
    """Flat parameter vector -> [(W (out x in), b (out))]."""
    out, k = [], 0
    p = np.asarray(params, dtype=np.float64)
    for i, o in dims:
        W = p[k:k + o * i].reshape(o, i)
        k += o * i
        b = p[k:k + o]
        k += o
        out.append((W, b))
    assert k == p.size
    return out


def pack(layers):
    return np.concatenate([np.concatenate([W.ravel(), b]) for W, b in layers])


def _silu(z):
    return z / (1.0 + np.exp(-z))


def _silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(params, dims, X, rounding=True):
    """Outputs (n x out) and the saved (input, pre-activation) of every layer."""
    r = bf16 if rounding else (lambda v: np.asarray(v, dtype=np.float64))
    layers = unpack(params, dims)
    a = r(X)
    saved = []
    for li, (W, b) in enumerate(layers):
        z = a @ r(W).T + b
        saved.append((a, z))
        if li + 1 < len(layers):
            a = r(_silu(z))
        else:
            return z, saved
    raise AssertionError


def loss_and_grad(params, dims, X, T, rounding=True):
    """Mean squared error over rows and outputs and its gradient (flat, like params)."""
    r = bf16 if rounding else (lambda v: np.asarray(v, dtype=np.float64))
    layers = unpack(params, dims)
    Y, saved = forward(params, dims, X, rounding)
    n, od = Y.shape
    e = Y - np.asarray(T, dtype=np.float64)
    loss = float(np.mean(e * e))
    dz = r(2.0 * e / (n * od))
    grads = [None] * len(layers)
    for li in range(len(layers) - 1, -1, -1):
        a_in, _ = saved[li]
        W, _ = layers[li]
        grads[li] = (dz.T @ a_in, dz.sum(axis=0))
        if li == 0:
            break
        da = dz @ r(W)
        dz = r(da * _silu_grad(saved[li - 1][1]))
    return loss, pack(grads)


def adam(params, grad, m1, m2, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One bias-corrected Adam step (returns new params, m1, m2)."""
    m1 = b1 * m1 + (1 - b1) * grad
    m2 = b2 * m2 + (1 - b2) * grad * grad
    c1, c2 = 1 - b1 ** step, 1 - b2 ** step
    return params - lr * (m1 / c1) / (np.sqrt(m2 / c2) + eps), m1, m2
