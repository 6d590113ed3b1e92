"""The engine's 20-node grid stencil equals the reference's 7-interpolation stencil.

The reference's K1 (gpu_batch_engine.py:65-123) takes the gradient of a trilinear
interpolant I as (I(x + h) - I(x - h)) / (2h) with h = spacing / 2, at 7 x 8 corner
gathers.  The CUDA stencil (``stencil`` in pystarc_b200/csrc/bd_device.cuh) computes the
same quantity from 20 distinct nodes: with c = floor(u) and s = u - c, the two probes of an
axis share the fraction |s - 1/2| and straddle one extra node e = c - 1 (s < 1/2) or c + 2
(s >= 1/2), so D = (1 - a)(v[c+1] - v[c]) + a * (adjacent difference at e), a = |s - 1/2|,
weighted bilinearly on the other two axes.

This restates that arithmetic in NumPy, node for node as the kernel reads them, and checks it
in FP64 against the oracle's K1 on random grids, including positions on a node and exactly
half-way between nodes (the s = 1/2 switch).  The GPU tests compare the kernel itself with
the oracle; this pins the algebra without a GPU.
"""

import numpy as np
import pytest

from oracle.forces import GRID_MARGIN, k1_batch_force


def stencil20(data, origin, sp, pos):
    """phi and grad from the 20 nodes the CUDA stencil reads (FP64)."""
    u = (pos - origin) / sp
    c = np.floor(u).astype(np.int64)
    s = u - c
    low = s < 0.5
    a = np.where(low, 0.5 - s, s - 0.5)
    e = np.where(low, c - 1, c + 2)  # extra node per axis
    cx, cy, cz = c[:, 0], c[:, 1], c[:, 2]

    def v(i, j, k):
        return data[i, j, k]

    w = [(1 - s[:, d], s[:, d]) for d in range(3)]
    phi = np.zeros(len(pos))
    for i in range(2):
        for j in range(2):
            for k in range(2):
                phi += w[0][i] * w[1][j] * w[2][k] * v(cx + i, cy + j, cz + k)
    grad = np.zeros((len(pos), 3))
    for j in range(2):  # x: centre differences of rows (y, z), extra x plane
        for k in range(2):
            d0 = v(cx + 1, cy + j, cz + k) - v(cx, cy + j, cz + k)
            ev = v(e[:, 0], cy + j, cz + k)
            de = np.where(low[:, 0], v(cx, cy + j, cz + k) - ev, ev - v(cx + 1, cy + j, cz + k))
            grad[:, 0] += w[1][j] * w[2][k] * ((1 - a[:, 0]) * d0 + a[:, 0] * de)
    for i in range(2):  # y: extra y row
        for k in range(2):
            d0 = v(cx + i, cy + 1, cz + k) - v(cx + i, cy, cz + k)
            ev = v(cx + i, e[:, 1], cz + k)
            de = np.where(low[:, 1], v(cx + i, cy, cz + k) - ev, ev - v(cx + i, cy + 1, cz + k))
            grad[:, 1] += w[0][i] * w[2][k] * ((1 - a[:, 1]) * d0 + a[:, 1] * de)
    for i in range(2):  # z: extra z node
        for j in range(2):
            d0 = v(cx + i, cy + j, cz + 1) - v(cx + i, cy + j, cz)
            ev = v(cx + i, cy + j, e[:, 2])
            de = np.where(low[:, 2], v(cx + i, cy + j, cz) - ev, ev - v(cx + i, cy + j, cz + 1))
            grad[:, 2] += w[0][i] * w[1][j] * ((1 - a[:, 2]) * d0 + a[:, 2] * de)
    return phi, grad / sp


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_twenty_node_stencil_equals_reference_k1(seed):
    rng = np.random.default_rng(seed)
    n = np.array([17, 14, 19])
    sp = rng.uniform(0.4, 1.1, 3)
    origin = rng.uniform(-10, 10, 3)
    # a smooth field plus node noise, FP32 values as the grids hold them
    x = [origin[d] + sp[d] * np.arange(n[d]) for d in range(3)]
    X, Y, Z = np.meshgrid(*x, indexing="ij")
    data = (np.exp(-0.01 * (X ** 2 + Y ** 2 + Z ** 2)) + 0.1 * rng.standard_normal(tuple(n)))
    data = data.astype(np.float32).astype(np.float64)
    lo = origin + GRID_MARGIN * sp
    hi = origin + (n - 1 - GRID_MARGIN) * sp
    pos = rng.uniform(lo + 1e-6, hi - 1e-6, (4000, 3))
    # on a node and exactly half-way between nodes, on each axis
    nodes = origin + sp * rng.integers(GRID_MARGIN + 1, n - GRID_MARGIN - 1, (200, 3))
    half = origin + sp * (rng.integers(GRID_MARGIN + 1, n - GRID_MARGIN - 2, (200, 3)) + 0.5)
    pos = np.concatenate([pos, nodes, half])
    phi, grad = stencil20(data, origin, sp, pos)
    q = -np.ones(len(pos))  # K1's elec force is -q grad: +grad for q = -1, energy q phi
    f, e = k1_batch_force(pos, q, data, origin, sp, 0.0, False)
    scale = np.abs(f).max()
    np.testing.assert_allclose(grad, f, rtol=0, atol=1e-12 * scale)
    np.testing.assert_allclose(phi, -e, rtol=0, atol=1e-12 * np.abs(e).max())
