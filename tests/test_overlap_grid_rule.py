"""The occupancy-grid rule of the overlap test, restated on the host (no GPU).

The device classifies 0.5 A cells over the receptor's box (widened by 1.5 A + one cell):
EMPTY when every atom is at least 1.5 A + 1e-9 from the whole cell, FULL when one atom is
within 1.5 A - 1e-9 of all of it, MIXED otherwise with the atoms that come within 1.5 A + 1e-9
of the cell.  A query reads its cell and, for MIXED, tests the listed atoms.  This test checks
that rule against the reference's brute-force test (gpu_batch_simulator.py:1106-1128, restated
in oracle/stepper.py `_overlap_inside`) on centroids 1e-12 A either side of atoms' 1.5 A spheres,
on cell faces and anywhere in the box.  The GPU tests check the kernels against the same oracle.
"""

import numpy as np

H, R, EPS = 0.5, 1.5, 1e-9


def _grid(rec):
    lo, hi = rec.min(0), rec.max(0)
    o = lo - (R + H)
    n = np.ceil((hi + R + H - o) / H).astype(int)
    idx = np.stack(np.meshgrid(*[np.arange(k) for k in n], indexing="ij"), -1).reshape(-1, 3)
    clo = o + idx * H
    chi = clo + H
    full = np.zeros(len(idx), bool)
    lists = [[] for _ in range(len(idx))]
    for a, x in enumerate(rec):
        e = np.maximum(np.maximum(clo - x, x - chi), 0.0)
        dn = np.sqrt((e * e).sum(1))
        f = np.maximum(np.abs(x - clo), np.abs(x - chi))
        df = np.sqrt((f * f).sum(1))
        full |= df < R - EPS
        for c in np.nonzero(dn < R + EPS)[0]:
            lists[c].append(a)
    return o, n, full, lists


def _query(rec, grid, p):
    o, n, full, lists = grid
    u = (p - o) / H
    if not np.all((u >= 0) & (u < n)):
        return False
    i, j, k = u.astype(int)
    c = (i * n[1] + j) * n[2] + k
    if full[c]:
        return True
    return any(np.sqrt(((p - rec[a]) ** 2).sum()) < R for a in lists[c])


def test_grid_rule_is_exact():
    from oracle.stepper import _overlap_inside
    from pystarc_b200.synth import _protein

    rec, _, _ = _protein(120, 6.6, 2.0, 0.35, 2001)
    grid = _grid(rec)
    rng = np.random.default_rng(3)
    pts = [rng.uniform(rec.min(0) - 3, rec.max(0) + 3, (1500, 3))]
    for d in (-1e-12, 1e-12, -1e-9, 1e-9):
        a = rec[rng.integers(0, len(rec), 300)]
        u = rng.standard_normal(a.shape)
        u /= np.linalg.norm(u, axis=1, keepdims=True)
        pts.append(a + u * (R + d))
    o = grid[0]
    pts.append(o + H * rng.integers(0, 40, (500, 3)))  # cell corners
    pts = np.concatenate(pts)
    want = _overlap_inside(pts, rec, R)
    got = np.array([_query(rec, grid, p) for p in pts])
    np.testing.assert_array_equal(got, want)
    assert 0.1 < want.mean() < 0.9
