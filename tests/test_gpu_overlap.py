"""The stepper's overlap test through the occupancy grid against the chunk sweep and the oracle.

The reference rejects a move when the new centroid lies within 1.5 A of any receptor atom
(gpu_batch_simulator.py:770-781, 1102-1128; oracle/stepper.py `_overlap_inside`).  The grid
answers from a cell word and a short atom list; the answer must be the sweep's for every
centroid, including centroids 1e-12 A either side of the 1.5 A sphere of an atom.
"""

import numpy as np
import pytest

from tests.helpers import system

pytestmark = pytest.mark.gpu


class _MP:
    def __init__(self, s):
        self.dipole, self.quadrupole, self.four_pi_eps = s.multipole_moments()


def _engine(s, layout):
    from pystarc_b200.engine import B200ForceEngine

    eng = B200ForceEngine(**s.engine_kwargs(), multipole_expansion=_MP(s) if s.multipole else None, layout=layout)
    eng.set_ligand(s.lig_pos - s.lig_pos.mean(axis=0), s.lig_q)
    return eng


def _points(rec, seed, n_shell=20000, n_box=20000):
    rng = np.random.default_rng(seed)
    pts = []
    # on and near the 1.5 A sphere of random atoms
    for delta in (-0.3, -1e-3, -1e-9, -1e-12, 1e-12, 1e-9, 1e-3, 0.3):
        a = rec[rng.integers(0, len(rec), n_shell // 8)]
        u = rng.standard_normal(a.shape)
        u /= np.linalg.norm(u, axis=1, keepdims=True)
        pts.append(a + u * (1.5 + delta))
    # anywhere in the receptor's box and around it
    lo, hi = rec.min(axis=0) - 4.0, rec.max(axis=0) + 4.0
    pts.append(rng.uniform(lo, hi, (n_box, 3)))
    # far away, on the box faces and at a quarter-angstrom lattice (cell boundaries of the grid)
    pts.append(rng.standard_normal((200, 3)) * 200.0)
    steps = np.floor((hi - lo) / 0.25).astype(np.int64)
    pts.append(lo + 0.25 * rng.integers(0, steps + 1, (5000, 3)))
    return np.concatenate(pts)


@pytest.mark.parametrize("name", ["c2", "c3"])
def test_overlap_grid_matches_the_sweep_and_the_oracle(name):
    from oracle.stepper import _overlap_inside
    from pystarc_b200 import _lib

    s = system(name)
    rec = np.asarray(s.rec_pos, dtype=np.float64)
    pts = _points(rec, 7)
    want = _overlap_inside(pts, rec, 1.5)
    grid = _engine(s, _lib.LAYOUT_DEFAULT)
    sweep = _engine(s, _lib.LAYOUT_DEFAULT & ~_lib.LAYOUT_OVERLAP_GRID)
    got_grid = grid.eval_overlap(pts)
    got_sweep = sweep.eval_overlap(pts)
    np.testing.assert_array_equal(got_sweep, want)
    np.testing.assert_array_equal(got_grid, want)
    assert 0.05 < want.mean() < 0.95  # both answers occur
    grid.close()
    sweep.close()


def test_overlap_grid_at_full_size():
    """Protein + small ligand at its benchmark size (3,200 receptor atoms)."""
    from oracle.stepper import _overlap_inside
    from pystarc_b200 import _lib
    from tests import fullsize as fs

    s = fs.system("c2")
    rec = np.asarray(s.rec_pos, dtype=np.float64)
    pts = _points(rec, 11, n_shell=40000, n_box=40000)
    want = _overlap_inside(pts, rec, 1.5)
    eng = _engine(s, _lib.LAYOUT_DEFAULT)
    np.testing.assert_array_equal(eng.eval_overlap(pts), want)
    eng.close()


def test_overlap_grid_keeps_fp64_trajectories():
    """Whole FP64 runs (fused and split step) with and without the grid: the same fates, steps and
    counters, rejections included."""
    from pystarc_b200 import _lib
    from pystarc_b200.engine import B200ForceEngine
    from pystarc_b200.simulator import B200BatchSimulator

    s = system("c2")
    outs = []
    for layout in (_lib.LAYOUT_DEFAULT, _lib.LAYOUT_DEFAULT & ~_lib.LAYOUT_OVERLAP_GRID):
        for group in (65, 66):
            eng = B200ForceEngine(**s.engine_kwargs(), multipole_expansion=_MP(s) if s.multipole else None,
                                  precision="fp64", layout=layout)
            mol1, mol2 = s.molecules()
            sim = B200BatchSimulator(mol1, mol2, s.mobility(), s.pathway_set(), s.params(n_traj=700, max_steps=400),
                                     eng, termination="complete", steps_per_launch=16, slots=700)
            eng.handle.call("bd_set_launch", group, 256)
            res = sim.run()
            outs.append((sim.outcomes(), res.counters))
            eng.close()
    assert outs[0][1]["overlap"] > 0
    for o, c in outs[1:]:
        for x, y in zip(outs[0][0], o):
            np.testing.assert_array_equal(x, y)
        for k in ("steps", "reacted", "escaped", "returns", "overlap", "bridge"):
            assert c[k] == outs[0][1][k], k
