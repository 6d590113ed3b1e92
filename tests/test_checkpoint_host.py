"""Resume from a checkpoint that cannot be used: the run starts fresh, as the reference does.

The reference prints "Checkpoint load failed ... Starting fresh." for any error while it reads
``checkpoint.npz`` (gpu_batch_simulator.py:548-575).  Here the simulator's host loop runs on
CPU with its device calls answered by the oracle stepper (the mocked handle of the multi-rank
tests); a garbage file, a truncated file and another run's checkpoint must each give the result
of a run without any checkpoint, and the file is removed at the end of the run.
"""

import numpy as np
import pytest

from tests.helpers import system
from tests.test_multi_rank import _FakeEngine


def _run(tmp_path, n_traj=48):
    from pystarc_b200.simulator import B200BatchSimulator

    s = system("two_sphere")
    mol1, mol2 = s.molecules()
    p = s.params(n_traj=n_traj, max_steps=5000)
    p.checkpoint_interval = 10
    p._work_dir = str(tmp_path)
    sim = B200BatchSimulator(mol1, mol2, s.mobility(), s.pathway_set(), p, _FakeEngine(s), termination="complete")
    return sim.run()


def _bad_files(tmp_path):
    yield "garbage", b"this is not a checkpoint"
    good = tmp_path / "other.npz"
    np.savez(good, c=np.zeros(300), q=np.zeros(400), n_traj=48, seed=1, cap=100)
    data = good.read_bytes()
    yield "truncated", data[: len(data) // 2]
    np.savez(good, n_traj=7, seed=1, cap=100)  # another run's checkpoint
    yield "foreign", good.read_bytes()


def test_unusable_checkpoint_starts_fresh(tmp_path, capsys):
    clean = _run(tmp_path / "clean")
    for kind, blob in _bad_files(tmp_path):
        work = tmp_path / kind
        work.mkdir()
        (work / "checkpoint_b200.npz").write_bytes(blob)
        res = _run(work)
        out = capsys.readouterr().out
        assert "Checkpoint load failed" in out and "Starting fresh" in out, kind
        assert (res.n_reacted, res.n_escaped, res.n_max_steps, res.total_steps) == \
            (clean.n_reacted, clean.n_escaped, clean.n_max_steps, clean.total_steps), kind
        np.testing.assert_array_equal(res.sim_data["outcome"], clean.sim_data["outcome"])
        assert not (work / "checkpoint_b200.npz").exists(), kind


@pytest.mark.parametrize("n", [1, 5])
def test_clean_run_leaves_no_checkpoint(tmp_path, n):
    res = _run(tmp_path, n_traj=n)
    assert res.n_trajectories == n and res.n_reacted + res.n_escaped + res.n_max_steps == n
    assert not (tmp_path / "checkpoint_b200.npz").exists()
