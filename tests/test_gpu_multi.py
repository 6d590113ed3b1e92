"""Heterogeneous batch: several systems in one pool give each trajectory its single-system fate."""

import numpy as np
import pytest

from tests.helpers import system

pytestmark = pytest.mark.gpu


class _MP:
    def __init__(self, s):
        self.dipole, self.quadrupole, self.four_pi_eps = s.multipole_moments()


def make_sim(s, n_traj, max_steps, precision, seed):
    from pystarc_b200.engine import B200ForceEngine
    from pystarc_b200.simulator import B200BatchSimulator

    eng = B200ForceEngine(**s.engine_kwargs(), multipole_expansion=_MP(s) if s.multipole else None,
                          precision=precision)
    mol1, mol2 = s.molecules()
    return B200BatchSimulator(mol1, mol2, s.mobility(), s.pathway_set(),
                              s.params(n_traj=n_traj, max_steps=max_steps, seed=seed), eng, termination="complete",
                              steps_per_launch=16, launches_per_poll=4)


CASE = [("c2", 300, 300, 11), ("two_sphere", 500, 100000, 12), ("c3", 120, 80, 13)]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_matches_each_system_alone(precision):
    from pystarc_b200.multi import B200MultiBatch

    alone = []
    for name, n, ms, seed in CASE:
        sim = make_sim(system(name), n, ms, precision, seed)
        sim.run()
        alone.append(sim.outcomes())
        sim.engine.close()
    sims = [make_sim(system(name), n, ms, precision, seed) for name, n, ms, seed in CASE]
    batch = B200MultiBatch(sims, steps_per_launch=16, launches_per_poll=4)
    results = batch.run()
    for (name, n, _, _), sim, ref, res in zip(CASE, sims, alone, results):
        got = sim.outcomes()
        for x, y in zip(ref, got):
            np.testing.assert_array_equal(x, y, err_msg=name)
        assert res.n_reacted + res.n_escaped + res.n_max_steps == n
    c = batch.last_counters
    assert c["started"] == sum(n for _, n, _, _ in CASE)
    assert c["steps"] == sum(int(r.total_steps) for r in results)
    batch.close()
    for s in sims:
        s.engine.close()


def test_mixed_precision_modes_are_rejected():
    from pystarc_b200._lib import BdError
    from pystarc_b200.multi import B200MultiBatch

    a = make_sim(system("c2"), 64, 50, "fp64", 1)
    b = make_sim(system("two_sphere"), 64, 50, "mixed", 2)
    with pytest.raises(BdError, match="same precision"):
        B200MultiBatch([a, b]).run()
