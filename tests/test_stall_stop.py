"""The reference's stall stop (gpu_batch_simulator.py:1347-1356) in the simulator's host loop.

The device is replaced by a scripted handle whose finished-trajectory count is a function of
the BD steps the pool has taken, so the loop's decisions are checked on CPU: with
``termination="reference"`` the run stops at the first 10,000-step check where more than 95 %
are done and fewer than max(2, N/1000) finished since the previous check.
"""

import numpy as np

from tests.helpers import system


class _ScriptedHandle:
    def __init__(self, n, done_at):
        self.n, self.done_at = n, done_at
        self.device = 0
        self.K = None
        self.launches = 0

    def done(self):
        return min(self.n, self.done_at(self.launches * self.K))

    def call(self, name, *args):
        from pystarc_b200 import _lib

        if name == "bd_sim_run":
            self.launches += int(args[0])
            self.K = int(args[1])
        elif name == "bd_sim_counters":
            d = self.done()
            vals = {"started": self.n, "reacted": d // 2, "escaped": d - d // 2, "steps": self.launches * self.K * 10}
            for i, k in enumerate(_lib.CTR_NAMES):
                args[0][i] = int(vals.get(k, 0))
        elif name == "bd_sim_live":
            args[0]._obj.value = self.n - self.done()
        elif name == "bd_sim_outcomes":
            d = self.done()
            for i in range(self.n):
                args[0][i] = 1 if i < d // 2 else 2 if i < d else 0
                args[1][i] = 1
                args[2][i] = 0
        return 0


class _Engine:
    def __init__(self, handle, s):
        self.handle = handle
        self.precision, self.torque_mode, self._debye = "fp64", "zero", s.debye

    def set_ligand(self, body, q):
        pass


def _run(n, done_at, termination="reference", max_launches=400):
    from pystarc_b200.simulator import B200BatchSimulator

    s = system("two_sphere")
    mol1, mol2 = s.molecules()
    h = _ScriptedHandle(n, done_at)
    sim = B200BatchSimulator(mol1, mol2, s.mobility(), s.pathway_set(), s.params(n_traj=n, max_steps=10 ** 6),
                             _Engine(h, s), termination=termination, steps_per_launch=64, launches_per_poll=8)
    res = sim.run(max_launches=max_launches)
    return sim, res, h.launches * 64


def test_stall_stops_at_the_second_check():
    # 96 % done by step 9,600, then nothing: the check past 10,000 records 960, the one past 20,000 stops
    sim, res, steps = _run(1000, lambda g: min(960, g // 10))
    assert sim.stall_stopped
    assert 20000 <= steps < 20000 + 512
    assert (res.n_reacted, res.n_escaped, res.n_max_steps) == (480, 480, 40)


def test_slow_progress_above_the_threshold_runs_on():
    # past 96 %, 5 finish per 10,000 steps: more than max(2, N/1000) = 2, so no stall stop
    sim, res, steps = _run(1000, lambda g: 960 + 5 * max(0, g - 9600) // 10000 if g >= 9600 else g // 10,
                           max_launches=800)
    assert not sim.stall_stopped and steps >= 800 * 64


def test_no_stall_stop_below_95_percent_or_in_complete_mode():
    sim, _, _ = _run(1000, lambda g: min(900, g // 10))
    assert not sim.stall_stopped
    sim, _, _ = _run(1000, lambda g: min(960, g // 10), termination="complete")
    assert not sim.stall_stopped


def test_stall_threshold_scales_with_n():
    # N = 100,000: the threshold is 100 trajectories between checks (10,240 steps apart here, as the
    # loop polls every 512 steps)
    n = 100_000
    sim, res, steps = _run(n, lambda g: 96_000 + (95 * max(0, g - 9600)) // 10000 if g >= 9600 else g * 10)
    assert sim.stall_stopped and 20000 <= steps < 20000 + 512
    sim, _, _ = _run(n, lambda g: 96_000 + (105 * max(0, g - 9600)) // 10000 if g >= 9600 else g * 10,
                     max_launches=800)
    assert not sim.stall_stopped
    assert np.isfinite(res.steps_per_sec)
