"""The simulator's console reports mirror the reference loop's (gpu_batch_simulator.py:1357-1399,
1491-1510): convergence milestones, a progress line every 10 s, and the closing totals."""

import math

from pystarc_b200.simulator import ProgressLog
from tests.helpers import system
from tests.test_multi_rank import _FakeEngine


def test_milestones_progress_and_final_lines():
    lines = []
    log = ProgressLog(1000, 57.449, 10, t0=0.0, out=lines.append)
    assert log.marks == [100, 200, 300, 400, 500, 600, 700, 800, 900]
    assert math.isclose(log.CONV, 6.022e8, rel_tol=1e-12)
    log.poll(50, 10, 40, now=1.0)
    assert lines == []
    log.poll(100, 20, 80, now=2.0)  # exactly the first milestone
    assert lines[-1].startswith("  -- 10% converged --  P_rxn=0.20000  k_on=") and "[2s]" in lines[-1]
    assert f"k_on={6.022e8 * 57.449 * 0.2:.3e}" in lines[-1]
    log.poll(250, 50, 200, now=3.0)  # past 200: one line for the poll
    assert len(lines) == 2 and lines[-1].startswith("  -- 25% converged --")
    log.poll(260, 52, 208, now=4.0)  # no new milestone, under 10 s
    assert len(lines) == 2
    log.poll(270, 54, 216, now=10.5)  # the 10-second progress line
    assert lines[-1].startswith("  [T]") and "done=270/1,000 (27.0%)" in lines[-1] and "P_rxn=0.20000" in lines[-1]
    log.final(600, 390, 10, 123456, 2.0, 77, True)
    assert lines[-5:] == ["  BD complete: 600 reacted, 390 escaped, 10 max-steps",
                          "  Total steps: 123,456  (61,728 steps/sec)",
                          "  Overlap rejections: 77",
                          f"  Final: P_rxn={600 / 990:.6f}  k_on={6.022e8 * 57.449 * 600 / 990:.4e} M-1 s-1",
                          "  Checkpoint removed (run completed successfully)"]


def test_no_milestones_when_interval_is_zero():
    lines = []
    log = ProgressLog(1000, 1.0, 0, t0=0.0, out=lines.append)
    log.poll(1000, 500, 500, now=1.0)
    assert log.marks == [] and lines == []


def test_verbose_run_prints_the_reports(capsys):
    from pystarc_b200.simulator import B200BatchSimulator

    s = system("two_sphere")
    mol1, mol2 = s.molecules()
    sim = B200BatchSimulator(mol1, mol2, s.mobility(), s.pathway_set(), s.params(n_traj=64, max_steps=5000),
                             _FakeEngine(s), termination="complete", verbose=True)
    res = sim.run()
    out = capsys.readouterr().out
    assert out.startswith("  B200 batch BD: 64 trajectories x up to 5,000 steps\n  D_rel=")
    assert f"return_prob={sim._return_prob:.4f}" in out and f"k_b={sim._k_b:.4f}" in out
    assert f"  BD complete: {res.n_reacted} reacted, {res.n_escaped} escaped, {res.n_max_steps} max-steps" in out
    assert f"  Total steps: {res.total_steps:,}" in out
    assert f"  Final: P_rxn={res.reaction_probability:.6f}" in out
    assert "% converged --" in out
