"""CUDA stepper against the oracle stepper (same keyed Philox draws) and the reference's statistics."""

import numpy as np
import pytest

from oracle import stepper as ost
from tests.helpers import golden, oracle_engine, step_params, step_system, system

pytestmark = pytest.mark.gpu


class _MP:
    def __init__(self, s):
        self.dipole, self.quadrupole, self.four_pi_eps = s.multipole_moments()


def make_sim(s, n_traj, max_steps, precision="fp64", torque="zero", seed=None, layout=None, use_lj=False,
             pathway=None, min_core_rxn_dt=0.0, **kw):
    from pystarc_b200.engine import B200ForceEngine
    from pystarc_b200.simulator import B200BatchSimulator

    lj = dict(rec_radii=s.rec_r, lig_radii=s.lig_r, use_lj=True) if use_lj else {}
    eng = B200ForceEngine(**s.engine_kwargs(), multipole_expansion=_MP(s) if s.multipole else None,
                          precision=precision, torque_mode=torque, layout=layout, **lj)
    mol1, mol2 = s.molecules()
    kw.setdefault("termination", "complete")
    params = s.params(n_traj=n_traj, max_steps=max_steps, seed=seed)
    params.minimum_core_reaction_dt = min_core_rxn_dt
    return B200BatchSimulator(mol1, mol2, s.mobility(), pathway or s.pathway_set(), params, eng, **kw)


def oracle_keyed(s, n_traj, max_steps, torque="zero", seed=None, use_lj=False):
    eng = oracle_engine(s, born_chunk_skip=False, use_lj=use_lj)
    fn = (lambda *a, **k: eng(*a, torque_mode="centroid", **k)) if torque == "centroid" else eng
    return ost.run(step_system(s, fn), step_params(s, n_traj, seed or s.seed, max_steps), noise="philox",
                   termination="complete")


CASES = [("two_sphere", 400, 100000, "zero"), ("c2", 96, 300, "zero"), ("c3", 32, 80, "centroid")]


@pytest.mark.parametrize("group", [None, 66])
@pytest.mark.parametrize("sysname,n,max_steps,torque", CASES)
def test_fp64_trajectories_match_oracle_exactly(sysname, n, max_steps, torque, group):
    s = system(sysname)
    sim = make_sim(s, n, max_steps, "fp64", torque, steps_per_launch=16, launches_per_poll=4)
    if group:
        sim.engine.handle.call("bd_set_launch", group, 0)
    res = sim.run()
    st, steps, rets = sim.outcomes()
    o = oracle_keyed(s, n, max_steps, torque)
    np.testing.assert_array_equal(st, o.status)
    np.testing.assert_array_equal(steps, o.n_steps)
    np.testing.assert_array_equal(rets, o.n_returns)
    assert res.total_steps == o.total_steps
    assert sim._return_prob == o.return_prob and sim._k_b == o.k_b
    assert res.n_reacted == o.n_reacted and res.n_escaped == o.n_escaped


# The reaction-surface dt refinement shrinks dt with the squared height above the surface; with
# no floor (minimum_core_reaction_dt = 0) that height is a difference of nearly equal distances,
# and a 1-ulp change of any input moves about a tenth of the fates (the oracle alone shows it).
# Exact trajectory parity is therefore tested with the floor the reference pipeline sets (0.05 ps);
# without it the test is statistical.
SM_CASES = [("run_sm_two_sphere", "two_sphere", 200, 100000, "zero", 0.05),
            ("run_sm_c2", "c2", 96, 600, "centroid", 0.05)]


def _sm_oracle(s, g, n, max_steps, torque, floor):
    from dataclasses import replace

    from tests.helpers import sm_step_system

    eng = oracle_engine(s, born_chunk_skip=False)
    fn = (lambda *a, **k: eng(*a, torque_mode="centroid", **k)) if torque == "centroid" else eng
    prm = replace(step_params(s, n, s.seed, max_steps), min_core_rxn_dt=floor)
    return ost.run(sm_step_system(s, g, fn), prm, noise="philox", termination="complete")


@pytest.mark.parametrize("name,sysname,n,max_steps,torque,floor", SM_CASES)
def test_state_machine_trajectories_match_oracle_exactly(name, sysname, n, max_steps, torque, floor):
    """State-machine reactions (reference rxns.xml state labels): per trajectory the same fate, step and
    return count as the oracle with the same keyed draws, and the same per-reaction fire counts."""
    from tests.helpers import sm_pathway

    g = golden(name)
    s = system(sysname)
    sim = make_sim(s, n, max_steps, "fp64", torque, pathway=sm_pathway(g), min_core_rxn_dt=floor,
                   steps_per_launch=16, launches_per_poll=4)
    res = sim.run()
    st, steps, rets = sim.outcomes()
    o = _sm_oracle(s, g, n, max_steps, torque, floor)
    np.testing.assert_array_equal(st, o.status)
    np.testing.assert_array_equal(steps, o.n_steps)
    np.testing.assert_array_equal(rets, o.n_returns)
    d, b = sim.reaction_fires()
    np.testing.assert_array_equal(d, o.sm_fires_discrete)
    np.testing.assert_array_equal(b, o.sm_fires_bridge)
    assert ((o.sm_fires_discrete + o.sm_fires_bridge) > 0).sum() >= 2  # the test sees transitions
    rec = res.sim_data["completed_reactions"]
    assert [r["name"] for r in rec] == [str(x) for x in g["rx_names"]]
    assert [r["n_fired"] for r in rec] == list(d + b)
    assert res.n_reacted == o.n_reacted


def test_state_machine_without_dt_floor_is_statistically_the_oracle():
    """No reaction-surface dt floor (ill-conditioned near the surface): most fates agree and the
    reaction probabilities' Wilson intervals overlap."""
    from pystarc_b200.hostphys import wilson_ci
    from tests.helpers import sm_pathway

    g = golden("run_sm_two_sphere")
    s = system("two_sphere")
    n = 200
    sim = make_sim(s, n, 100000, "fp64", pathway=sm_pathway(g), min_core_rxn_dt=0.0, steps_per_launch=16,
                   launches_per_poll=4)
    res = sim.run()
    st, _, _ = sim.outcomes()
    o = _sm_oracle(s, g, n, 100000, "zero", 0.0)
    assert (st == o.status).mean() >= 0.75
    lo_a, hi_a = wilson_ci(res.n_reacted, res.n_escaped)
    lo_b, hi_b = wilson_ci(o.n_reacted, o.n_escaped)
    assert lo_a <= hi_b and lo_b <= hi_a


def test_state_machine_checkpoint_keeps_states(tmp_path):
    """A resumed state-machine run continues every trajectory from its saved state."""
    from tests.helpers import sm_pathway

    g = golden("run_sm_c2")
    s = system("c2")
    kw = dict(pathway=sm_pathway(g), min_core_rxn_dt=float(g["min_core_rxn_dt"]), slots=256, steps_per_launch=8,
              launches_per_poll=1)
    sim = make_sim(s, 200, 600, "fp64", **kw)
    sim._setup()
    sim.engine.handle.call("bd_sim_reset", None)
    sim.engine.handle.call("bd_sim_run", 40, 8, None)  # 320 steps: a few trajectories have left the first state
    path = sim.save_checkpoint(tmp_path / "ck.npz")
    assert np.any(np.load(path)["state"] != 0)
    _run_to_completion(sim, 8)
    a = sim.outcomes()
    sim2 = make_sim(s, 200, 600, "fp64", **kw)
    sim2._setup()
    sim2.engine.handle.call("bd_sim_reset", None)
    sim2.load_checkpoint(path)
    _run_to_completion(sim2, 8)
    for x, y in zip(a, sim2.outcomes()):
        np.testing.assert_array_equal(x, y)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_contact_forces_in_the_stepper(precision):
    """use_lj=True: the stepper's forces include the WCA term, trajectory for trajectory as the oracle's."""
    s = system("c2")
    n, max_steps = 96, 300
    sim = make_sim(s, n, max_steps, precision, use_lj=True, steps_per_launch=16, launches_per_poll=4)
    sim.run()
    st, steps, rets = sim.outcomes()
    o = oracle_keyed(s, n, max_steps, use_lj=True)
    plain = oracle_keyed(s, n, max_steps)
    moved = (o.status != plain.status) | (o.n_steps != plain.n_steps)
    assert moved.any()  # the contact term changes some fates at these sizes
    same = (st == o.status) & (steps == o.n_steps)
    if precision == "fp64":
        assert same.all(), np.flatnonzero(~same)
        np.testing.assert_array_equal(rets, o.n_returns)
    else:
        assert same.mean() >= 0.9, same.mean()


@pytest.mark.parametrize("sysname,n,max_steps,torque", CASES[1:])
def test_mixed_precision_trajectories_mostly_identical(sysname, n, max_steps, torque):
    s = system(sysname)
    sim = make_sim(s, n, max_steps, "mixed", torque, steps_per_launch=16, launches_per_poll=4)
    sim.run()
    st, steps, _ = sim.outcomes()
    o = oracle_keyed(s, n, max_steps, torque)
    same = (st == o.status) & (steps == o.n_steps)
    assert same.mean() >= 0.9, same.mean()


def test_two_sphere_k_on_within_reference_ci():
    """Reference run (2000 trajectories through its own stepper) vs 200k GPU trajectories: Wilson CIs overlap."""
    g = golden("run_two_sphere")
    s = system("two_sphere")
    sim = make_sim(s, 200_000, 1_000_000, "fp64", termination="reference", seed=int(g["seed"]))
    res = sim.run()
    lo, hi = res.reaction_probability_ci()
    rlo, rhi = g["ci"]
    assert lo <= rhi and rlo <= hi, ((lo, hi), (rlo, rhi))
    assert abs(sim._k_b - float(g["k_b"])) < 1e-12


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_every_trajectory_gets_one_outcome(precision):
    s = system("c2")
    N = 5000
    sim = make_sim(s, N, 200, precision, slots=1024, steps_per_launch=8, launches_per_poll=2)
    res = sim.run()
    st, steps, _ = sim.outcomes()
    assert set(np.unique(st)) <= {1, 2, 3}
    assert res.counters["started"] == N
    assert int(steps.sum()) == res.total_steps
    assert res.n_reacted + res.n_escaped + res.n_max_steps == N
    assert res.counters["reacted"] == res.n_reacted and res.counters["escaped"] == res.n_escaped
    assert np.all(steps[st == 3] == 200)


def _run_to_completion(sim, K):
    from pystarc_b200 import _lib

    h = sim.engine.handle
    for _ in range(10000):
        h.call("bd_sim_run", 4, K, None)
        live = _lib.C.c_int32()
        h.call("bd_sim_live", _lib.C.byref(live))
        if live.value == 0 and sim.read_counters()["started"] >= int(sim.params.n_trajectories):
            return
    raise AssertionError("did not complete")


def test_checkpoint_resume_replays_exactly(tmp_path):
    """Resume from a mid-run checkpoint gives every trajectory the same outcome as the uninterrupted run."""
    s = system("c2")
    sim = make_sim(s, 3000, 400, "mixed", slots=512, steps_per_launch=8, launches_per_poll=1)
    sim._setup()
    h = sim.engine.handle
    h.call("bd_sim_reset", None)
    h.call("bd_sim_run", 5, 8, None)
    path = sim.save_checkpoint(tmp_path / "ck.npz")
    _run_to_completion(sim, 8)
    a = sim.outcomes()
    sim2 = make_sim(s, 3000, 400, "mixed", slots=512, steps_per_launch=8, launches_per_poll=1)
    sim2._setup()
    sim2.engine.handle.call("bd_sim_reset", None)
    sim2.load_checkpoint(path)
    _run_to_completion(sim2, 8)
    b = sim2.outcomes()
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)
    assert set(np.unique(a[0])) <= {1, 2, 3}


def test_launch_shape_does_not_change_fates():
    s = system("c2")
    outs = []
    for group, slots in [(4, 300), (16, 2000), (64, 500), (65, 150), (66, 400), (66, 150)]:
        sim = make_sim(s, 600, 250, "fp64", slots=slots, steps_per_launch=4 if group in (4, 65) or slots == 150 else 32)
        sim.engine.handle.call("bd_set_launch", group, 128)
        sim.run()
        outs.append(sim.outcomes())
    for other in outs[1:]:
        for x, y in zip(outs[0], other):
            np.testing.assert_array_equal(x, y)


@pytest.mark.parametrize("precision,group", [("fp64", 64), ("mixed", 65), ("mixed", 8), ("mixed", 66)])
def test_data_layouts_do_not_change_fates(precision, group):
    """Grid windows and the shared-memory receptor table change loads, not values: same fates and counters."""
    from pystarc_b200 import _lib

    s = system("c2")
    outs = []
    for layout in (0, _lib.LAYOUT_DEFAULT, _lib.LAYOUT_WINDOWS_1 | _lib.LAYOUT_WINDOWS_2 | _lib.LAYOUT_STAGE_RECEPTOR,
                   _lib.LAYOUT_CUBES_1 | _lib.LAYOUT_WINDOWS_1, _lib.LAYOUT_DEFAULT & ~_lib.LAYOUT_XY_1,
                   _lib.LAYOUT_DEFAULT & ~_lib.LAYOUT_ZTEX_1, _lib.LAYOUT_DEFAULT | _lib.LAYOUT_XYTEX_1,
                   _lib.LAYOUT_DEFAULT | _lib.LAYOUT_PTEX_2):
        sim = make_sim(s, 800, 250, precision, slots=400, steps_per_launch=16, layout=layout)
        sim.engine.handle.call("bd_set_launch", group, 128)
        res = sim.run()
        outs.append((sim.outcomes(), res.counters))
    for other in outs[1:]:
        for x, y in zip(outs[0][0], other[0]):
            np.testing.assert_array_equal(x, y)
        assert other[1] == outs[0][1]


@pytest.mark.parametrize("sysname,n,max_steps,group", [("c2", 96, 300, 64), ("two_sphere", 300, 100000, 1),
                                                       ("c2", 96, 300, 8), ("c2", 96, 300, 66)])
def test_statistics_match_oracle(sysname, n, max_steps, group):
    """Device statistics (the reference's output-file data) against the oracle with the same draws."""
    s = system(sysname)
    sim = make_sim(s, n, max_steps, "fp64", stats=True, steps_per_launch=16)
    sim.engine.handle.call("bd_set_launch", group, 128)
    res = sim.run()
    sd = res.sim_data
    st = oracle_keyed(s, n, max_steps).stats
    # The device draws its normals with log/sincospi(2u) and the oracle with numpy's
    # log/cos(2*pi*u): the same draws to a few ulps, so poses agree to ~1e-14 and a
    # count moves bins only when a position sits within that of a bin edge.
    np.testing.assert_allclose(sd["start_pos"], st.start_pos, rtol=0, atol=1e-12)
    np.testing.assert_allclose(sd["start_q"], st.start_q, rtol=0, atol=1e-14)
    np.testing.assert_allclose(sd["min_dist"], st.min_dist, rtol=1e-10)
    assert np.mean(sd["step_at_min"] == st.step_at_min) >= 0.97
    np.testing.assert_allclose(sd["total_time_ps"], st.total_time, rtol=1e-9)
    np.testing.assert_array_equal(sd["bb_triggered"], st.bridge)
    for k, mine in [("radial_counts", st.rad_counts), ("angular_counts", st.ang_counts)]:
        assert sd[k].sum() == mine.sum(), k
        assert np.abs(sd[k] - mine).sum() <= 4, (k, np.abs(sd[k] - mine).sum())
    # Milestone 0 is the b-sphere, where every start and return is placed: whether the
    # first step counts as crossing it outward depends on the last bit of |start|.
    d0 = 0
    for k, mine in [("milestone_flux_out", st.ms_out), ("milestone_flux_in", st.ms_in)]:
        d = sd[k].astype(np.int64) - mine
        assert np.abs(d[1:]).sum() <= 4, (k, d)
        assert abs(d[0]) <= 0.05 * (n + res.counters["returns"]) + 2, (k, d)
        d0 += abs(d[0])
    dt = np.abs(sd["trans_matrix"].astype(np.int64) - st.trans).sum()
    assert dt <= 4 + 2 * d0, dt
    P = len(s.pairs)
    assert np.abs(sd["contact_pair_counts"] - st.contact[:P]).sum() <= 2
    assert abs(int(sd["contact_total_steps"]) - int(st.contact_total)) <= 2
    rx = sd["encounter_traj"]
    np.testing.assert_array_equal(sd["encounter_step"], st.enc_step[rx])
    np.testing.assert_allclose(sd["encounter_pos"], st.enc_pos[rx], rtol=1e-10, atol=1e-10)
    esc = sd["near_miss_traj"]
    np.testing.assert_allclose(sd["near_miss_pos"], st.nm_pos[esc], rtol=1e-10, atol=1e-10)


@pytest.mark.parametrize("sysname,n,max_steps,group", [("c2", 96, 300, 64), ("c2", 96, 300, 8), ("c2", 96, 300, 66)])
def test_path_and_energy_traces_match_oracle(sysname, n, max_steps, group):
    """Path and energy rows every save_interval steps (gpu_batch_simulator.py:1319-1340), sorted by
    (step, trajectory) as the reference appends them, against the oracle with the same draws."""
    s = system(sysname)
    sim = make_sim(s, n, max_steps, "fp64", stats=True, steps_per_launch=16, trace_capacity=100_000)
    sim.engine.handle.call("bd_set_launch", group, 128)
    res = sim.run()
    sd = res.sim_data
    st = oracle_keyed(s, n, max_steps).stats
    assert res.counters["trace_dropped"] == 0
    for key, mine in (("path_steps", st.path_steps), ("energy_steps", st.energy_steps)):
        rows = np.vstack(sd[key])
        ref = np.vstack(mine)
        assert rows.shape == ref.shape, (key, rows.shape, ref.shape)
        np.testing.assert_array_equal(rows[:, :2], ref[:, :2])
        np.testing.assert_allclose(rows[:, 2:], ref[:, 2:], rtol=1e-9, atol=1e-10, err_msg=key)
        assert all(len(np.unique(a[:, 1])) == 1 for a in sd[key])  # one array per recorded step
    assert np.all(np.vstack(sd["path_steps"])[:, 1] % 10 == 0)


def test_trace_capacity_drops_and_counts_extra_rows():
    s = system("c2")
    sim = make_sim(s, 96, 300, "fp64", stats=True, steps_per_launch=16, trace_capacity=500)
    res = sim.run()
    rows = np.vstack(res.sim_data["path_steps"])
    assert len(rows) == 500
    assert res.counters["trace_dropped"] > 0


@pytest.mark.parametrize("precision,torque", [("fp64", "zero"), ("mixed", "zero"), ("mixed", "centroid")])
def test_split_stepper_matches_the_fused_stepper(precision, torque):
    """The three-kernel step (ligand forces, Born direction 2 in its own kernel, the rest) sums the same
    terms in the same order as the fused kernel: the same fates, steps, returns and counters.

    With refill (more trajectories than slots) the fused kernel hands pending ids to slots in the order
    its warps reach them, so a refilled trajectory may start at another global step than in the split
    stepper.  Its launch boundaries then fall at other steps of its own, and a launch boundary ends the
    reuse of forces over overlap-rejected steps: the evaluation counters may differ by a few poses while
    every fate, step count and pose stays the same.  Without refill the counters are exact too."""
    s = system("c2")
    for n, slots, exact_evals in ((700, 700, True), (1500, 700, False)):
        outs = []
        for group in (65, 66):
            sim = make_sim(s, n, 400, precision, torque, slots=slots, steps_per_launch=16)
            sim.engine.handle.call("bd_set_launch", group, 256)
            res = sim.run()
            outs.append((sim.outcomes(), res.counters))
        for x, y in zip(outs[0][0], outs[1][0]):
            np.testing.assert_array_equal(x, y)
        for k in ("steps", "reacted", "escaped", "returns", "overlap", "bridge"):
            assert outs[0][1][k] == outs[1][1][k], k
        for k in ("grid_evals", "rev_evals", "ff_evals"):
            a, b = outs[0][1][k], outs[1][1][k]
            if exact_evals:
                assert a == b, k
            else:
                assert abs(a - b) <= 1e-3 * max(a, b), (k, a, b)
        assert outs[0][1]["rev_evals"] > 0
