"""Multi-process (world size 2, gloo on CPU) sharding and tally pooling.

Each rank runs its shard of trajectory ids through the oracle stepper with the
engine's keyed noise (the CUDA engine uses the same ids and draws), then the
tallies are all-reduced.  The pooled result must equal one process running every
trajectory, trajectory by trajectory.
"""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from pystarc_b200.shard import TALLY_KEYS, shard_range


def test_shard_ranges_partition_ids():
    for n in (1, 7, 100, 1001):
        for w in (1, 2, 3, 8):
            got = []
            for r in range(w):
                off, m = shard_range(n, r, w)
                got.extend(range(off, off + m))
            assert got == list(range(n))
    with pytest.raises(ValueError):
        shard_range(10, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _run_shard(n_total, rank, world):
    from oracle import stepper as ost
    from tests.helpers import step_params, step_system, system

    s = system("two_sphere")
    off, n = shard_range(n_total, rank, world)
    prm = step_params(s, n, s.seed, 5000)
    res = ost.run(step_system(s), prm, noise="philox", termination="complete", id_offset=off)
    return res


def _worker(rank, world, port, n_total, out):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from pystarc_b200.shard import allreduce_tallies

        res = _run_shard(n_total, rank, world)
        tallies = {"started": len(res.status), "reacted": res.n_reacted, "escaped": res.n_escaped,
                   "max_steps": res.n_max_steps, "steps": res.total_steps, "returns": int(res.n_returns.sum())}
        pooled = allreduce_tallies(tallies)
        out[rank] = (pooled, res.status.tolist(), res.n_steps.tolist())
    finally:
        dist.destroy_process_group()


def test_two_rank_pooling_equals_single_process():
    n_total = 120
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        mp.start_processes(_worker, args=(2, port, n_total, out), nprocs=2, join=True, start_method="spawn")
        results = dict(out)
    single = _run_shard(n_total, 0, 1)
    pooled = results[0][0]
    assert results[1][0] == pooled
    assert pooled["started"] == n_total
    assert pooled["reacted"] == single.n_reacted and pooled["escaped"] == single.n_escaped
    assert pooled["steps"] == single.total_steps
    status = np.array(results[0][1] + results[1][1])
    steps = np.array(results[0][2] + results[1][2])
    np.testing.assert_array_equal(status, single.status)
    np.testing.assert_array_equal(steps, single.n_steps)
    assert set(TALLY_KEYS) >= set(pooled)


def _run_sm_shard(n_total, rank, world):
    from dataclasses import replace

    from oracle import stepper as ost
    from tests.helpers import golden, sm_step_system, step_params, system

    s = system("two_sphere")
    off, n = shard_range(n_total, rank, world)
    prm = replace(step_params(s, n, s.seed, 20000), min_core_rxn_dt=0.05)
    return ost.run(sm_step_system(s, golden("run_sm_two_sphere")), prm, noise="philox", termination="complete",
                   id_offset=off)


def _sm_worker(rank, world, port, n_total, out):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from pystarc_b200.shard import allreduce_reaction_fires

        res = _run_sm_shard(n_total, rank, world)
        out[rank] = allreduce_reaction_fires(res.sm_fires_discrete, res.sm_fires_bridge)
    finally:
        dist.destroy_process_group()


def test_two_rank_state_machine_fire_counts_pool():
    """Per-reaction fire counts of sharded state-machine runs add up to the single-process counts."""
    n_total = 40
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        mp.start_processes(_sm_worker, args=(2, port, n_total, out), nprocs=2, join=True, start_method="spawn")
        results = dict(out)
    single = _run_sm_shard(n_total, 0, 1)
    assert results[0] == results[1]
    assert results[0] == (single.sm_fires_discrete.tolist(), single.sm_fires_bridge.tolist())
    assert sum(results[0][0]) + sum(results[0][1]) > 0


class _FakeHandle:
    """The engine's C entry points as the stepper drives them, answered by the oracle stepper with
    the engine's keyed draws: bd_sim_configure runs the configured shard (n_traj trajectories from
    global id id_offset), the counter and outcome calls copy its results out."""

    def __init__(self, s):
        self.s = s
        self.device = 0
        self.res = None
        self.configured = None

    def call(self, name, *args):
        from oracle import stepper as ost
        from tests.helpers import step_params, step_system

        if name == "bd_sim_configure":
            sp = args[0]._obj
            self.configured = (int(sp.n_traj), int(sp.id_offset))
            prm = step_params(self.s, int(sp.n_traj), int(sp.seed), int(sp.max_steps))
            self.res = ost.run(step_system(self.s), prm, noise="philox", termination="complete",
                               id_offset=int(sp.id_offset))
        elif name == "bd_sim_counters":
            r = self.res
            vals = {"started": len(r.status), "reacted": r.n_reacted, "escaped": r.n_escaped,
                    "max_steps": r.n_max_steps, "steps": r.total_steps, "returns": int(r.n_returns.sum()),
                    "overlap": r.n_overlap_rejected}
            from pystarc_b200 import _lib

            for i, k in enumerate(_lib.CTR_NAMES):
                args[0][i] = int(vals.get(k, 0))
        elif name == "bd_sim_live":
            args[0]._obj.value = 0
        elif name == "bd_sim_outcomes":
            for i in range(len(self.res.status)):
                args[0][i] = int(self.res.status[i])
                args[1][i] = int(self.res.n_steps[i])
                args[2][i] = int(self.res.n_returns[i])
        return 0


class _FakeEngine:
    def __init__(self, s):
        self.handle = _FakeHandle(s)
        self.precision, self.torque_mode, self._debye = "fp64", "zero", s.debye

    def set_ligand(self, body, q):
        pass


def _sim_worker(rank, world, port, n_total, out):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from pystarc_b200.simulator import B200BatchSimulator
        from tests.helpers import system

        s = system("two_sphere")
        mol1, mol2 = s.molecules()
        eng = _FakeEngine(s)
        sim = B200BatchSimulator(mol1, mol2, s.mobility(), s.pathway_set(), s.params(n_traj=n_total, max_steps=5000),
                                 eng, termination="complete")
        res = sim.run(dist=True)
        out[rank] = (res.n_trajectories, res.n_reacted, res.n_escaped, res.n_max_steps, res.total_steps,
                     eng.handle.configured, res.sim_data["shard"], res.sim_data["outcome"].tolist(),
                     res.sim_data["n_steps"].tolist())
    finally:
        dist.destroy_process_group()


def test_simulator_run_shards_and_pools_over_two_ranks():
    """B200BatchSimulator.run(dist=True): each rank configures its contiguous id shard, runs it, and
    the result carries the pooled tallies; fates per global id equal one process running everything."""
    n_total = 101
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        mp.start_processes(_sim_worker, args=(2, port, n_total, out), nprocs=2, join=True, start_method="spawn")
        results = dict(out)
    single = _run_shard(n_total, 0, 1)
    for r in (0, 1):
        n, nr, ne, nm, steps, cfg, shard, _, _ = results[r]
        assert (n, nr, ne, nm, steps) == (n_total, single.n_reacted, single.n_escaped, single.n_max_steps,
                                          single.total_steps)
        assert cfg == (shard["n_local"], shard["id_offset"]) == shard_range(n_total, r, 2)[::-1]
    outcome = np.array(results[0][7] + results[1][7])
    expect = single.status.copy()
    expect[(expect != 1) & (expect != 2)] = 0
    np.testing.assert_array_equal(outcome, expect)
    np.testing.assert_array_equal(np.array(results[0][8] + results[1][8]), single.n_steps)


def _bench_pool_worker(rank, world, port, out):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench

        counters = {k: 10 * (rank + 1) + i for i, k in enumerate(TALLY_KEYS)}
        counters["steps"] = 1000 * (rank + 1)
        out[rank] = bench.pool_over_ranks(dist, None, 2.0 + rank, counters, e2e_seconds=5.0 - rank,
                                          e2e_steps=300 * (rank + 1), h2d=7 + rank, d2h=11 + rank)
    finally:
        dist.destroy_process_group()


def test_bench_pools_time_steps_tallies_and_e2e_over_two_ranks():
    """bench.py under torchrun: time is the slowest rank's, steps, tallies and copied bytes are summed,
    and the end-to-end rate is the summed steps over the slowest rank's end-to-end time."""
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_bench_pool_worker, args=(2, _free_port(), out), nprocs=2, join=True,
                           start_method="spawn")
        res = dict(out)
    t_max, steps, tallies, e2e, h2d, d2h = res[0]
    assert res[0] == res[1]
    assert t_max == 3.0 and steps == 3000
    assert tallies["steps"] == 3000 and tallies["reacted"] == (10 + 1) + (20 + 1)
    assert e2e == 900 / 5.0 and (h2d, d2h) == (15, 23)
