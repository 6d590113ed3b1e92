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
