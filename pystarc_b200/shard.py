"""Trajectory sharding across GPUs (one process per GPU).

Trajectories are independent Bernoulli trials, so the path shards with no
data-path exchange: rank r of W runs the contiguous global-id range
``shard_range(n_total, r, W)`` (its ``id_offset`` keys the noise, so results do
not depend on W), and the integer tallies are summed once at the end -- the one
collective, as the reference's process-level combine step pools counts
(pystarc/multi_GPU/combine_data.py:66-87).
"""

from __future__ import annotations

TALLY_KEYS = ("started", "reacted", "escaped", "max_steps", "steps", "returns", "overlap", "bridge")


def shard_range(n_total: int, rank: int, world: int):
    """(id_offset, n_local) of `rank`: contiguous ranges, sizes differing by at most one."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("need 0 <= rank < world")
    base, extra = divmod(int(n_total), int(world))
    n_local = base + (1 if rank < extra else 0)
    offset = rank * base + min(rank, extra)
    return offset, n_local


def allreduce_tallies(tallies: dict, group=None, device=None) -> dict:
    """Sum integer tallies over all ranks (int64 all-reduce; NCCL on GPUs, gloo on CPU)."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([int(tallies.get(k, 0)) for k in TALLY_KEYS], dtype=torch.int64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return dict(zip(TALLY_KEYS, (int(v) for v in t.cpu())))


def allreduce_reaction_fires(discrete, bridge, group=None, device=None):
    """Sum the per-reaction fire counts of state-machine runs over all ranks
    (``B200BatchSimulator.reaction_fires``); returns (discrete, bridge) as lists."""
    import torch
    import torch.distributed as dist

    n = len(discrete)
    t = torch.tensor([int(v) for v in discrete] + [int(v) for v in bridge], dtype=torch.int64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    v = [int(x) for x in t.cpu()]
    return v[:n], v[n:]
