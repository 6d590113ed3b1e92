"""Launch-shape autotuner for the persistent stepper.

The shapes differ in how a trajectory's step is spread over lanes:
  G = 1, 4, 8, 16, 32  the G lanes of a group share one trajectory's whole step
  G = 64 / 65          each lane owns one trajectory's step logic and the warp
                       sweeps each trajectory's atoms together (65: registers
                       capped at 128 per thread for more resident warps)
and in threads per block.  Which is fastest depends on the ligand size, on how
often trajectories are near the receptor (reverse-Born and overlap sweeps) and
on precision, so the tuner times short bursts of the real stepper on the
configured system and keeps the fastest.  Tuning consumes trajectories; the
simulator is reset afterwards, so results do not depend on it.
"""

from __future__ import annotations

from . import _lib

DEFAULT_CANDIDATES = ((1, 128), (8, 128), (16, 128), (32, 128), (64, 128), (64, 256), (65, 128), (65, 256))


def measure(sim, group, block, K=16, launches=4):
    """BD steps/s of `launches` launches of K steps after one warm-up launch."""
    import torch

    h = sim.engine.handle
    h.call("bd_set_launch", group, block)
    sim._setup()
    h.call("bd_sim_reset", None)
    h.call("bd_sim_run", 1, K, None)
    c0 = sim.read_counters()["steps"]
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record()
    h.call("bd_sim_run", launches, K, None)
    b.record()
    torch.cuda.synchronize()
    c1 = sim.read_counters()["steps"]
    return (c1 - c0) / (a.elapsed_time(b) / 1e3)


def autotune(sim, candidates=DEFAULT_CANDIDATES, K=16, launches=4):
    """Set the fastest (group, block) on ``sim``'s engine; returns (best, {shape: steps/s})."""
    table = {}
    for g, b in candidates:
        try:
            table[(g, b)] = measure(sim, g, b, K, launches)
        except _lib.BdError:
            continue
    best = max(table, key=table.get)
    sim.engine.handle.call("bd_set_launch", best[0], best[1])
    return best, table
