"""Autotuner for the stepper's launch shape and device data layout.

The tuned "tile shapes" of the stepper:

* lanes per trajectory and ligand atoms per pass -- the group G:
  G = 1, 4, 8, 16, 32   the G lanes of a group share one trajectory's whole step and sweep
                        its ligand atoms G at a time
  G = 64 / 65           each lane owns one trajectory's step logic and the warp sweeps each
                        trajectory's ligand atoms 32 at a time (65: registers capped at 128
                        per thread for more resident warps)
  G = 66                the split step: ligand atoms as in 64, Born direction 2 in a kernel of
                        its own capped at 64 registers (twice the resident warps)
* trajectories per CTA -- threads per block (128 or 256) divided by the lanes per trajectory;
* the receptor tile of Born direction 2 -- how the ligand Born grid is read: float4 windows of
  4 z-nodes (8 loads per stencil) or 2x2x2 node cubes (4 loads, 8x the grid's memory).
  A third candidate, the default layout, adds the xy records (x face and y edge of a cell half
  in one 32-byte record) and reads the z edge through the texture path: two global loads and
  one texture fetch per stencil.  Every candidate keeps the overlap occupancy grid (one lane per
  overlap test).

Which is fastest depends on the ligand and receptor sizes, on how often trajectories are near
the receptor and on precision, so the tuner times short bursts of the real stepper on the
configured system -- from a saved pool (``aged``: a ``save_checkpoint`` file) when given, so
that it tunes the regime that will be timed, else from fresh trajectories -- and keeps the
fastest.  The simulator is reset afterwards, so results do not depend on it.
"""

from __future__ import annotations

from . import _lib

DEFAULT_CANDIDATES = ((1, 128), (8, 128), (16, 128), (32, 128), (64, 128), (64, 256), (65, 128), (65, 256),
                      (66, 256))
DEFAULT_LAYOUTS = (_lib.LAYOUT_WINDOWS_1 | _lib.LAYOUT_OVERLAP_GRID,
                   _lib.LAYOUT_DEFAULT & ~(_lib.LAYOUT_XY_1 | _lib.LAYOUT_ZTEX_1), _lib.LAYOUT_DEFAULT)


def measure(sim, group, block, K=16, launches=4, aged=None):
    """BD steps/s of `launches` launches of K steps after one warm-up launch."""
    import torch

    h = sim.engine.handle
    h.call("bd_set_launch", group, block)
    sim._setup()
    h.call("bd_sim_reset", None)
    if aged is not None:
        sim.load_checkpoint(aged)
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


def autotune(sim, candidates=DEFAULT_CANDIDATES, K=16, launches=4, layouts=(None,), aged=None):
    """Set the fastest (group, block, layout) on ``sim``'s engine; returns (best, {(group, block, layout):
    steps/s}).  A layout of None keeps the engine's current one."""
    h = sim.engine.handle
    table = {}
    for layout in layouts:
        if layout is None:
            v = _lib.C.c_int32()
            h.call("bd_get_layout", _lib.C.byref(v))
            layout_now = int(v.value)
        else:
            layout_now = int(layout)
            h.call("bd_set_layout", layout_now)
        for g, b in candidates:
            try:
                table[(g, b, layout_now)] = measure(sim, g, b, K, launches, aged)
            except _lib.BdError:
                continue
    best = max(table, key=table.get)
    h.call("bd_set_layout", best[2])
    h.call("bd_set_launch", best[0], best[1])
    return best, table


def autotune_multi(batch, layouts=DEFAULT_LAYOUTS, K=16, launches=4):
    """Heterogeneous batch: time short bursts of the shared persistent launch with each layout applied
    to every system, keep the fastest; returns (best layout, {layout: steps/s})."""
    import torch

    table = {}
    for layout in layouts:
        for s in batch.sims:
            s.engine.handle.call("bd_set_layout", int(layout))
        batch.setup()
        batch._call("bd_multi_reset", None)
        batch._call("bd_multi_run", 1, K, None)
        c0 = batch.counters()["steps"]
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record()
        batch._call("bd_multi_run", launches, K, None)
        b.record()
        torch.cuda.synchronize()
        table[int(layout)] = (batch.counters()["steps"] - c0) / (a.elapsed_time(b) / 1e3)
    best = max(table, key=table.get)
    for s in batch.sims:
        s.engine.handle.call("bd_set_layout", best)
    return best, table
