"""Heterogeneous batch: several receptor-ligand systems in one persistent launch.

No reference counterpart: the reference runs one system per process.  Each
system is a configured ``B200BatchSimulator`` (its own engine, grids, atoms,
reactions and parameters; all with the same precision and torque mode).  The
batch shares one slot pool across the systems (``bd_multi_*``): trajectories
of every system are refilled into free slots as others finish, so small and
large systems keep the GPU full together.  Each trajectory runs exactly as in
its own simulator (same keyed noise), and outcomes land in each simulator's
arrays.  The counters are the batch's: state-machine fire counts are summed over
the systems, so the per-system results carry no ``completed_reactions`` record.
"""

from __future__ import annotations

import ctypes as C
import time

import numpy as np

from . import _lib
from .simulator import B200BatchResult


class B200MultiBatch:
    def __init__(self, sims, steps_per_launch=64, launches_per_poll=8, termination="complete"):
        if not sims:
            raise ValueError("at least one simulator")
        if any(getattr(s, "surrogate", None) is not None for s in sims):
            raise ValueError("the heterogeneous batch runs the exact kernels (no surrogate)")
        self.sims = list(sims)
        self.K, self.M = int(steps_per_launch), int(launches_per_poll)
        self.termination = termination
        self.lib = _lib.load()
        self.h = _lib.P()

    def _call(self, name, *args):
        return _lib.check_multi(getattr(self.lib, name)(self.h, *args), self.h)

    def setup(self):
        for s in self.sims:
            s.stats = False
            s._setup()
        arr = (_lib.P * len(self.sims))(*[s.engine.handle.h for s in self.sims])
        self.close()
        h = _lib.P()
        rc = self.lib.bd_multi_create(arr, len(self.sims), C.byref(h))
        _lib.check_multi(rc, None)
        self.h = h

    def counters(self):
        out = np.zeros(_lib.N_CTR, dtype=np.uint64)
        self._call("bd_multi_counters", _lib.ptr(out, C.c_uint64), _lib.N_CTR, None)
        return dict(zip(_lib.CTR_NAMES, (int(v) for v in out)))

    def run(self, max_launches=None):
        """Run every system to completion; one B200BatchResult per system (counters are the batch's).

        A system's ``total_steps`` sums the steps of its trajectories that ended; the batch's own
        step count over all systems, running trajectories included, is ``last_counters["steps"]``."""
        t0 = time.perf_counter()
        self.setup()
        self._call("bd_multi_reset", None)
        t_setup = time.perf_counter() - t0
        N = sum(int(s.params.n_trajectories) for s in self.sims)
        stop_at = int(N * 0.995) if self.termination == "reference" else N
        launches, stalled, last = 0, 0, -1
        while True:
            self._call("bd_multi_run", self.M, self.K, None)
            launches += self.M
            c = self.counters()
            if c["nonfinite"]:
                raise _lib.BdError(_lib.BD_ERR_NAN, f"{c['nonfinite']} trajectories produced a non-finite pose")
            done = c["reacted"] + c["escaped"] + c["max_steps"]
            if done >= stop_at:
                break
            live = C.c_int32()
            self._call("bd_multi_live", C.byref(live))
            if live.value == 0 and c["started"] >= N:
                break
            if c["steps"] == last:
                stalled += 1
                if stalled >= 50:
                    raise _lib.BdError(_lib.BD_ERR_STALL, f"no BD step in {stalled} polls")
            else:
                stalled, last = 0, c["steps"]
            if max_launches is not None and launches >= max_launches:
                break
        c = self.counters()
        elapsed = time.perf_counter() - t0
        # wall seconds of this run: device builds and configuration, then the launches
        self.last_timing = {"setup_s": round(t_setup, 3), "launches_s": round(elapsed - t_setup, 3),
                            "launches": launches}
        results = []
        for s in self.sims:
            st, steps, rets = s.outcomes()
            n = int(s.params.n_trajectories)
            nr, ne = int(np.sum(st == 1)), int(np.sum(st == 2))
            total = int(steps.sum())
            outcome = st.astype(np.int32)
            outcome[(outcome != 1) & (outcome != 2)] = 0
            results.append(B200BatchResult(
                n_trajectories=n, n_reacted=nr, n_escaped=ne, n_max_steps=n - nr - ne,
                reaction_counts={"stage_0": nr}, r_start=float(s.params.r_start), r_escape=float(s.params.r_escape),
                dt=float(getattr(s.params, "dt", 0.2)), elapsed_sec=elapsed,
                steps_per_sec=total / elapsed if elapsed > 0 else 0.0,
                sim_data={"outcome": outcome, "n_steps": steps.astype(np.int64), "n_returns": rets.astype(np.int64)},
                total_steps=total, counters=c))
        self.last_counters = c
        return results

    def close(self):
        if self.h:
            self.lib.bd_multi_destroy(self.h)
            self.h = _lib.P()

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown
            pass
