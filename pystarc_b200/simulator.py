"""``B200BatchSimulator``: drop-in for the reference's ``GPUBatchSimulator``.

Constructor and ``run()`` follow pystarc/simulation/gpu_batch_simulator.py:159-318 and
:462-1594; the result has ``GPUBatchResult``'s fields and methods (:45-140), and
``_k_b`` / ``_return_prob`` are set by ``run()`` as the pipeline expects
(pystarc/pipeline/pipeline.py:343-385).

The step loop runs on the GPU: a persistent kernel advances every live
trajectory ``steps_per_launch`` steps per launch with its state in registers,
starts pending trajectories as others finish, and a compaction drops finished
slots between launches; both are replayed from a CUDA graph.  The host only
polls a dozen counters between batches of launches.  Noise is Philox4x32-10
keyed by (seed, trajectory, step), so a run replays exactly and a trajectory's
fate does not depend on the launch shape.

Reaction criteria use the flattened-pairs mode of the reference (all pairs of
all reactions, ``n_needed`` of the first reaction, -1 meaning all pairs).
"""

from __future__ import annotations

import math
import time
from dataclasses import dataclass, field
from pathlib import Path
from typing import Dict

import numpy as np

from . import _lib
from .hostphys import bradius_cover, bridge_d_eff, rate_constant, return_prob_and_kb, wilson_ci


@dataclass
class B200BatchResult:
    """Same fields and methods as the reference's GPUBatchResult (gpu_batch_simulator.py:45-140)."""

    n_trajectories: int
    n_reacted: int
    n_escaped: int
    n_max_steps: int
    reaction_counts: Dict[str, int]
    r_start: float
    r_escape: float
    dt: float
    elapsed_sec: float
    steps_per_sec: float
    sim_data: Dict = None
    total_steps: int = 0
    counters: Dict = field(default_factory=dict)

    @property
    def n_completed(self) -> int:
        return self.n_reacted + self.n_escaped

    @property
    def reaction_probability(self) -> float:
        n = self.n_completed
        return self.n_reacted / n if n > 0 else 0.0

    def reaction_probability_ci(self, confidence: float = 0.95):
        return wilson_ci(self.n_reacted, self.n_escaped, confidence)

    def rate_constant(self, D_rel: float, k_b: float = 0.0) -> float:
        P = self.reaction_probability
        if P == 0.0:
            return 0.0
        return rate_constant(P, D_rel, k_b, self.r_start, self.r_escape)

    def rate_constant_ci(self, D_rel: float, k_b: float = 0.0, confidence: float = 0.95):
        lo, hi = self.reaction_probability_ci(confidence)
        return (rate_constant(lo, D_rel, k_b, self.r_start, self.r_escape),
                rate_constant(hi, D_rel, k_b, self.r_start, self.r_escape))

    def summary(self, D_rel: float, k_b: float = 0.0, confidence: float = 0.95) -> str:
        k = self.rate_constant(D_rel, k_b)
        k_lo, k_hi = self.rate_constant_ci(D_rel, k_b, confidence)
        p = self.reaction_probability
        p_lo, p_hi = self.reaction_probability_ci(confidence)
        pct = int(confidence * 100)
        lines = [f"  Trajectories : {self.n_trajectories:,}",
                 f"  Completed    : {self.n_completed:,}  ({self.n_reacted:,} reacted + {self.n_escaped:,} escaped)"]
        if self.n_max_steps:
            lines.append(f"  Max-steps    : {self.n_max_steps:,}  (excluded)")
        lines += [f"  P_rxn        : {p:.6f}  ({pct}% CI: [{p_lo:.6f}, {p_hi:.6f}])",
                  f"  k_on         : {k:.4e} M-1 s-1", f"  {pct}% CI     : [{k_lo:.4e}, {k_hi:.4e}] M-1 s-1"]
        if k > 0:
            lines.append(f"  log10(k_on)  : {math.log10(k):.3f}")
        lines += [f"  Wall time    : {self.elapsed_sec:.1f} s", f"  BD steps/sec : {self.steps_per_sec:,.0f}",
                  "  Backend      : B200 (sm_100a persistent kernel)"]
        return "\n".join(lines)


class ProgressLog:
    """The reference loop's console reports (gpu_batch_simulator.py:753-761, 1357-1399, 1491-1510).

    ``poll`` prints a "converged" line when the trajectories done pass a milestone (every
    ``conv_interval`` percent of n; the reference tests for equality at each step, this engine
    polls between launches, so the line comes at the first poll at or past the milestone) and
    a progress line every ``every_s`` seconds.  ``final`` prints the closing totals.  The live
    k_on is the reference's CONV * k_b * P, without the return-probability correction of the
    final result.
    """

    CONV = 6.022e23 * 1e-30 / 1e-12 / 1e-3  # A^3/ps -> M^-1 s^-1

    def __init__(self, n, k_b, conv_interval, t0, every_s=10.0, out=print):
        self.n, self.k_b, self.t0, self.every, self.out = int(n), float(k_b), t0, float(every_s), out
        ci = int(conv_interval or 0)
        self.marks = sorted({int(self.n * p / 100) for p in range(ci, 100, ci)}) if ci > 0 else []
        self.last_mark = 0
        self.last_t = t0

    def _k(self, p):
        return self.CONV * self.k_b * p if self.k_b > 0 else 0

    def start(self, max_steps, D_t, dt, dt_rxn, return_prob, r_escape):
        """The run's opening lines (gpu_batch_simulator.py:486-505)."""
        self.out(f"  B200 batch BD: {self.n:,} trajectories x up to {int(max_steps):,} steps")
        self.out(f"  D_rel={D_t:.5f} A2/ps  dt={dt}ps  dt_rxn={dt_rxn}ps")
        self.out(f"  Outer propagator (LMZ): return_prob={return_prob:.4f}  (applied at r_esc={r_escape:.1f}Å)  "
                 f"k_b={self.k_b:.4f} Å³/ps")

    def poll(self, done, reacted, escaped, now=None):
        now = time.perf_counter() if now is None else now
        crossed = [m for m in self.marks if self.last_mark < m <= done]
        n_comp = reacted + escaped
        if crossed:
            self.last_mark = crossed[-1]
            if n_comp > 0:
                p = reacted / n_comp
                self.out(f"  -- {done / self.n * 100:.0f}% converged --  P_rxn={p:.5f}  k_on={self._k(p):.3e}  "
                         f"({reacted:,} react / {escaped:,} esc)  [{now - self.t0:.0f}s]")
        if now - self.last_t >= self.every:
            self.last_t = now
            head = (f"  [T] {now - self.t0:6.0f}s  done={done:,}/{self.n:,} ({done / self.n * 100:.1f}%)  "
                    f"reacted={reacted:,}  escaped={escaped:,}")
            k = self._k(reacted / n_comp) if n_comp > 0 else 0
            if k > 0:
                e = int(math.floor(math.log10(k)))
                self.out(f"{head}  P_rxn={reacted / n_comp:.5f}  k_on={k / 10 ** e:.2f}e{e}")
            else:
                self.out(head)

    def stall(self, trapped, recent):
        self.out(f"  Stall detected: {trapped} trajectories trapped (+{recent} in last 10k steps). Stopping.")

    def final(self, reacted, escaped, max_steps, total_steps, elapsed, overlap, removed_checkpoint):
        sps = total_steps / elapsed if elapsed > 0 else 0
        self.out(f"  BD complete: {reacted} reacted, {escaped} escaped, {max_steps} max-steps")
        self.out(f"  Total steps: {total_steps:,}  ({sps:,.0f} steps/sec)")
        if overlap > 0:
            self.out(f"  Overlap rejections: {overlap:,}")
        if reacted + escaped > 0 and self.k_b > 0:
            p = reacted / (reacted + escaped)
            self.out(f"  Final: P_rxn={p:.6f}  k_on={self._k(p):.4e} M-1 s-1")
        if removed_checkpoint:
            self.out("  Checkpoint removed (run completed successfully)")


def flatten_pairs(pathway_set):
    """All pairs of all reactions; n_needed of the first reaction (gpu_batch_simulator.py:186-205)."""
    rec_idx, lig_idx, cut = [], [], []
    for rxn in pathway_set.reactions:
        for pair in rxn.criteria.pairs:
            rec_idx.append(int(pair.mol1_atom_index))
            lig_idx.append(int(pair.mol2_atom_index))
            cut.append(float(pair.distance_cutoff))
    if pathway_set.reactions:
        nn = pathway_set.reactions[0].criteria.n_needed
        n_needed = len(cut) if (nn < 0 or nn > len(cut)) else nn
    else:
        n_needed = 1
    return rec_idx, lig_idx, np.asarray(cut, dtype=float), n_needed


def state_machine(pathway_set):
    """State-machine reaction tables of ``pathway_set`` (gpu_batch_simulator.py:216-319), or None.

    Active when some reaction carries a ``state_before`` label.  Each reaction with
    pairs contributes its first pair; states are numbered in the reference's order
    (the first state, then each reaction's source and destination as met), an
    unlabelled state is -1, and a state is terminal when no reaction leaves it.
    Returns a dict with the reaction names, labels, state indices and terminal flags.
    """
    reactions = list(pathway_set.reactions)
    if not any(getattr(r, "state_before", None) is not None for r in reactions):
        return None
    names, sb, sa = [], [], []
    for rxn in reactions:
        if not rxn.criteria.pairs:
            continue
        if len(rxn.criteria.pairs) != 1:
            raise ValueError(f"state-machine reaction {rxn.name!r} has {len(rxn.criteria.pairs)} pairs; "
                             "each reaction needs exactly one")
        names.append(rxn.name)
        sb.append(getattr(rxn, "state_before", None))
        sa.append(getattr(rxn, "state_after", None))
    if not names:
        return None
    first = getattr(pathway_set, "first_state", None)
    if first is None:
        first = sb[0]
    index, labels = {}, []

    def idx(label):
        if label is None:
            return -1
        if label not in index:
            index[label] = len(labels)
            labels.append(label)
        return index[label]

    if first is not None:
        idx(first)
    before, after = [], []
    for b, a in zip(sb, sa):
        before.append(idx(b))
        after.append(idx(a))
    sources = set(before)
    terminal = [k not in sources for k in range(len(labels))]
    return {"names": names, "state_before": sb, "state_after": sa, "before": before, "after": after,
            "states": list(labels), "terminal": terminal, "first_state": first}


def zuk_kT_eta(mob):
    """kBT/eta of the RPY coupling: the geometric mean sqrt(D_t1 6 pi a1 D_t2 6 pi a2)
    (pystarc/hydrodynamics/rotne_prager.py:121-122)."""
    a, b = float(mob.radius1), float(mob.radius2)
    return math.sqrt(float(mob.D_trans1) * 6.0 * math.pi * a * float(mob.D_trans2) * 6.0 * math.pi * b)


class B200BatchSimulator:
    """Batched BD of all trajectories on one GPU.

    Extra keyword options (not in the reference): ``precision`` ("fp64" or
    "mixed"), ``torque_mode`` ("zero" or "centroid"), ``termination``
    ("reference": stop once 99.5 % are done, as the reference loop does;
    "complete": run every trajectory to an outcome or to ``max_steps``),
    ``steps_per_launch`` (K), ``launches_per_poll`` and ``hi_mode`` (with
    hydrodynamic interactions: "reference_gpu", the reference GPU stepper's
    line-of-centres D(r), or "zuk", D_t - (2/3) tr M12(r) with the three-regime
    RPY tensor of MobilityTensor, pystarc/hydrodynamics/rotne_prager.py:67-124, :177-200).
    ``verbose`` prints the reference loop's console reports while it runs: convergence
    milestones every ``params.convergence_interval`` percent, progress every 10 s and the
    closing totals (``ProgressLog``).

    With ``termination="reference"`` the run also stops on the reference's stall rule: at
    every STALL_STEPS BD steps of the pool (the reference's loop counter when every
    trajectory starts at once), once more than 95 % are done and fewer than max(2, N/1000)
    finished since the last check; ``stall_stopped`` records it.
    """

    STALL_STEPS = 10000

    def __init__(self, mol1, mol2, mob, pathway_set, params, batch_engine, *, precision=None, torque_mode=None,
                 termination="reference", steps_per_launch=64, launches_per_poll=8, slots=0, id_offset=0,
                 stats=None, surrogate=None, hi_mode="reference_gpu", trace_capacity=None, verbose=False):
        if hi_mode not in ("reference_gpu", "zuk"):
            raise ValueError("hi_mode must be 'reference_gpu' or 'zuk'")
        self.hi_mode = hi_mode
        if not hasattr(batch_engine, "handle"):
            raise TypeError("batch_engine must be a B200ForceEngine")
        self.mol1, self.mol2, self.mob = mol1, mol2, mob
        self.pathway_set = pathway_set
        self.params = params
        self.engine = batch_engine
        self.precision = precision or batch_engine.precision
        self.torque_mode = torque_mode or batch_engine.torque_mode
        self.termination = termination
        self.K = int(steps_per_launch)
        self.M = int(launches_per_poll)
        self.slots = int(slots)
        self.id_offset = int(id_offset)
        self._shard = None  # (rank, world, first global id, local count) of a sharded run
        # per-step statistics for write_all: on when the pipeline attached an output config
        self.stats = bool(getattr(params, "_output_cfg", None) is not None) if stats is None else bool(stats)
        # path / energy traces every save_interval steps (gpu_batch_simulator.py:579-581, :1319-1340): rows
        # kept on the device up to trace_capacity (default 4M rows, 448 MB); the rest are counted as dropped
        cfg = getattr(params, "_output_cfg", None)
        self._save_interval = max(int(getattr(cfg, "save_interval", 10) or 10), 1) if cfg is not None else 10
        self._want_paths = bool(getattr(cfg, "full_paths", True)) if cfg is not None else True
        self._want_energy = bool(getattr(cfg, "energetics", True)) if cfg is not None else True
        if trace_capacity is None:
            trace_capacity = 4_000_000 if (self._want_paths or self._want_energy) else 0
        self.trace_capacity = int(trace_capacity) if self.stats else 0
        self.verbose = verbose
        self.stall_stopped = False
        # (MLPEnsemble, SurrogateSpec): far-field + reverse Born from the learned surrogate inside its trust region
        self.surrogate = surrogate
        c0 = np.asarray(mol2.centroid(), dtype=float)
        self._mol2_pos0 = np.asarray(mol2.positions_array(), dtype=float) - c0
        self._charges = np.asarray(mol2.charges_array(), dtype=float)
        self._N_lig = len(self._charges)
        self._use_hi = bool(getattr(params, "hydrodynamic_interactions", False))
        rec_idx, lig_idx, cut, n_needed = flatten_pairs(pathway_set)
        rec_pos = np.asarray(mol1.positions_array(), dtype=float)
        self._rxn_rec = rec_pos[rec_idx].reshape(-1, 3) if rec_idx else np.zeros((0, 3))
        self._rxn_lig_body = self._mol2_pos0[lig_idx].reshape(-1, 3) if lig_idx else np.zeros((0, 3))
        self._rxn_cutoffs = cut
        self._rxn_n_needed = n_needed
        # state-machine reactions: reaction p is reaction pair p (one pair each)
        self._sm = state_machine(pathway_set)
        self._sm_active = self._sm is not None
        self._return_prob = 0.0
        self._k_b = 0.0
        self._qb_factor = 1.1
        self.counters = {}

    @property
    def _n_run(self):
        """Trajectories this process runs: all of them, or its shard of a sharded run."""
        return int(self.params.n_trajectories) if self._shard is None else self._shard[3]

    @property
    def _offset(self):
        return self.id_offset + (0 if self._shard is None else self._shard[2])

    # ------------------------------------------------------------------
    def _setup(self):
        p = self.params
        D_t = float(self.mob.relative_translational_diffusion())
        D_r = float(self.mob.relative_rotational_diffusion())
        q_rec = float(self.mol1.total_charge())
        q_lig = float(self.mol2.total_charge())
        r_h_rec = float(getattr(self.mob, "radius1", 0.0))
        r_h_lig = float(getattr(self.mob, "radius2", 0.0))
        debye = float(getattr(self.engine, "_debye", 7.858))
        kT = float(getattr(p, "_kT_scale", 1.0))
        self._return_prob, self._k_b = return_prob_and_kb(p.r_start, p.r_escape, q_rec, q_lig, debye, D_t,
                                                          self._use_hi, r_h_rec, r_h_lig, kT)
        # cover-zone boundary (unused by the stepper): 0 for uncharged pairs, 1.05 b when it fails
        # (gpu_batch_simulator.py:183, 394-403)
        self._bradius_cover = 0.0
        if abs(q_rec * q_lig) >= 1e-9:
            try:
                self._bradius_cover = bradius_cover(float(p.r_start), q_rec, q_lig, debye)
            except (OverflowError, ValueError, ZeroDivisionError):
                self._bradius_cover = float(p.r_start) * 1.05
        h = self.engine.handle
        self.engine.set_ligand(self._mol2_pos0, self._charges)
        P = len(self._rxn_cutoffs)
        if P:
            # lever-arm radii default to 1 A when the mobility has none (gpu_batch_simulator.py:644-645)
            d_eff = np.ascontiguousarray(bridge_d_eff(D_t, float(getattr(self.mob, "radius1", 1.0)),
                                                      float(getattr(self.mob, "radius2", 1.0)), self._rxn_rec,
                                                      self._rxn_lig_body), dtype=np.float64)
            rr = np.ascontiguousarray(self._rxn_rec, dtype=np.float64)
            lb = np.ascontiguousarray(self._rxn_lig_body, dtype=np.float64)
            cc = np.ascontiguousarray(self._rxn_cutoffs, dtype=np.float64)
            h.call("bd_set_reactions", P, _lib.ptr(rr), _lib.ptr(lb), _lib.ptr(cc), _lib.ptr(d_eff),
                   int(self._rxn_n_needed))
        else:
            h.call("bd_set_reactions", 0, None, None, None, None, 1)
        if self._sm_active:
            sm = self._sm
            before = np.ascontiguousarray(sm["before"], dtype=np.int32)
            after = np.ascontiguousarray(sm["after"], dtype=np.int32)
            n_states = max(1, len(sm["states"]))
            term = np.zeros(n_states, dtype=np.uint8)
            term[:len(sm["terminal"])] = sm["terminal"]
            h.call("bd_set_reaction_states", len(before), _lib.ptr(before, _lib.C.c_int32),
                   _lib.ptr(after, _lib.C.c_int32), n_states, _lib.ptr(term, _lib.C.c_uint8))
        else:
            h.call("bd_set_reaction_states", 0, None, None, 0, None)
        sp = _lib.BdSimParams()
        sp.n_traj = self._n_run
        sp.seed = int(p.seed if p.seed is not None else 0) & 0xFFFFFFFFFFFFFFFF
        sp.r_start = float(p.r_start)
        sp.r_escape = float(p.r_escape)
        sp.return_prob = float(self._return_prob)
        sp.max_steps = int(min(p.max_steps, 2 ** 31 - 1))
        sp.max_dt = float(getattr(p, "max_dt", 0.0) or 0.0)
        sp.min_core_dt = float(getattr(p, "minimum_core_dt", 0.0) or 0.0)
        sp.min_core_rxn_dt = float(getattr(p, "minimum_core_reaction_dt", 0.0) or 0.0)
        sp.use_hi = int(self._use_hi)
        sp.overlap = int(bool(getattr(p, "_overlap_check", True)))
        sp.D_t = D_t
        sp.D_r = D_r
        sp.q_rec_total = q_rec
        sp.q_lig_total = q_lig
        sp.adt_debye = debye
        sp.r_hydro_rec = r_h_rec
        sp.r_hydro_lig = r_h_lig
        sp.precision = {"fp64": _lib.PREC_FP64, "mixed": _lib.PREC_MIXED}[self.precision]
        sp.torque_mode = {"zero": _lib.TORQUE_ZERO, "centroid": _lib.TORQUE_CENTROID}[self.torque_mode]
        sp.slots = self.slots
        sp.id_offset = self._offset
        sp.stats = int(self.stats)
        sp.save_interval = self._save_interval
        sp.trace_capacity = self.trace_capacity
        sp.hi_mode = _lib.HI_ZUK if self.hi_mode == "zuk" else _lib.HI_REFERENCE_GPU
        sp.hi_kT_eta = zuk_kT_eta(self.mob) if self.hi_mode == "zuk" else 0.0
        h.call("bd_sim_configure", _lib.C.byref(sp))
        if self.surrogate is not None:
            ens, spec = self.surrogate
            h.call("bd_sim_set_surrogate", ens.h, _lib.C.byref(spec.c_params()))
        else:
            h.call("bd_sim_set_surrogate", None, None)
        return D_t

    def read_counters(self):
        out = np.zeros(_lib.N_CTR, dtype=np.uint64)
        self.engine.handle.call("bd_sim_counters", _lib.ptr(out, _lib.C.c_uint64), _lib.N_CTR, None)
        d = dict(zip(_lib.CTR_NAMES, (int(v) for v in out)))
        if self.surrogate is not None:
            s = np.zeros(2, dtype=np.uint64)
            self.engine.handle.call("bd_sim_surrogate_counters", _lib.ptr(s, _lib.C.c_uint64))
            d["surrogate_evals"], d["surrogate_fallbacks"] = int(s[0]), int(s[1])
        return d

    def read_stats(self):
        """Per-step statistics as host arrays (requires ``stats=True``)."""
        N = self._n_run
        P = len(self._rxn_cutoffs)
        L = _lib
        a = {"start_pos": np.zeros((N, 3)), "start_q": np.zeros((N, 4)), "min_dist": np.zeros(N),
             "near_miss_pos": np.zeros((N, 3)), "near_miss_q": np.zeros((N, 4)), "total_time": np.zeros(N),
             "encounter_pos": np.zeros((N, 3)), "encounter_q": np.zeros((N, 4)),
             "step_at_min": np.zeros(N, dtype=np.int32), "encounter_step": np.zeros(N, dtype=np.int32),
             "bridge": np.zeros(N, dtype=np.int8), "radial": np.zeros(L.ST_RAD_BINS, dtype=np.uint64),
             "angular": np.zeros((L.ST_THETA, L.ST_PHI), dtype=np.uint64),
             "milestone_out": np.zeros(L.ST_MILESTONES, dtype=np.uint64),
             "milestone_in": np.zeros(L.ST_MILESTONES, dtype=np.uint64),
             "transition": np.zeros((L.ST_TRANS, L.ST_TRANS), dtype=np.uint64),
             "contact": np.zeros(max(P, 1), dtype=np.uint64), "radial_edges": np.zeros(L.ST_RAD_BINS + 1),
             "transition_edges": np.zeros(L.ST_TRANS + 1), "milestone_radii": np.zeros(L.ST_MILESTONES)}
        out = L.BdStatsOut()
        ctypes_of = {np.float64: L.C.c_double, np.int32: L.C.c_int32, np.int8: L.C.c_int8, np.uint64: L.C.c_uint64}
        for k, v in a.items():
            setattr(out, k, v.ctypes.data_as(L.C.POINTER(ctypes_of[v.dtype.type])))
        self.engine.handle.call("bd_sim_stats", L.C.byref(out))
        a["contact"] = a["contact"][:P]
        return a

    def read_traces(self):
        """Path rows [traj_id, step, x, y, z, q0, q1, q2] and energy rows [traj_id, step, fx, fy, fz, dt]
        recorded every save_interval steps, sorted by (step, traj_id) as the reference appends them,
        and the number of rows that did not fit the trace capacity."""
        n = max(self.trace_capacity, 0)
        path = np.zeros((n, 8))
        energy = np.zeros((n, 6))
        rows, dropped = _lib.C.c_int64(), _lib.C.c_int64()
        self.engine.handle.call("bd_sim_traces", _lib.ptr(path), _lib.ptr(energy), n, _lib.C.byref(rows),
                                _lib.C.byref(dropped))
        k = rows.value
        path, energy = path[:k], energy[:k]
        order = np.lexsort((path[:, 0], path[:, 1]))
        eorder = np.lexsort((energy[:, 0], energy[:, 1]))
        return path[order], energy[eorder], int(dropped.value)

    @staticmethod
    def _per_step(rows):
        """Rows sorted by step as a list with one array per recorded step (the reference's list)."""
        if len(rows) == 0:
            return []
        cut = np.nonzero(np.diff(rows[:, 1]))[0] + 1
        return np.split(rows, cut)

    def sim_data(self, status, steps, rets, total_steps):
        """The reference's ``sim_data`` dict (gpu_batch_simulator.py:1511-1557) from the device statistics.

        ``path_steps`` / ``energy_steps`` hold one array per recorded step (every
        save_interval steps, as the reference records them); rows beyond the trace
        capacity are dropped and counted in ``counters["trace_dropped"]``.
        """
        a = self.read_stats()
        path, energy, dropped = self.read_traces() if self.trace_capacity > 0 else (np.zeros((0, 8)),
                                                                                       np.zeros((0, 6)), 0)
        self.counters["trace_dropped"] = dropped
        if dropped:
            print(f" [b200] {dropped} path/energy rows beyond the trace capacity of {self.trace_capacity} were dropped")
        outcome = status.astype(np.int32)
        outcome[(outcome != 1) & (outcome != 2)] = 0
        rx = np.where(outcome == 1)[0]
        esc = np.where(outcome == 2)[0]
        return {
            "outcome": outcome, "n_steps": steps.astype(np.int64), "start_pos": a["start_pos"],
            "start_q": a["start_q"], "min_dist": a["min_dist"], "step_at_min": a["step_at_min"].astype(np.int64),
            "total_time_ps": a["total_time"], "n_returns": rets.astype(np.int64),
            "bb_triggered": a["bridge"].astype(np.int64), "encounter_pos": a["encounter_pos"][rx],
            "encounter_q": a["encounter_q"][rx], "encounter_traj": rx.astype(np.int64),
            "encounter_step": a["encounter_step"][rx].astype(np.int64),
            "encounter_n_pairs": np.full(len(rx), self._rxn_n_needed, dtype=np.int64),
            "near_miss_pos": a["near_miss_pos"][esc], "near_miss_q": a["near_miss_q"][esc],
            "near_miss_traj": esc.astype(np.int64), "near_miss_dist": a["min_dist"][esc],
            "path_steps": self._per_step(path) if self._want_paths else [],
            "energy_steps": self._per_step(energy) if self._want_energy else [],
            "radial_bins": a["radial_edges"], "radial_counts": a["radial"].astype(np.int64),
            "angular_theta": np.linspace(0, np.pi, _lib.ST_THETA), "angular_phi": np.linspace(0, 2 * np.pi, _lib.ST_PHI),
            "angular_counts": a["angular"].astype(np.int64), "milestone_radii": a["milestone_radii"],
            "milestone_flux_out": a["milestone_out"].astype(np.int64),
            "milestone_flux_in": a["milestone_in"].astype(np.int64),
            "contact_pair_counts": a["contact"].astype(np.int64),
            "contact_total_steps": int(total_steps) if len(self._rxn_cutoffs) else 0,
            "trans_bins": a["transition_edges"], "trans_matrix": a["transition"].astype(np.int64),
        }

    def outcomes(self):
        N = self._n_run
        st = np.zeros(N, dtype=np.int8)
        steps = np.zeros(N, dtype=np.int32)
        rets = np.zeros(N, dtype=np.int32)
        self.engine.handle.call("bd_sim_outcomes", _lib.ptr(st, _lib.C.c_int8), _lib.ptr(steps, _lib.C.c_int32),
                                _lib.ptr(rets, _lib.C.c_int32))
        return st, steps, rets

    def _checkpoint_path(self):
        name = "checkpoint_b200.npz" if self._shard is None else f"checkpoint_b200_rank{self._shard[0]}.npz"
        return Path(getattr(self.params, "_work_dir", "bd_sims")) / name

    def reaction_fires(self):
        """State-machine mode: per-reaction fire counts (discrete test, Brownian bridge) since the reset."""
        n = len(self._sm["names"]) if self._sm_active else 0
        d = np.zeros(max(n, 1), dtype=np.uint64)
        b = np.zeros(max(n, 1), dtype=np.uint64)
        self.engine.handle.call("bd_sim_reaction_fires", _lib.ptr(d, _lib.C.c_uint64), _lib.ptr(b, _lib.C.c_uint64), n)
        return d[:n].astype(np.int64), b[:n].astype(np.int64)

    def save_checkpoint(self, path=None):
        """Slots, counters and outcomes: enough to resume the same trajectories exactly."""
        h = self.engine.handle
        cap = _lib.C.c_int32()
        h.call("bd_sim_capacity", _lib.C.byref(cap))
        C = cap.value
        c = np.zeros(3 * C)
        q = np.zeros(4 * C)
        traj, steps, rets = (np.zeros(C, dtype=np.int32) for _ in range(3))
        status = np.zeros(C, dtype=np.int8)
        live = _lib.C.c_int32()
        ctr = np.zeros(_lib.N_CTR, dtype=np.uint64)
        h.call("bd_sim_snapshot", _lib.ptr(c), _lib.ptr(q), _lib.ptr(traj, _lib.C.c_int32),
               _lib.ptr(steps, _lib.C.c_int32), _lib.ptr(rets, _lib.C.c_int32), _lib.ptr(status, _lib.C.c_int8),
               _lib.C.byref(live), _lib.ptr(ctr, _lib.C.c_uint64))
        state = np.zeros(C, dtype=np.int8)
        h.call("bd_sim_get_states", _lib.ptr(state, _lib.C.c_int8))
        o_st, o_steps, o_rets = self.outcomes()
        path = Path(path or self._checkpoint_path())
        path.parent.mkdir(parents=True, exist_ok=True)
        # uncompressed: the poses are FP64 noise that barely compresses, and a resume should not wait on zlib
        np.savez(path, c=c, q=q, traj=traj, steps=steps, rets=rets, status=status, state=state,
                            n_live=live.value,
                            counters=ctr, out_status=o_st, out_steps=o_steps, out_returns=o_rets,
                            n_traj=self._n_run, seed=int(self.params.seed or 0), cap=C)
        return path

    def load_checkpoint(self, path):
        """Restore a checkpoint written by ``save_checkpoint`` (same system, seed and n_trajectories)."""
        d = np.load(path)
        if int(d["n_traj"]) != self._n_run or int(d["seed"]) != int(self.params.seed or 0):
            raise ValueError(f"{path}: checkpoint is for another run (n_trajectories/seed differ)")
        h = self.engine.handle
        cap = _lib.C.c_int32()
        h.call("bd_sim_capacity", _lib.C.byref(cap))
        if int(d["cap"]) != cap.value:
            raise ValueError(f"{path}: slot capacity {int(d['cap'])} != {cap.value}")
        arr = {}
        for k in d.files:  # each NpzFile lookup reads the member again: one lookup per key
            v = d[k]
            arr[k] = np.ascontiguousarray(v) if v.ndim else v[()]
        h.call("bd_sim_restore", _lib.ptr(arr["c"]), _lib.ptr(arr["q"]), _lib.ptr(arr["traj"], _lib.C.c_int32),
               _lib.ptr(arr["steps"], _lib.C.c_int32), _lib.ptr(arr["rets"], _lib.C.c_int32),
               _lib.ptr(arr["status"], _lib.C.c_int8), int(arr["n_live"]), _lib.ptr(arr["counters"], _lib.C.c_uint64),
               _lib.ptr(arr["out_status"], _lib.C.c_int8), _lib.ptr(arr["out_steps"], _lib.C.c_int32),
               _lib.ptr(arr["out_returns"], _lib.C.c_int32))
        state = np.ascontiguousarray(arr["state"], dtype=np.int8) if "state" in arr else np.zeros(cap.value, np.int8)
        h.call("bd_sim_set_states", _lib.ptr(state, _lib.C.c_int8))

    # ------------------------------------------------------------------
    def run(self, max_launches=None, dist=None) -> B200BatchResult:
        """Run every trajectory; see the class docstring.

        ``dist``: None for one process, or ``True`` (the default process group) or a
        ``torch.distributed`` process group for one process per GPU.  Rank r of W then
        runs the contiguous global-id shard ``shard.shard_range(n, r, W)`` (its ids key
        the noise, so a trajectory's fate does not depend on W), and the tallies, the
        per-reaction fire counts and the wall time (max) are pooled over the ranks once
        at the end, as pystarc/multi_GPU/combine_data.py:66-87 pools separate runs.  The
        result's counts are the pooled ones; ``sim_data`` holds this rank's trajectories
        (local ids, global id = local id + ``sim_data["shard"]["id_offset"]``).
        """
        group = None
        if dist is not None:
            import torch.distributed as td

            from .shard import shard_range

            group = None if dist is True else dist
            rank, world = td.get_rank(group), td.get_world_size(group)
            off, n_local = shard_range(int(self.params.n_trajectories), rank, world)
            self._shard = (rank, world, off, n_local)
        t0 = time.perf_counter()
        if self._n_run == 0:
            result = self._empty_result()
        else:
            result = self._run_local(t0, max_launches)
        if dist is not None:
            result = self._pool(result, group)
        return result

    def _empty_result(self):
        """A shard without trajectories (more ranks than trajectories)."""
        self.counters = {k: 0 for k in _lib.CTR_NAMES}
        sd = {"outcome": np.zeros(0, np.int32), "n_steps": np.zeros(0, np.int64), "n_returns": np.zeros(0, np.int64)}
        return B200BatchResult(n_trajectories=0, n_reacted=0, n_escaped=0, n_max_steps=0, reaction_counts={},
                               r_start=float(self.params.r_start), r_escape=float(self.params.r_escape),
                               dt=float(getattr(self.params, "dt", 0.2)), elapsed_sec=0.0, steps_per_sec=0.0,
                               sim_data=sd, total_steps=0, counters=dict(self.counters))

    def _pool(self, res, group):
        """Sum the shards' tallies and fire counts, take the longest wall time (every rank makes the same
        collective calls in the same order)."""
        import torch
        import torch.distributed as td

        from .shard import allreduce_reaction_fires, allreduce_tallies

        device = torch.device("cuda", self.engine.handle.device) if td.get_backend(group) == "nccl" else None
        c = res.counters
        local = {"started": c.get("started", 0), "reacted": res.n_reacted, "escaped": res.n_escaped,
                 "max_steps": res.n_max_steps, "steps": res.total_steps, "returns": c.get("returns", 0),
                 "overlap": c.get("overlap", 0), "bridge": c.get("bridge", 0)}
        pooled = allreduce_tallies(local, group, device)
        t = torch.tensor([res.elapsed_sec], dtype=torch.float64, device=device)
        td.all_reduce(t, op=td.ReduceOp.MAX, group=group)
        elapsed = float(t.item())
        sd = res.sim_data
        rank, world, off, n_local = self._shard
        sd["shard"] = {"rank": rank, "world": world, "id_offset": self.id_offset + off, "n_local": n_local}
        if self._sm_active:
            n = len(self._sm["names"])
            d, b = self.reaction_fires() if n_local else (np.zeros(n, np.int64), np.zeros(n, np.int64))
            d, b = allreduce_reaction_fires(d, b, group, device)
            sd["completed_reactions"] = [
                {"name": self._sm["names"][i], "n_fired": int(d[i] + b[i]),
                 "state_before": self._sm["state_before"][i], "state_after": self._sm["state_after"][i]}
                for i in range(n)]
        counters = dict(res.counters)
        counters.update(pooled)
        self.counters = counters
        N = int(self.params.n_trajectories)
        return B200BatchResult(n_trajectories=N, n_reacted=pooled["reacted"], n_escaped=pooled["escaped"],
                               n_max_steps=N - pooled["reacted"] - pooled["escaped"],
                               reaction_counts={"stage_0": pooled["reacted"]}, r_start=res.r_start,
                               r_escape=res.r_escape, dt=res.dt, elapsed_sec=elapsed,
                               steps_per_sec=pooled["steps"] / elapsed if elapsed > 0 else 0.0, sim_data=sd,
                               total_steps=pooled["steps"], counters=counters)

    def _run_local(self, t0, max_launches):
        N = self._n_run
        self._setup()
        h = self.engine.handle
        h.call("bd_sim_reset", None)
        ckpt_interval = int(getattr(self.params, "checkpoint_interval", 0) or 0)
        ckpt = self._checkpoint_path()
        if ckpt_interval > 0 and ckpt.exists():
            try:
                self.load_checkpoint(ckpt)
            except Exception as e:  # unreadable, truncated or another run's file (gpu_batch_simulator.py:574-575)
                print(f" Checkpoint load failed: {e}. Starting fresh.")
                h.call("bd_sim_reset", None)
        last_ckpt_done = 0
        launches = 0
        stalled, last_steps = 0, -1
        stop_at = int(N * 0.995) if self.termination == "reference" else N
        # the reference's stall stop (gpu_batch_simulator.py:1349-1356): every STALL_STEPS BD steps of the
        # pool, stop once more than 95 % are done and fewer than max(2, 0.1 % of N) finished since the last check
        next_stall, stall_done = self.STALL_STEPS, 0
        self.stall_stopped = False
        log = ProgressLog(N, self._k_b, getattr(self.params, "convergence_interval", 10), t0) if self.verbose else None
        if log is not None:
            p = self.params
            log.start(p.max_steps, float(self.mob.relative_translational_diffusion()), getattr(p, "dt", None),
                      getattr(p, "dt_rxn", None), self._return_prob, float(p.r_escape))
        while True:
            h.call("bd_sim_run", self.M, self.K, None)
            launches += self.M
            c = self.read_counters()
            if c["nonfinite"]:
                raise _lib.BdError(_lib.BD_ERR_NAN, f"{c['nonfinite']} trajectories produced a non-finite pose")
            done = c["reacted"] + c["escaped"] + c["max_steps"]
            if log is not None:
                log.poll(done, c["reacted"], c["escaped"])
            if ckpt_interval > 0 and done - last_ckpt_done >= ckpt_interval:
                last_ckpt_done = done
                self.save_checkpoint(ckpt)
            if done >= stop_at:
                break
            if self.termination == "reference" and launches * self.K >= next_stall:
                next_stall = (launches * self.K // self.STALL_STEPS + 1) * self.STALL_STEPS
                if done > int(N * 0.95) and done - stall_done < max(2, int(N * 0.001)):
                    self.stall_stopped = True
                    if log is not None:
                        log.stall(N - done, done - stall_done)
                    break
                stall_done = done
            live = _lib.C.c_int32()
            h.call("bd_sim_live", _lib.C.byref(live))
            if live.value == 0 and c["started"] >= N:
                break
            # watchdog: live slots but no step taken for many polls means the device work stopped
            if c["steps"] == last_steps:
                stalled += 1
                if stalled >= 50:
                    raise _lib.BdError(_lib.BD_ERR_STALL, f"no BD step in {stalled} polls with {live.value} live "
                                                          f"slots, {done}/{N} trajectories done")
            else:
                stalled, last_steps = 0, c["steps"]
            if max_launches is not None and launches >= max_launches:
                break
        c = self.read_counters()
        status, steps, rets = self.outcomes()
        elapsed = time.perf_counter() - t0
        n_reacted = int(np.sum(status == 1))
        n_escaped = int(np.sum(status == 2))
        n_max = N - n_reacted - n_escaped
        removed = ckpt_interval > 0 and ckpt.exists()
        if removed:
            ckpt.unlink()
        if log is not None:
            log.final(n_reacted, n_escaped, n_max, int(c["steps"]), elapsed, int(c["overlap"]), removed)
        self.counters = c
        total = int(c["steps"])
        if self.stats:
            sim_data = self.sim_data(status, steps, rets, total)
        else:
            outcome = status.astype(np.int32)
            outcome[(outcome != 1) & (outcome != 2)] = 0
            sim_data = {"outcome": outcome, "n_steps": steps.astype(np.int64), "n_returns": rets.astype(np.int64)}
        if self._sm_active:
            # per-reaction fire counts (gpu_batch_simulator.py:1571-1581)
            d, b = self.reaction_fires()
            sim_data["completed_reactions"] = [
                {"name": self._sm["names"][i], "n_fired": int(d[i] + b[i]),
                 "state_before": self._sm["state_before"][i], "state_after": self._sm["state_after"][i]}
                for i in range(len(self._sm["names"]))]
        return B200BatchResult(n_trajectories=N, n_reacted=n_reacted, n_escaped=n_escaped, n_max_steps=n_max,
                               reaction_counts={"stage_0": n_reacted}, r_start=float(self.params.r_start),
                               r_escape=float(self.params.r_escape), dt=float(getattr(self.params, "dt", 0.2)),
                               elapsed_sec=elapsed, steps_per_sec=total / elapsed if elapsed > 0 else 0.0,
                               sim_data=sim_data, total_steps=total, counters=c)
