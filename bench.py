"""BD steps/s of the batched rigid-body BD step on B200 (protein + small ligand workload).

Workload: the synthetic protein + small-ligand system (3200-atom receptor in a
22 A ball, +8 e; 18-atom ligand, +1 e; nested 193^3 @ 0.5 A and 129^3 @ 2 A
FP32 electrostatic grids, matching Born grids, a 65^3 ligand Born grid), b = 60 A,
max_dt 20 ps, 1e6 trajectories seeded on the b-sphere.  Data are synthetic
(seeded; no structure files).

One bench "step" = one launch of the persistent stepper: every live
trajectory advances ``--inner`` BD steps (finished ones are replaced from the
pending pool inside the launch), then finished slots are compacted.  The
metric is the reference's BD steps/s: trajectory-steps completed / time.
L2 is flushed (a 256 MiB write) between timed launches, outside the timed
region.

Arms:
  default            the B200 engine (mixed precision, the headline) plus a plain
                     FP64 measurement in the same run
  --impl reference   the reference's batched stepper restated in NumPy (the same
                     algorithm, its own PCG64 draw order) on all host cores
"""

from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "BD steps/sec on 1 B200, surrogate vs plain at k_on within Wilson 95% CI"
UNIT = "BD steps/s"
ALGO_BYTES_PER_GATHER = 224  # 7 trilinear interpolations x 8 corners x 4 B per (atom, grid)
STATE_BYTES_PER_STEP = 128  # FP64 pose read + write and status/counters per trajectory-step


def _find_key(d, key):
    if isinstance(d, dict):
        if key in d and isinstance(d[key], (int, float)):
            return float(d[key])
        for v in d.values():
            r = _find_key(v, key)
            if r is not None:
                return r
    return None


def peaks():
    """The measured HBM copy bandwidth (GB/s) of MEASURED_PEAKS.json, else a fallback of 6,650 GB/s."""
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            v = _find_key(json.loads(p.read_text()), "hbm_gbs")
            if v and v > 0:
                return v, "measured"
        except (OSError, ValueError):
            pass
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.index), "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


WORKLOADS = {
    "protein-ligand": ("protein+small-ligand (3200/18 atoms, 193^3 elec+Born grids, 65^3 ligand Born grid, 1e6 trajectories)", 1_000_000),
    "two-spheres": ("two charged spheres (+5/-5 e, 129^3 grid, 1e5 trajectories, FP64 physics)", 100_000),
    "protein-protein": ("protein-protein (1700/1400 atoms, 3 x 161^3 grids, HI, 1e7 trajectories)", 10_000_000),
    "heterogeneous": ("16 synthetic receptor-ligand systems in one persistent launch (500-8000 / 10-2000 atoms, "
                      "97^3-225^3 grids at 0.5-1.0 A, 1e4-1e6 trajectories each, b 50-90 A)", 0),
}


def build_system(device, workload="protein-ligand"):
    from pystarc_b200 import synth

    if workload == "heterogeneous":
        return synth.config5(0, device=device)
    if workload == "two-spheres":
        return synth.config1()
    if workload == "protein-protein":
        return synth.config3(scale=1.0, device=device)
    return synth.config2(n_traj=1_000_000, scale=1.0, device=device)


class _MP:
    def __init__(self, s):
        self.dipole, self.quadrupole, self.four_pi_eps = s.multipole_moments()


_OPTS = {"layout": None}


def make_sim(s, precision, n_traj, K, id_offset=0, torque="zero", surrogate=None, termination="complete", seed=None,
             slots=0, hi_mode="reference_gpu"):
    from pystarc_b200.engine import B200ForceEngine
    from pystarc_b200.simulator import B200BatchSimulator

    eng = B200ForceEngine(**s.engine_kwargs(), multipole_expansion=_MP(s), precision=precision, torque_mode=torque,
                          device=int(os.environ.get("LOCAL_RANK", 0)), layout=_OPTS["layout"])
    mol1, mol2 = s.molecules()
    sim = B200BatchSimulator(mol1, mol2, s.mobility(), s.pathway_set(), s.params(n_traj=n_traj, seed=seed), eng,
                             termination=termination, steps_per_launch=K, id_offset=id_offset, surrogate=surrogate,
                             slots=slots, hi_mode=hi_mode)
    return sim


def pool_slots(n_traj):
    """One slot-pool size for every arm (8 waves of 512 threads per SM), so aged pools can be restored."""
    import torch

    n_sm = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    return int(min(n_traj, 8 * n_sm * 512))


def age_pool(sim, K, age, path):
    """Advance a fresh pool by ``age`` launches (untimed) and save it, so that every arm times the
    same state past the start-up transient (trajectories start on the b-sphere, where steps are
    cheap; the per-step cost rises several-fold as they reach the receptor)."""
    sim._setup()
    h = sim.engine.handle
    h.call("bd_sim_reset", None)
    for _ in range(age):
        h.call("bd_sim_run", 1, K, None)
    return sim.save_checkpoint(path)


def time_device_arm(s, precision, steps, warmup, K, n_traj, id_offset, dist, fixed_launch=None, aged=None,
                    surrogate=None, candidates=None, hi_mode="reference_gpu"):
    """Per-launch CUDA-event times (graph launches) with L2 flushes in between, from the aged pool."""
    import torch

    from pystarc_b200 import _lib
    from pystarc_b200.autotune import DEFAULT_LAYOUTS, autotune

    sim = make_sim(s, precision, n_traj, K, id_offset, surrogate=surrogate, slots=pool_slots(n_traj), hi_mode=hi_mode)
    table = {}
    if fixed_launch:
        sim.engine.handle.call("bd_set_launch", fixed_launch[0], fixed_launch[1])
    elif surrogate is None:
        # untimed, on the aged pool that is timed below; the run then starts again from it
        layouts = DEFAULT_LAYOUTS if _OPTS["layout"] is None else (_OPTS["layout"],)
        kw = {} if candidates is None else {"candidates": candidates}
        best, table = autotune(sim, layouts=layouts, aged=aged, **kw)
    sim._setup()
    h = sim.engine.handle
    h.call("bd_sim_reset", None)
    if aged is not None:
        sim.load_checkpoint(aged)
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    sptr = _lib.P(stream.cuda_stream)
    for _ in range(warmup):
        h.call("bd_sim_run", 1, K, sptr)
    c0 = sim.read_counters()
    times = []
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    for i in range(steps):
        flush.zero_()
        ev[i][0].record(stream)
        h.call("bd_sim_run", 1, K, sptr)
        ev[i][1].record(stream)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    times = [a.elapsed_time(b) / 1e3 for a, b in ev]
    c1 = sim.read_counters()
    d = {k: c1[k] - c0[k] for k in c1}
    d["started_total"] = c1["started"]
    g = np.zeros(3, dtype=np.int32)
    h.call("bd_get_launch", _lib.ptr(g[0:1], _lib.C.c_int32), _lib.ptr(g[1:2], _lib.C.c_int32),
           _lib.ptr(g[2:3], _lib.C.c_int32))
    lay = np.zeros(1, dtype=np.int32)
    h.call("bd_get_layout", _lib.ptr(lay, _lib.C.c_int32))
    sim.engine.close()
    launch = {"group": int(g[0]), "block": int(g[1]), "grid": int(g[2]), "layout_flags": int(lay[0]),
              "autotune_steps_per_s": {f"{a}x{b}/layout{c}": round(v) for (a, b, c), v in table.items()}}
    return sum(times), times, d, launch


def aged_poses(path, n, seed=7):
    """A sample of running poses (centroids, quaternions) from a saved pool."""
    d = np.load(path)
    C = int(d["cap"])
    live = int(d["n_live"])
    run = np.nonzero(d["status"][:live] == 0)[0]
    rng = np.random.default_rng(seed)
    pick = rng.choice(run, size=min(n, run.size), replace=False)
    c = d["c"].reshape(3, C)[:, pick].T.copy()
    q = d["q"].reshape(4, C)[:, pick].T.copy()
    return c, q


def e2e_arm(s, precision, steps, K, n_traj, id_offset, launch, aged=None):
    """Through the public API with host buffers: the engine is built from host arrays (grid and atom
    uploads); ``run()`` resumes the saved aged pool through its checkpoint mechanism (the slots and
    per-trajectory outcomes are copied to the device), advances ``steps`` launches in the regime the
    device arms time, polling the counters after every launch, and copies the outcomes back.
    Without an aged pool it starts from the b-sphere."""
    import shutil

    import torch

    from pystarc_b200 import _lib

    work = tempfile.mkdtemp(prefix="bench_e2e_")
    steps0, h2d_pool = 0, 0
    if aged is not None:
        shutil.copy(aged, os.path.join(work, "checkpoint_b200.npz"))
        with np.load(aged) as d:
            steps0 = int(d["counters"][_lib.CTR_NAMES.index("steps")])
            h2d_pool = sum(d[k].nbytes for k in ("c", "q", "traj", "steps", "rets", "status", "state", "counters",
                                                  "out_status", "out_steps", "out_returns"))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    sim = make_sim(s, precision, n_traj, K, id_offset, slots=pool_slots(n_traj))
    torch.cuda.synchronize()
    t_engine = time.perf_counter() - t0
    if aged is not None:
        sim.params.checkpoint_interval = 1 << 60  # resume the saved pool; never write a new checkpoint
        sim.params._work_dir = work
    sim.engine.handle.call("bd_set_launch", launch[0], launch[1])
    sim.M = 1
    res = sim.run(max_launches=steps)
    torch.cuda.synchronize()
    el = time.perf_counter() - t0
    h2d = sum(np.asarray(g.data).nbytes for g in s.elec_grids[:1] + s.born_grids[:1] + s.lig_born_grids)
    h2d += np.asarray(s.elec_grids[0].data).nbytes * 2  # interleaved elec+Born copy of the shared lattice
    h2d += (len(s.rec_q) + len(s.lig_q)) * 32 + h2d_pool
    d2h = n_traj * 9 + steps * (_lib.N_CTR * 8 + 4)  # outcomes, and the counters and live count of every poll
    sim.engine.close()
    shutil.rmtree(work, ignore_errors=True)
    launches = max(1, steps)
    res.e2e_split = {"engine_s": round(t_engine, 3), "run_s": round(el - t_engine, 3)}
    res.e2e_steps, res.e2e_seconds = res.total_steps - steps0, el
    return (res.total_steps - steps0) / el, h2d / launches, d2h / launches, res


def surrogate_arm(s, steps, warmup, K, n_traj, n_poses, train_steps, members, kon_traj, kon_launches=1500, log=None,
                  aged=None, n_held=100_000, hi_mode="reference_gpu", r_hi=None, terms=None, sample_traj=None):
    """Config 4: train the surrogate on exact-kernel BD poses, evaluate it on held-out poses, time the
    surrogate stepper like the exact one, and compare k_on of exact and surrogate runs (each run to the
    reference's stopping rule, 99.5 % of the trajectories ended)."""
    import torch

    from pystarc_b200 import surrogate as sg

    out = {}
    t0 = time.perf_counter()
    say = log or (lambda m: None)
    from pystarc_b200 import _lib

    terms = (_lib.TERM_FARFIELD | _lib.TERM_REV_BORN) if terms is None else int(terms)
    r_lo, r_hi = 25.0, min(80.0, float(s.r_escape)) if r_hi is None else float(r_hi)
    # the poses come from fresh trajectories (all live at once) in their first few launches
    n_s = sample_traj or n_traj
    sampler = make_sim(s, "mixed", n_s, 16, slots=n_s, hi_mode=hi_mode)
    c, q = sg.sample_poses(sampler, n_poses + n_held, r_lo=r_lo, r_hi=r_hi, max_seconds=300.0)
    say(f"surrogate: {len(c)} poses sampled in {time.perf_counter() - t0:.1f} s")
    eng = sampler.engine
    eng.set_ligand(s.lig_pos - s.lig_pos.mean(axis=0), s.lig_q)
    T = sg.exact_targets(eng, c, q, precision="mixed", terms=terms)
    eng.close()
    out["data_s"] = round(time.perf_counter() - t0, 1)
    say(f"surrogate: exact targets, {out['data_s']} s with the sampling")
    centres, width = sg.rbf_default(r_lo, r_hi)
    spec = sg.SurrogateSpec(r_scale=max(80.0, r_hi), rbf_centres=centres, rbf_width=width, terms=terms)
    spec.r_min = sg.contact_distance(s.rec_pos, s.lig_pos) + 8.0
    spec.r_max = r_hi
    ens = sg.MLPEnsemble(n_members=members, seed=20261203)
    rep = sg.fit(ens, spec, c[:n_poses], q[:n_poses], T[:n_poses], steps=train_steps, batch=8192, lr=1e-3, log=log)
    out["training"] = {"poses": int(n_poses), "steps": rep.steps, "batch": rep.batch, "members": members,
                       "seconds": round(rep.seconds, 2), "final_loss": [round(v, 6) for v in rep.final_loss],
                       "tflops": round(members * train_steps * rep.batch * 3 * 2 *
                                       sum(i * o for i, o in ens.dims) / rep.seconds / 1e12, 1)}
    out["heldout"] = sg.heldout_error(ens, spec, c[n_poses:], q[n_poses:], T[n_poses:])
    trusted = spec.trusted(c[n_poses:])
    if trusted.any():
        ch, qh, Th = c[n_poses:][trusted], q[n_poses:][trusted], T[n_poses:][trusted]
        out["heldout_trust_region"] = sg.heldout_error(ens, spec, ch, qh, Th)
    say(f"surrogate: trained in {rep.seconds:.1f} s, held-out {out['heldout']}")
    out["trust_region_A"] = [round(spec.r_min, 2), round(spec.r_max, 2)]
    out["terms"] = {6: "far-field + reverse Born", 7: "grid + far-field + reverse Born (total force)"}.get(terms, terms)
    # timed like the exact arm: graph launches of K steps, L2 flushed in between
    sim = make_sim(s, "mixed", n_traj, K, surrogate=(ens, spec), slots=pool_slots(n_traj), hi_mode=hi_mode)
    sim._setup()
    h = sim.engine.handle
    h.call("bd_sim_reset", None)
    if aged is not None:
        sim.load_checkpoint(aged)
    stream = torch.cuda.current_stream()
    sptr = _lib_P(stream.cuda_stream)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    for _ in range(warmup):
        h.call("bd_sim_run", 1, K, sptr)
    c0 = sim.read_counters()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    torch.cuda.synchronize()
    for i in range(steps):
        flush.zero_()
        ev[i][0].record(stream)
        h.call("bd_sim_run", 1, K, sptr)
        ev[i][1].record(stream)
    torch.cuda.synchronize()
    t = sum(a.elapsed_time(b) for a, b in ev) / 1e3
    c1 = sim.read_counters()
    d = {k: c1[k] - c0[k] for k in c1}
    sim.engine.close()
    out["bd_steps_per_s"] = d["steps"] / t
    out["surrogate_share"] = d["surrogate_evals"] / max(d["steps"], 1)
    out["fallback_fraction"] = d["surrogate_fallbacks"] / max(d["surrogate_evals"], 1)
    out["counters"] = {k: int(v) for k, v in d.items()}
    say(f"surrogate: stepper {out['bd_steps_per_s']:.3e} steps/s, fallback {out['fallback_fraction']:.3f}")
    # k_on: the same trajectories (seed, keyed noise) with and without the surrogate, each run until the
    # reference's stopping rule (99.5 % ended) or kon_launches launches, whichever comes first; the
    # trajectories still running then count as max-steps in both
    kon = {}
    D_rel = s.mobility().relative_translational_diffusion()
    for name, sur in (() if kon_traj <= 0 else (("plain", None), ("surrogate", (ens, spec)))):
        sm = make_sim(s, "mixed", kon_traj, K, surrogate=sur, termination="reference", seed=4242)
        t1 = time.perf_counter()
        res = sm.run(max_launches=kon_launches)
        lo, hi = res.reaction_probability_ci()
        kon[name] = {"n": int(kon_traj), "reacted": int(res.n_reacted), "escaped": int(res.n_escaped),
                     "p_rxn": res.n_reacted / max(res.n_reacted + res.n_escaped, 1), "wilson95": [lo, hi],
                     "k_on": res.rate_constant(D_rel, sm._k_b), "k_on_wilson95": list(res.rate_constant_ci(D_rel, sm._k_b)),
                     "max_steps_or_unfinished": int(kon_traj - res.n_reacted - res.n_escaped),
                     "wall_s": round(time.perf_counter() - t1, 1)}
        say(f"surrogate: k_on run {name}: {kon[name]}")
        sm.engine.close()
    if kon:
        a, b = kon["plain"]["wilson95"], kon["surrogate"]["wilson95"]
        kon["cis_overlap"] = bool(a[0] <= b[1] and b[0] <= a[1])
        out["k_on"] = kon
    ens.close()
    return out


PP_CANDIDATES = ((65, 256), (66, 256))


def protein_protein_section(args, log):
    """Config 3 beside the headline: plain FP64, mixed precision, and mixed + surrogate, each timed
    like the headline arms on an aged protein-protein pool (Zuk RPY mobility).  The pool is a
    sample of the 1e7-trajectory workload (``--pp-traj`` trajectories, all live at once, aged
    ``--pp-age`` launches) so that the section takes about a minute."""
    from pystarc_b200 import synth

    t0 = time.perf_counter()
    s = synth.config3(scale=1.0, device="cuda")
    n = args.pp_traj
    work = tempfile.mkdtemp(prefix="bench_pp_")
    ager = make_sim(s, "mixed", n, args.inner, slots=pool_slots(n), hi_mode="zuk")
    aged = age_pool(ager, args.inner, args.pp_age, os.path.join(work, "aged.npz"))
    ager.engine.close()
    log(f"protein-protein: system and {args.pp_age}-launch aging in {time.perf_counter() - t0:.1f} s")
    out = {"workload": WORKLOADS["protein-protein"][0].replace("HI", "Zuk RPY HI"),
           "timed_pool": f"{n} trajectories aged {args.pp_age} launches of {args.inner} BD steps"}
    for prec in ("mixed", "fp64"):
        t, _, d, launch = time_device_arm(s, prec, args.pp_steps, args.warmup, args.inner, n, 0, None, aged=aged,
                                          candidates=PP_CANDIDATES, hi_mode="zuk")
        out[prec] = {"bd_steps_per_s": d["steps"] / t, "steps": int(d["steps"]), "launch": launch,
                     "rev_stencils_per_step": d["rev_evals"] / max(d["steps"], 1),
                     "grid_stencils_per_step": d["grid_evals"] / max(d["steps"], 1)}
        log(f"protein-protein {prec}: {d['steps'] / t:.3e} steps/s")
    out["mixed_over_fp64"] = out["mixed"]["bd_steps_per_s"] / out["fp64"]["bd_steps_per_s"]
    if args.pp_surrogate and not args.no_surrogate:
        sur = surrogate_arm(s, args.pp_steps, args.warmup, args.inner, n, args.pp_sur_poses, args.pp_sur_train_steps,
                            args.sur_members, kon_traj=0, log=log, aged=aged, n_held=20_000, hi_mode="zuk")
        out["surrogate"] = sur
        out["surrogate_over_fp64"] = sur["bd_steps_per_s"] / out["fp64"]["bd_steps_per_s"]
    import shutil

    shutil.rmtree(work, ignore_errors=True)
    out["seconds"] = round(time.perf_counter() - t0, 1)
    return out


def hetero_arm(systems, precision, steps, warmup, K):
    """BD steps/s of the 16-system batch: graph launches of K steps, L2 flushed in between."""
    import torch

    from pystarc_b200.multi import B200MultiBatch

    from pystarc_b200.autotune import autotune_multi

    sims = [make_sim(s, precision, s.n_traj, K) for s in systems]
    batch = B200MultiBatch(sims, steps_per_launch=K)
    best_layout, tune = autotune_multi(batch)  # untimed; the timed run below starts fresh
    batch.setup()
    batch._call("bd_multi_reset", None)
    stream = torch.cuda.current_stream()
    sptr = _lib_P(stream.cuda_stream)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    for _ in range(warmup):
        batch._call("bd_multi_run", 1, K, sptr)
    c0 = batch.counters()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    torch.cuda.synchronize()
    for i in range(steps):
        flush.zero_()
        ev[i][0].record(stream)
        batch._call("bd_multi_run", 1, K, sptr)
        ev[i][1].record(stream)
    torch.cuda.synchronize()
    t = sum(a.elapsed_time(b) for a, b in ev) / 1e3
    c1 = batch.counters()
    batch.close()
    for sm in sims:
        sm.engine.close()
    d = {k: c1[k] - c0[k] for k in c1}
    d["autotune"] = {"layout": best_layout, "steps_per_s": {f"layout{k}": round(v) for k, v in tune.items()}}
    return t, d


def hetero_main(args):
    import torch

    from pystarc_b200 import synth

    t0 = time.perf_counter()
    systems = [synth.config5(i, device="cuda") for i in range(16)]
    _progress(f"16 systems built in {time.perf_counter() - t0:.1f} s")
    clocks = Clocks(0)
    clocks.start()
    t_mixed, d_mixed = hetero_arm(systems, "mixed", args.steps, args.warmup, args.inner)
    ck = clocks.stop()
    t_fp64, d_fp64 = hetero_arm(systems, "fp64", args.steps, args.warmup, args.inner)
    _progress(f"mixed {d_mixed['steps'] / t_mixed:.3e}, fp64 {d_fp64['steps'] / t_fp64:.3e} steps/s")
    # end to end through the public API (engines built from host arrays inside the timed region)
    from pystarc_b200.multi import B200MultiBatch

    torch.cuda.synchronize()
    _OPTS["layout"] = d_mixed["autotune"]["layout"]  # the tuned layout, through the public API
    te = time.perf_counter()
    sims = [make_sim(s, "mixed", s.n_traj, args.inner) for s in systems]
    t_eng = time.perf_counter() - te
    batch = B200MultiBatch(sims, steps_per_launch=args.inner, launches_per_poll=1)
    res = batch.run(max_launches=max(args.steps, 20))
    torch.cuda.synchronize()
    t_all = time.perf_counter() - te
    # every BD step of the run, from the batch's counters (a system's result counts only the steps of
    # its trajectories that ended)
    e2e = batch.last_counters["steps"] / t_all
    batch.close()
    h2d = sum(np.asarray(g.data).nbytes for s in systems for g in s.elec_grids + s.born_grids + s.lig_born_grids)
    d2h = sum(s.n_traj * 9 for s in systems)
    peak, peak_kind = peaks()
    gathers = d_mixed["grid_evals"] + d_mixed["rev_evals"]
    achieved = (gathers * ALGO_BYTES_PER_GATHER + d_mixed["steps"] * STATE_BYTES_PER_STEP) / t_mixed / 1e9
    line = {
        "metric": METRIC, "value": d_mixed["steps"] / t_mixed, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * t_mixed / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 forces / f64 poses", "data": "synthetic",
        "config": {"workload": WORKLOADS["heterogeneous"][0], "bd_steps_per_launch": args.inner,
                   "systems": [s.meta | {"n_traj": s.n_traj} for s in systems],
                   "l2": "flushed (256 MiB write) between launches", "parallelism": "one persistent launch"},
        "variants": {"fp64": {"bd_steps_per_s": d_fp64["steps"] / t_fp64, "steps": d_fp64["steps"]}},
        "counters": {k: int(v) for k, v in d_mixed.items() if k != "autotune"},
        "autotune": d_mixed["autotune"],
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "peak_kind": peak_kind,
                     "algorithmic_bytes": "224 B per (atom, grid) stencil + 128 B per trajectory-step"},
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": int(h2d / max(args.steps, 20)),
                "d2h_bytes_per_step": int(d2h / max(args.steps, 20)),
                "note": "B200ForceEngine x16 + B200MultiBatch.run() from host arrays, incl. grid upload",
                "seconds": {"engines_s": round(t_eng, 3), "run_s": round(t_all - t_eng, 3),
                            **getattr(batch, "last_timing", {})}},
        "gpu_launches": 3 * args.steps,
        "clocks": ck,
    }
    if not args.no_cpu_baseline:
        _, info = cpu_baseline(systems[0], os.cpu_count() or 1, n_steps=args.cpu_steps)
        info["sample"] = "system 0 of the batch only: " + info["sample"]
        line["cpu_baseline"] = info
    print(json.dumps(line))


def _progress(msg):
    print(f"[bench {time.strftime('%H:%M:%S')}] {msg}", file=sys.stderr, flush=True)


def _lib_P(v):
    from pystarc_b200 import _lib

    return _lib.P(v)


# --------------------------------------------------------------------------- CPU baseline
def oracle_system(grid_file, n_traj, seed, n_steps):
    """The oracle's (StepSystem, StepParams) of a system saved by ``save_cpu_inputs``."""
    from oracle import stepper as ost
    from oracle.forces import FarField, OracleForceEngine, OracleGrid

    d = np.load(grid_file, allow_pickle=False)
    grids = lambda k: [OracleGrid(d[f"{k}{i}_data"].astype(np.float64), d[f"{k}{i}_origin"], d[f"{k}{i}_sp"])
                       for i in range(int(d[f"n_{k}"]))]
    ff = FarField(float(d["Q"]), float(d["debye"]), float(d["sdie"]), d["dip"], d["quad"], float(d["fpe"]))
    eng = OracleForceEngine(grids("elec"), grids("born"), float(d["alpha"]), ff, grids("lig_born"), d["rec_pos"],
                            d["rec_q"])
    P = len(d["pair_cut"])
    ss = ost.StepSystem(lig_body=d["lig_body"], lig_q=d["lig_q"], rec_pos=d["rec_pos"], engine=eng,
                        rxn_rec_pos=d["pair_rec"].reshape(P, 3), rxn_lig_idx=d["pair_lig"], rxn_cutoff=d["pair_cut"],
                        n_needed=int(d["n_needed"]), D_t=float(d["D_t"]), D_r=float(d["D_r"]),
                        r_h_rec=float(d["r_h_rec"]), r_h_lig=float(d["r_h_lig"]), q_rec_total=float(d["Q"]),
                        q_lig_total=float(d["q_lig"]), debye=float(d["debye"]))
    prm = ost.StepParams(n_traj=n_traj, seed=seed, r_b=float(d["r_b"]), r_esc=float(d["r_esc"]), max_steps=n_steps,
                         max_dt=float(d["max_dt"]), use_hi=bool(d["hi"]), overlap=bool(d["overlap"]))
    return ss, prm


def _cpu_worker(args):
    grid_file, n_traj, seed, n_steps, init = args
    from oracle import stepper as ost

    ss, prm = oracle_system(grid_file, n_traj, seed, n_steps)
    t0 = time.perf_counter()
    res = ost.run(ss, prm, noise="pcg64", termination="reference", init=init)
    return res.total_steps, time.perf_counter() - t0


def save_cpu_inputs(s, path):
    mob = s.mobility()
    dip, quad, fpe = s.multipole_moments()
    arr = dict(Q=float(np.sum(s.rec_q)), q_lig=float(np.sum(s.lig_q)), debye=s.debye, sdie=s.sdie, dip=dip, quad=quad,
               fpe=fpe, alpha=s.alpha, rec_pos=s.rec_pos, rec_q=s.rec_q, lig_body=s.lig_pos - s.lig_pos.mean(0),
               lig_q=s.lig_q, pair_rec=np.array([s.rec_pos[a] for a, _, _ in s.pairs]),
               pair_lig=np.array([b for _, b, _ in s.pairs]), pair_cut=np.array([c for _, _, c in s.pairs]),
               n_needed=s.n_needed, D_t=mob.relative_translational_diffusion(),
               D_r=mob.relative_rotational_diffusion(), r_h_rec=s.r_hydro_rec, r_h_lig=s.r_hydro_lig,
               r_b=s.r_start, r_esc=s.r_escape, max_dt=s.max_dt, hi=s.hi, overlap=s.overlap)
    for k, gl in (("elec", s.elec_grids), ("born", s.born_grids), ("lig_born", s.lig_born_grids)):
        arr[f"n_{k}"] = len(gl)
        for i, g in enumerate(gl):
            arr[f"{k}{i}_data"] = np.asarray(g.data, dtype=np.float32)
            arr[f"{k}{i}_origin"] = np.asarray(g.origin)
            arr[f"{k}{i}_sp"] = np.asarray([g.delta[j, j] for j in range(3)])
    np.savez(path, **arr)


def force_error_check(s, c, q):
    """Force and torque error of the engine against the FP64 oracle on the poses (c, q), both
    precisions: plain relative error ||F - F_ref|| / ||F_ref|| (max, p99) and the tested metric
    of ``oracle.forces.force_error``.  The oracle is the checker here, never the thing timed."""
    from oracle.forces import FarField, OracleForceEngine, OracleGrid, force_error
    from oracle.stepper import rotmats
    from pystarc_b200.engine import B200ForceEngine

    dip, quad, fpe = s.multipole_moments()
    ff = FarField(float(np.sum(s.rec_q)), s.debye, s.sdie, dip, quad, fpe)
    oe = OracleForceEngine([OracleGrid.from_dx(g) for g in s.elec_grids], [OracleGrid.from_dx(g) for g in s.born_grids],
                           s.alpha, ff, [OracleGrid.from_dx(g) for g in s.lig_born_grids] or None, s.rec_pos, s.rec_q,
                           born_chunk_skip=False)
    body = s.lig_pos - s.lig_pos.mean(axis=0)
    R = rotmats(q)
    pos = np.einsum("nij,kj->nki", R, body) + c[:, None, :]
    Fo, To, _, scale = oe(pos, s.lig_q, R, c, torque_mode="centroid", return_scale=True)
    out = {"poses": int(len(c)), "poses_from": "the GPU arm's aged pool", "reference": "FP64 oracle of "
           "GPUBatchForceEngine.__call__ on identical poses (torque about the centroid)"}
    nf, nt = np.linalg.norm(Fo, axis=1), np.linalg.norm(To, axis=1)
    okf, okt = nf > 1e-6 * np.median(nf), nt > 1e-6 * np.median(nt)
    lever = float(np.max(np.linalg.norm(body, axis=1)))
    for prec in ("fp64", "mixed"):
        eng = B200ForceEngine(**s.engine_kwargs(), multipole_expansion=_MP(s), precision=prec, torque_mode="centroid",
                              device=int(os.environ.get("LOCAL_RANK", 0)))
        eng.set_ligand(body, s.lig_q)
        F, T, _ = eng.eval_poses(c, q)
        eng.close()
        pf = np.linalg.norm(F - Fo, axis=1)[okf] / nf[okf]
        pt = np.linalg.norm(T - To, axis=1)[okt] / nt[okt]
        out[prec] = {"force_rel_max": float(pf.max()), "force_rel_p99": float(np.percentile(pf, 99)),
                     "torque_rel_max": float(pt.max()), "torque_rel_p99": float(np.percentile(pt, 99)),
                     "force_metric_max": float(force_error(F, Fo, scale).max()),
                     "torque_metric_max": float(force_error(T, To, scale * lever).max())}
    return out


def cpu_baseline(s, cores, traj_per_proc=256, n_steps=40, init=None, where=None):
    """The reference's step loop restated in NumPy on `cores` processes, each a bounded sample.

    ``init`` = (centroids, quaternions): start the processes' trajectories from these poses (a
    sample of the GPU arm's aged pool) instead of the b-sphere, so both arms time the same regime.
    """
    if init is not None:
        traj_per_proc = max(1, min(traj_per_proc, len(init[0]) // cores))
    jobs = []
    for i in range(cores):
        sl = None
        if init is not None:
            sl = (init[0][i * traj_per_proc:(i + 1) * traj_per_proc], init[1][i * traj_per_proc:(i + 1) * traj_per_proc])
        jobs.append((traj_per_proc, 1000 + i, n_steps, sl))
    with tempfile.TemporaryDirectory() as td:
        f = os.path.join(td, "inputs.npz")
        save_cpu_inputs(s, f)
        ctx = mp.get_context("spawn")
        t0 = time.perf_counter()
        with ctx.Pool(cores) as pool:
            out = pool.map(_cpu_worker, [(f, n, sd, ns, sl) for n, sd, ns, sl in jobs])
        wall = time.perf_counter() - t0
    steps = sum(o[0] for o in out)
    busy = max(o[1] for o in out)
    # one single-threaded process's own rate (median over the processes, all running at once)
    per_proc = float(np.median([o[0] / o[1] for o in out if o[1] > 0])) if any(o[1] > 0 for o in out) else 0.0
    if where is None:
        where = "poses sampled from the GPU arm's aged pool" if init is not None else "the b-sphere"
    return steps / busy, {"value": steps / busy, "unit": UNIT, "cores": cores, "kind": "port",
                          "sample": f"{cores} processes x {traj_per_proc} trajectories x <= {n_steps} steps of the "
                                    f"same system from {where} ({steps} trajectory-steps, {busy:.1f} s)",
                          "one_process_value": per_proc,
                          "wall_s": round(wall, 1)}


# --------------------------------------------------------------------------- main
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--inner", type=int, default=64, help="BD steps per trajectory per launch")
    ap.add_argument("--n-traj", type=int, default=0, help="trajectories per GPU (0: the workload's own count)")
    ap.add_argument("--workload", default="protein-ligand", choices=sorted(WORKLOADS))
    ap.add_argument("--launch", default="", help="fixed launch shape GROUPxBLOCK (default: autotune)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--layout", type=int, default=-1,
                    help="device data layout flags (1 stage receptor, 2 windows for 1-channel grids, "
                         "4 windows for the paired grid, 8 cubes for the ligand Born grid, 16 overlap "
                         "occupancy grid, 32 xy records with the cubes, 64 z-edge texture records with the cubes, "
                         "128 xy records read through the texture path, 256 a texture view of the paired grid; "
                         "-1: autotuned)")
    ap.add_argument("--cpu-steps", type=int, default=40)
    ap.add_argument("--no-surrogate", action="store_true", help="skip the surrogate arm (config 4)")
    ap.add_argument("--age", type=int, default=-1,
                    help="untimed launches that age the pool before every timed arm (0: time from the b-sphere; "
                         "default: 64, 16 for protein-protein, 0 for the two spheres, whose trajectories are all "
                         "done well before 64 launches)")
    ap.add_argument("--sur-poses", type=int, default=2_000_000)
    ap.add_argument("--sur-train-steps", type=int, default=20_000)
    ap.add_argument("--sur-members", type=int, default=5)
    ap.add_argument("--sur-kon-traj", type=int, default=8_000)
    ap.add_argument("--no-protein-protein", action="store_true",
                    help="skip the protein-protein variants (config 3) of the default run")
    ap.add_argument("--pp-traj", type=int, default=200_000)
    ap.add_argument("--pp-age", type=int, default=16)
    ap.add_argument("--pp-steps", type=int, default=3)
    ap.add_argument("--pp-surrogate", action="store_true",
                    help="also train and time a surrogate on the protein-protein workload (minutes)")
    ap.add_argument("--pp-sur-poses", type=int, default=200_000)
    ap.add_argument("--pp-sur-train-steps", type=int, default=8000)
    args = ap.parse_args()
    if args.age < 0:
        args.age = {"two-spheres": 0, "protein-protein": 16}.get(args.workload, 64)
    _OPTS["layout"] = None if args.layout < 0 else args.layout
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        s = build_system("cuda" if _has_cuda() else "cpu", args.workload)
        cores = os.cpu_count() or 1
        init, where = None, "the b-sphere"
        sample = ROOT / "oracle" / "samples" / "aged_protein_ligand.npz"
        if args.workload == "protein-ligand" and args.age > 0 and sample.exists():
            d = np.load(sample)
            init = (d["c"], d["q"])
            where = (f"a committed sample of {len(d['c'])} poses aged {int(d['aged_steps'])} BD steps from the "
                     f"b-sphere by the oracle alone ({sample.name})")
        vals = []
        for i in range(args.warmup + args.steps):
            v, info = cpu_baseline(s, cores, traj_per_proc=64, n_steps=args.cpu_steps, init=init,
                                   where=where)
            if i >= args.warmup:
                vals.append(v)
        val = float(np.mean(vals))
        info["value"] = val
        print(json.dumps({"impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus,
                          "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
                          "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                          "config": {"workload": WORKLOADS[args.workload][0],
                                     "arm": "reference batched stepper restated in NumPy "
                                     "(PCG64 order), CPU"},
                          "cpu_baseline": info, "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0,
                                                        "d2h_bytes_per_step": 0}}))
        return

    if args.workload == "heterogeneous":
        if world > 1:
            print(json.dumps({"error": "the heterogeneous batch is a single-GPU workload"}))
            return
        hetero_main(args)
        return

    import torch

    dist = None
    if world > 1:
        import datetime

        import torch.distributed as td

        torch.cuda.set_device(local)
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = td
    s = build_system("cuda", args.workload)
    n_traj = args.n_traj or WORKLOADS[args.workload][1]
    id_offset = rank * n_traj
    clocks = Clocks(local)
    fixed = tuple(int(v) for v in args.launch.split("x")) if args.launch else None
    work = tempfile.mkdtemp(prefix="bench_pool_")
    aged = None
    if args.age > 0:
        t_age = time.perf_counter()
        ager = make_sim(s, "mixed", n_traj, args.inner, id_offset, slots=pool_slots(n_traj))
        aged = age_pool(ager, args.inner, args.age, os.path.join(work, "aged.npz"))
        ager.engine.close()
        _progress(f"pool aged {args.age} launches ({args.age * args.inner} BD steps) in "
                  f"{time.perf_counter() - t_age:.1f} s")
    clocks.start()
    t_mixed, tl_mixed, d_mixed, launch = time_device_arm(s, "mixed", args.steps, args.warmup, args.inner, n_traj,
                                                         id_offset, dist, fixed, aged=aged)
    ck = clocks.stop()
    t_fp64, tl_fp64, d_fp64, launch64 = time_device_arm(s, "fp64", args.steps, args.warmup, args.inner, n_traj,
                                                        id_offset, dist, fixed, aged=aged)
    _progress(f"exact arms: mixed {d_mixed['steps'] / t_mixed:.3e}, fp64 {d_fp64['steps'] / t_fp64:.3e} steps/s")
    layout_cli = _OPTS["layout"]
    _OPTS["layout"] = launch["layout_flags"]  # the tuned shape and layout, through the public API
    e2e_val, h2d, d2h, e2e_res = e2e_arm(s, "mixed", max(args.steps, 10), args.inner, n_traj, id_offset,
                                         (launch["group"], launch["block"]), aged=aged)
    _OPTS["layout"] = layout_cli
    _progress(f"e2e arm: {e2e_val:.3e} steps/s")
    t_max, steps_all, pooled_tallies = t_mixed, d_mixed["steps"], None
    if dist is not None:
        t_max, steps_all, pooled_tallies, e2e_val, h2d, d2h = pool_over_ranks(
            dist, torch.device("cuda", local), t_mixed, d_mixed, e2e_res.e2e_seconds, e2e_res.e2e_steps, h2d, d2h)
    value = steps_all / t_max
    peak, peak_kind = peaks()
    gathers = d_mixed["grid_evals"] + d_mixed["rev_evals"]
    algo_bytes = gathers * ALGO_BYTES_PER_GATHER + d_mixed["steps"] * STATE_BYTES_PER_STEP
    achieved = algo_bytes / t_mixed / 1e9
    traffic, traffic_note = None, None
    tf = ROOT / "profiles" / "stepper_traffic.json"
    if args.workload == "protein-ligand" and tf.exists():
        # DRAM bytes (read + write) of one stepper launch, from the ncu capture of a small case scaled by the
        # trajectory-steps of this launch (the figure and its scaling are stated in the file)
        t = json.loads(tf.read_text())
        traffic = int(t["dram_bytes_per_trajectory_step"] * d_mixed["steps"] / args.steps)
        traffic_note = t["note"]
    if rank != 0:
        import shutil

        shutil.rmtree(work, ignore_errors=True)
        if dist is not None:
            dist.destroy_process_group()
        return
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * t_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 forces / f64 poses", "data": "synthetic",
        "config": {"workload": WORKLOADS[args.workload][0], "trajectories_per_gpu": n_traj,
                   "bd_steps_per_launch": args.inner,
                   "timed_window": (f"BD steps {(args.age + args.warmup) * args.inner}-"
                                    f"{(args.age + args.warmup + args.steps) * args.inner} of the run: the pool is "
                                    f"aged {args.age} launches (restored for each arm), then {args.warmup} warm-up "
                                    f"launches"),
                   "parallelism": f"trajectory shards x{world}", "l2": "flushed (256 MiB write) between launches",
                   "launch": launch,
                   "force_reuse": ("a step rejected by the overlap test leaves the pose unchanged; the next step "
                                   "reuses its forces instead of evaluating the same pose again (trajectories are "
                                   "bit-identical to evaluating every step)")},
        "variants": {
            "mixed": {"bd_steps_per_s": d_mixed["steps"] / t_mixed, "steps": d_mixed["steps"],
                      # trajectories this rank finished in the timed window (reacted, escaped or max steps)
                      "trajectories_per_s": (d_mixed["reacted"] + d_mixed["escaped"] + d_mixed["max_steps"]) / t_mixed},
            "fp64": {"bd_steps_per_s": d_fp64["steps"] / t_fp64, "steps": d_fp64["steps"], "launch": launch64},
            "mixed_over_fp64": (d_mixed["steps"] / t_mixed) / (d_fp64["steps"] / t_fp64),
        },
        "counters": {k: int(v) for k, v in d_mixed.items()},
        "counters_all_ranks": pooled_tallies,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "traffic_note": traffic_note, "peak_kind": peak_kind,
                     "algorithmic_bytes": "224 B per (atom, grid) stencil + 128 B per trajectory-step"},
        "cupy_reference": cupy_reference(),
        "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "note": ("B200ForceEngine from host arrays (grid uploads) + B200BatchSimulator.run() resuming the "
                         "aged pool from its checkpoint file (slots copied host-to-device), "
                         f"{max(args.steps, 10)} launches with a counter poll after each, outcomes copied back"),
                "seconds": getattr(e2e_res, "e2e_split", None)},
        # kernels per timed launch: the split step is three kernels per BD step plus the compaction's two;
        # the fused stepper is one kernel plus the compaction's two
        "gpu_launches": ((3 * args.inner + 2) if launch["group"] == 66 else 3) * args.steps,
        "clocks": ck,
    }
    if world == 1 and not args.no_surrogate and args.workload != "two-spheres":
        line["variants"]["surrogate"] = surrogate_arm(s, args.steps, args.warmup, args.inner, n_traj, args.sur_poses,
                                                      args.sur_train_steps, args.sur_members, args.sur_kon_traj,
                                                      log=_progress, aged=aged)
    if world == 1 and args.workload == "protein-ligand" and not args.no_protein_protein:
        line["variants"]["protein_protein"] = protein_protein_section(args, _progress)
    if world == 1 and not args.no_cpu_baseline:
        cores = os.cpu_count() or 1
        init = aged_poses(aged, cores * 64) if aged is not None else None
        _, info = cpu_baseline(s, cores, n_steps=args.cpu_steps, init=init)
        line["cpu_baseline"] = info
        if aged is not None and args.workload != "two-spheres":
            line["force_error"] = force_error_check(s, *aged_poses(aged, 256, seed=11))
    print(json.dumps(line))
    import shutil

    shutil.rmtree(work, ignore_errors=True)
    if dist is not None:
        dist.destroy_process_group()


def pool_over_ranks(dist, device, t_local, counters, e2e_seconds, e2e_steps, h2d, d2h):
    """The whole job's figures under torchrun, the same collectives in the same order on every rank:
    the timed window's time (max over ranks) and BD steps (sum), the outcome tallies (sum, the one
    data collective), and the end-to-end arm's steps and copied bytes (sum) over its slowest rank's
    time.  Returns (t_max, steps, tallies, e2e_value, h2d_bytes, d2h_bytes)."""
    import torch

    from pystarc_b200.shard import allreduce_tallies

    tt = torch.tensor([t_local, e2e_seconds], device=device, dtype=torch.float64)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    st = torch.tensor([counters["steps"], e2e_steps, int(h2d), int(d2h)], device=device, dtype=torch.int64)
    dist.all_reduce(st)
    tallies = allreduce_tallies(counters, device=device)
    t_max, e2e_t = float(tt[0].item()), float(tt[1].item())
    steps, e2e_steps_all, h2d_all, d2h_all = (int(v) for v in st.cpu())
    return t_max, steps, tallies, e2e_steps_all / e2e_t, h2d_all, d2h_all


def cupy_reference():
    """The reference's own CuPy path (GPUBatchSimulator on the GPU) can only run where CuPy imports."""
    try:
        import cupy  # noqa: F401
    except Exception as e:  # ImportError, or a CuPy without a usable CUDA runtime
        return f"unavailable (CuPy not installed: import cupy fails with {type(e).__name__})"
    return "unavailable (CuPy imports, but the reference source is not shipped to the GPU box)"


def _has_cuda():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


if __name__ == "__main__":
    main()
