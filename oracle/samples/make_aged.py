"""Seeded sample of aged poses for the reference arm of ``bench.py`` (test infrastructure).

The GPU arm of the benchmark times the step loop after every trajectory has advanced
4,096 BD steps from the b-sphere, because the per-step cost rises several-fold as the
trajectories reach the receptor.  The reference arm has to time the same regime without
using the engine, so this script ages trajectories with the oracle alone, on the CPU:
``oracle.stepper.run`` (the reference step loop, pystarc/simulation/gpu_batch_simulator.py
:783-1254) with its own PCG64 draws, started on the b-sphere of the protein + small-ligand
workload (3,200/18 atoms, 193^3 + 129^3 grids, 65^3 ligand Born grid, b = 60 A), for
``--steps`` steps.  The poses of the trajectories still running at the end are saved.

``--workers W`` splits the trajectories over W processes (worker w runs its share with seed
``seed + w``); the grids are filled once, in torch on the CPU, and handed to the workers in
the file format of ``bench.save_cpu_inputs``.

    python oracle/samples/make_aged.py [--n 1024] [--steps 4096] [--seed 20261204] [--workers 1]

Writes ``oracle/samples/aged_protein_ligand.npz`` (centroids, quaternions, steps).
"""

from __future__ import annotations

import argparse
import multiprocessing as mp
import os
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]


def _age(args):
    inputs, n, seed, steps = args
    sys.path.insert(0, str(REPO))
    from bench import oracle_system
    from oracle import stepper as ost

    ss, prm = oracle_system(inputs, n, seed, steps)
    # the reference loop stops after max_steps loop steps; with no refill that is each trajectory's step count
    res = ost.run(ss, prm, noise="pcg64", termination="reference")
    run = (res.status == 3) & (res.n_steps == steps)
    return res.pos[run], res.q[run], res.n_steps[run], res.n_reacted, res.n_escaped


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=1024)
    ap.add_argument("--steps", type=int, default=4096)
    ap.add_argument("--seed", type=int, default=20261204)
    ap.add_argument("--workers", type=int, default=1)
    ap.add_argument("--scale", type=float, default=1.0, help="system scale (1.0: the benchmark's size)")
    ap.add_argument("--out", default=str(HERE / "aged_protein_ligand.npz"))
    args = ap.parse_args()
    sys.path.insert(0, str(REPO))
    from bench import save_cpu_inputs
    from pystarc_b200 import synth

    t0 = time.time()
    s = synth.config2(scale=args.scale, device="cpu")
    print(f"system built in {time.time() - t0:.0f} s", flush=True)
    W = max(1, args.workers)
    share = [args.n // W + (w < args.n % W) for w in range(W)]
    with tempfile.TemporaryDirectory() as td:
        inputs = os.path.join(td, "inputs.npz")
        save_cpu_inputs(s, inputs)
        t0 = time.time()
        jobs = [(inputs, share[w], args.seed + w, args.steps) for w in range(W) if share[w] > 0]
        with mp.get_context("spawn").Pool(len(jobs)) as pool:
            parts = pool.map(_age, jobs)
    c = np.concatenate([p[0] for p in parts])
    q = np.concatenate([p[1] for p in parts])
    steps = np.concatenate([p[2] for p in parts])
    print(f"aged {args.n} trajectories {args.steps} steps in {time.time() - t0:.0f} s on {len(jobs)} processes; "
          f"{len(c)} still running (reacted {sum(p[3] for p in parts)}, escaped {sum(p[4] for p in parts)})",
          flush=True)
    np.savez_compressed(args.out, c=c, q=q, steps=steps, n=args.n, aged_steps=args.steps, seed=args.seed,
                        workers=len(jobs), system=s.name)


if __name__ == "__main__":
    main()
