"""Seeded sample of aged poses for the reference arm of ``bench.py`` (test infrastructure).

The GPU arm of the benchmark times the step loop after every trajectory has advanced
4,096 BD steps from the b-sphere, because the per-step cost rises several-fold as the
trajectories reach the receptor.  The reference arm has to time the same regime without
using the engine, so this script ages trajectories with the oracle alone, on the CPU:
``oracle.stepper.run`` (the reference step loop, pystarc/simulation/gpu_batch_simulator.py
:783-1254) with its own PCG64 draws, started on the b-sphere of the protein + small-ligand
workload (3,200/18 atoms, 193^3 + 129^3 grids, 65^3 ligand Born grid, b = 60 A), for
``--steps`` steps.  The poses of the trajectories still running at the end are saved.

    python oracle/samples/make_aged.py [--n 1024] [--steps 4096] [--seed 20261204]

Writes ``oracle/samples/aged_protein_ligand.npz`` (centroids, quaternions, steps).
"""

from __future__ import annotations

import argparse
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=1024)
    ap.add_argument("--steps", type=int, default=4096)
    ap.add_argument("--seed", type=int, default=20261204)
    ap.add_argument("--out", default=str(HERE / "aged_protein_ligand.npz"))
    args = ap.parse_args()
    sys.path.insert(0, str(REPO))
    from oracle import stepper as ost
    from pystarc_b200 import synth
    from tests.helpers import oracle_engine, step_params, step_system

    t0 = time.time()
    s = synth.config2(scale=1.0)
    print(f"system built in {time.time() - t0:.0f} s", flush=True)
    t0 = time.time()
    # the reference loop stops after max_steps loop steps; with no refill that is each trajectory's step count
    res = ost.run(step_system(s, oracle_engine(s)), step_params(s, args.n, args.seed, args.steps), noise="pcg64",
                  termination="reference")
    run = (res.status == 3) & (res.n_steps == args.steps)
    print(f"aged {args.n} trajectories {args.steps} steps in {time.time() - t0:.0f} s; {int(run.sum())} still "
          f"running (reacted {res.n_reacted}, escaped {res.n_escaped})", flush=True)
    np.savez_compressed(args.out, c=res.pos[run], q=res.q[run], steps=res.n_steps[run], n=args.n,
                        aged_steps=args.steps, seed=args.seed, system=s.name)


if __name__ == "__main__":
    main()
