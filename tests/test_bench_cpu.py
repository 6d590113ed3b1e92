"""The benchmark's CPU legs: the baseline record and the ``--impl reference`` JSON line.

Both time the reference's step loop restated in NumPy (the oracle) on host processes; these
tests run them on the two-sphere system with a few trajectories so that the record's shape
is checked without a GPU.
"""

import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def test_cpu_baseline_record():
    import bench
    from pystarc_b200 import synth

    v, info = bench.cpu_baseline(synth.config1(), 2, traj_per_proc=8, n_steps=5)
    assert v > 0 and info["value"] == v
    assert info["kind"] == "port" and info["cores"] == 2 and info["unit"] == bench.UNIT
    # the rate of one single-threaded process is reported beside the pooled rate
    assert 0 < info["one_process_value"] <= v
    assert "2 processes x 8 trajectories" in info["sample"]


def test_reference_arm_line():
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--workload", "two-spheres",
                          "--steps", "1", "--warmup", "1", "--cpu-steps", "4"],
                         cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["metric"] and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
