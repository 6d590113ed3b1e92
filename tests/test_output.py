"""The output files against the reference's ``write_all`` (pystarc/pipeline/output_writer.py:15-304).

The fixture holds a reference run of the two-sphere example (300 trajectories, paths every 100
steps): its sim_data and result fields, and the content of the 14 files the reference wrote from
them.  ``pystarc_b200.output.write_all`` must write the same files from the same inputs: CSV text
identical, npz arrays identical, results.json values equal.
"""

import json

import numpy as np

from tests.helpers import golden


def _inputs(g):
    from pystarc_b200.pipeline import OutputConfig
    from pystarc_b200.simulator import B200BatchResult

    sd = {}
    for k in g:
        if k.startswith("sd:"):
            v = g[k]
            sd[k[3:]] = [v] if k[3:] in ("path_steps", "energy_steps") else v
    sd["contact_total_steps"] = int(sd["contact_total_steps"])
    f = {k[4:]: g[k][()] for k in g if k.startswith("res:")}
    res = B200BatchResult(n_trajectories=int(f["n_trajectories"]), n_reacted=int(f["n_reacted"]),
                          n_escaped=int(f["n_escaped"]), n_max_steps=int(f["n_max_steps"]), reaction_counts={},
                          r_start=float(f["r_start"]), r_escape=float(f["r_escape"]), dt=float(f["dt"]),
                          elapsed_sec=float(f["elapsed_sec"]), steps_per_sec=float(f["steps_per_sec"]))
    cfg = OutputConfig()
    cfg.save_interval = int(g["save_interval"])
    return res, sd, cfg


def test_write_all_writes_the_reference_files(tmp_path):
    from pystarc_b200.output import write_all

    g = golden("writer_two_sphere")
    res, sd, cfg = _inputs(g)
    written = write_all(tmp_path, res, sd, cfg, float(g["k_b"]), float(g["D_rel"]), 0.95, verbose=False)
    assert [n for n, _ in written] == [str(x) for x in g["written"]]
    assert len(written) == 14
    for name, path in written:
        if name == "results.json":
            mine, ref = json.loads(path.read_text()), json.loads(str(g["file:results.json"]))
            assert list(mine) == list(ref)
            for k in ref:
                if isinstance(ref[k], float):
                    assert abs(mine[k] - ref[k]) <= 1e-13 * abs(ref[k]), (k, mine[k], ref[k])
                else:
                    assert mine[k] == ref[k], k
        elif name.endswith(".npz"):
            with np.load(path) as z:
                keys = sorted(k.split(":", 2)[2] for k in g if k.startswith(f"file:{name}:"))
                assert sorted(z.files) == keys, name
                for k in keys:
                    np.testing.assert_array_equal(z[k], g[f"file:{name}:{k}"], err_msg=f"{name}:{k}")
        else:
            assert path.read_text() == str(g[f"file:{name}"]), name


def test_write_all_honours_the_flags(tmp_path):
    from pystarc_b200.output import write_all

    g = golden("writer_two_sphere")
    res, sd, cfg = _inputs(g)
    cfg.full_paths = False
    cfg.energetics = False
    cfg.trajectories_csv = False
    written = {n for n, _ in write_all(tmp_path, res, sd, cfg, float(g["k_b"]), float(g["D_rel"]), verbose=False)}
    assert not written & {"paths.npz", "energetics.npz", "trajectories.csv"}
    assert len(written) == 11
