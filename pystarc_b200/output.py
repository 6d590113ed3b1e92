"""The run's output files, with the names, columns and number formats of the reference's
``write_all`` (pystarc/pipeline/output_writer.py:15-304).

``write_all(work_dir, result, sim_data, output_cfg, k_b, D_rel, confidence)`` writes the
files that ``output_cfg`` enables (every flag defaults to on):

====  =======================  ======================================================
 1    results.json             k_on, P_rxn and their confidence interval, tallies
 2    trajectories.csv         one row per trajectory: outcome, steps, start pose, ...
 3    encounters.csv           pose at each reaction
 4    near_misses.csv          closest-approach pose of each escaped trajectory
 5    paths.npz                path rows every save_interval steps
 6    radial_density.csv       radial histogram with shell densities
 7    angular_map.npz          (theta, phi) occupancy
 8    fpt_distribution.csv     first-passage time of each reacted trajectory
 9    contact_frequency.csv    per reaction pair: steps within the cutoff
10    milestone_flux.csv       outward / inward crossings of 11 shells
11    p_commit.npz             reaction probability binned by start radius
12    transition_matrix.npz    radial transition counts
13    energetics.npz           force / dt rows every save_interval steps
14    pose_clusters.csv        reaction poses binned by rotation angle (more than 5 reactions)
====  =======================  ======================================================

Rows are formatted a column at a time with NumPy instead of a Python loop per row, so
1e6-trajectory runs write in seconds; the text is the same as the reference's
(``"%.6f" % x`` and ``f"{x:.6f}"`` round identically).
"""

from __future__ import annotations

import json
import math
from pathlib import Path

import numpy as np

OUTCOME_NAMES = {1: "reacted", 2: "escaped", 3: "max_steps", 0: "running"}


def _col(fmt, values):
    return np.char.mod(fmt, np.asarray(values))


def _write_rows(path, header, columns):
    """One CSV row per entry: ``columns`` are arrays of preformatted strings (equal length)."""
    with open(path, "w") as f:
        f.write(header)
        if len(columns) and len(columns[0]):
            rows = columns[0].astype(object)
            for c in columns[1:]:
                rows = rows + "," + c.astype(object)
            f.write("\n".join(rows.tolist()))
            f.write("\n")


def results_record(result, sim_data, k_b, D_rel, confidence):
    """The results.json record (output_writer.py:76-116)."""
    k_on = result.rate_constant(D_rel, k_b)
    k_lo, k_hi = result.rate_constant_ci(D_rel, k_b, confidence)
    p_lo, p_hi = result.reaction_probability_ci(confidence)
    data = {"k_on": k_on, "k_on_low": k_lo, "k_on_high": k_hi, "k_on_units": "M-1 s-1",
            "P_rxn": result.reaction_probability, "P_rxn_low": p_lo, "P_rxn_high": p_hi, "k_b": k_b,
            "k_b_units": "A3/ps", "D_rel": D_rel, "D_rel_units": "A2/ps", "n_trajectories": result.n_trajectories,
            "n_reacted": result.n_reacted, "n_escaped": result.n_escaped, "n_max_steps": result.n_max_steps,
            "r_start": result.r_start, "r_escape": result.r_escape, "wall_time_sec": result.elapsed_sec,
            "steps_per_sec": result.steps_per_sec, "confidence_level": confidence}
    if k_on > 0:
        data["log10_k_on"] = math.log10(k_on)
    if "completed_reactions" in sim_data:
        data["completed_reactions"] = sim_data["completed_reactions"]
    return data


def write_all(work_dir, result, sim_data, output_cfg, k_b, D_rel, confidence=0.95, verbose=True):
    """Write every enabled output file into ``work_dir``; returns [(name, path)] in writing order."""
    W = Path(work_dir)
    W.mkdir(parents=True, exist_ok=True)
    sd = sim_data
    on = lambda flag: bool(getattr(output_cfg, flag, True))
    written = []

    if on("results_json"):
        p = W / "results.json"
        p.write_text(json.dumps(results_record(result, sd, k_b, D_rel, confidence), indent=2))
        written.append(("results.json", p))

    if on("trajectories_csv") and "outcome" in sd:
        N = len(sd["outcome"])
        sp, sq = np.asarray(sd["start_pos"]), np.asarray(sd["start_q"])
        names = np.array([OUTCOME_NAMES.get(int(o), "unknown") for o in np.unique(sd["outcome"])] or ["x"])
        lookup = dict(zip(np.unique(sd["outcome"]).tolist(), names.tolist()))
        ostr = np.array([lookup[int(o)] for o in sd["outcome"]]) if N else np.zeros(0, dtype=str)
        cols = [_col("%d", np.arange(N)), ostr, _col("%d", np.asarray(sd["n_steps"]).astype(np.int64))]
        cols += [_col("%.6f", sp[:, k]) for k in range(3)] + [_col("%.6f", sq[:, k]) for k in range(4)]
        cols += [_col("%.6f", sd["min_dist"]), _col("%d", np.asarray(sd["step_at_min"]).astype(np.int64)),
                 _col("%.4f", sd["total_time_ps"]), _col("%d", np.asarray(sd["n_returns"]).astype(np.int64)),
                 _col("%d", np.asarray(sd["bb_triggered"]).astype(np.int64))]
        p = W / "trajectories.csv"
        _write_rows(p, "traj_id,outcome,n_steps,start_x,start_y,start_z,start_q0,start_q1,start_q2,start_q3,"
                       "min_distance,step_at_min,total_time_ps,n_returns,bb_triggered\n", cols)
        written.append(("trajectories.csv", p))

    if on("encounters_csv") and "encounter_pos" in sd and len(sd["encounter_pos"]) > 0:
        ep, eq = np.asarray(sd["encounter_pos"]), np.asarray(sd["encounter_q"])
        cols = [_col("%d", np.asarray(sd["encounter_traj"]).astype(np.int64)),
                _col("%d", np.asarray(sd["encounter_step"]).astype(np.int64))]
        cols += [_col("%.6f", ep[:, k]) for k in range(3)] + [_col("%.6f", eq[:, k]) for k in range(4)]
        cols += [_col("%d", np.asarray(sd["encounter_n_pairs"]).astype(np.int64))]
        p = W / "encounters.csv"
        _write_rows(p, "traj_id,step,x,y,z,q0,q1,q2,q3,n_pairs_satisfied\n", cols)
        written.append(("encounters.csv", p))

    if on("near_misses_csv") and "near_miss_pos" in sd and len(sd["near_miss_pos"]) > 0:
        npos, nq = np.asarray(sd["near_miss_pos"]), np.asarray(sd["near_miss_q"])
        cols = [_col("%d", np.asarray(sd["near_miss_traj"]).astype(np.int64)), _col("%.6f", sd["near_miss_dist"])]
        cols += [_col("%.6f", npos[:, k]) for k in range(3)] + [_col("%.6f", nq[:, k]) for k in range(4)]
        p = W / "near_misses.csv"
        _write_rows(p, "traj_id,min_distance,x,y,z,q0,q1,q2,q3\n", cols)
        written.append(("near_misses.csv", p))

    if on("full_paths") and "path_steps" in sd and len(sd["path_steps"]) > 0:
        p = W / "paths.npz"
        np.savez_compressed(p, data=np.vstack(sd["path_steps"]),
                            columns=np.array(["traj_id", "step", "x", "y", "z", "q0", "q1", "q2"]))
        written.append(("paths.npz", p))

    if on("radial_density") and "radial_bins" in sd:
        bins = np.asarray(sd["radial_bins"], dtype=np.float64)
        counts = np.asarray(sd["radial_counts"])
        total = counts.sum() if counts.sum() > 0 else 1
        lo, hi = bins[:-1], bins[1:]
        vol = 4.0 / 3.0 * math.pi * (hi ** 3 - lo ** 3)
        with np.errstate(divide="ignore", invalid="ignore"):
            rho = np.where(vol > 0, counts / (total * vol), 0.0)
        cols = [_col("%.4f", 0.5 * (lo + hi)), _col("%.4f", lo), _col("%.4f", hi),
                _col("%d", counts.astype(np.int64)), _col("%.8e", rho)]
        p = W / "radial_density.csv"
        _write_rows(p, "r_center,r_low,r_high,count,density\n", cols)
        written.append(("radial_density.csv", p))

    if on("angular_map") and "angular_counts" in sd:
        p = W / "angular_map.npz"
        np.savez_compressed(p, counts=sd["angular_counts"], theta_centers=sd["angular_theta"],
                            phi_centers=sd["angular_phi"])
        written.append(("angular_map.npz", p))

    if on("fpt_distribution") and "outcome" in sd:
        rx = np.nonzero(np.asarray(sd["outcome"]) == 1)[0]
        if rx.size:
            p = W / "fpt_distribution.csv"
            _write_rows(p, "traj_id,first_passage_time_ps,min_distance\n",
                        [_col("%d", rx), _col("%.4f", np.asarray(sd["total_time_ps"])[rx]),
                         _col("%.6f", np.asarray(sd["min_dist"])[rx])])
            written.append(("fpt_distribution.csv", p))

    if on("contact_frequency") and "contact_pair_counts" in sd:
        counts = np.asarray(sd["contact_pair_counts"])
        total = sd.get("contact_total_steps", 1)
        freq = counts / total if total > 0 else np.zeros(len(counts))
        p = W / "contact_frequency.csv"
        _write_rows(p, "pair_index,n_contacts,frequency\n",
                    [_col("%d", np.arange(len(counts))), _col("%d", counts.astype(np.int64)), _col("%.8e", freq)])
        written.append(("contact_frequency.csv", p))

    if on("milestone_flux") and "milestone_radii" in sd:
        fo = np.asarray(sd["milestone_flux_out"]).astype(np.int64)
        fi = np.asarray(sd["milestone_flux_in"]).astype(np.int64)
        p = W / "milestone_flux.csv"
        _write_rows(p, "radius,flux_outward,flux_inward,net_flux\n",
                    [_col("%.4f", sd["milestone_radii"]), _col("%d", fo), _col("%d", fi), _col("%d", fo - fi)])
        written.append(("milestone_flux.csv", p))

    if on("p_commit") and "outcome" in sd:
        # start radii in 50 equal bins between their extremes (output_writer.py:247-270)
        r = np.linalg.norm(np.asarray(sd["start_pos"]), axis=1)
        n_bins = 50
        bins = np.linspace(r.min(), r.max(), n_bins + 1)
        idx = np.clip(np.minimum(np.searchsorted(bins, r) - 1, n_bins - 1), 0, None)
        n_count = np.bincount(idx, minlength=n_bins).astype(np.float64)
        p_react = np.bincount(idx, weights=(np.asarray(sd["outcome"]) == 1).astype(np.float64), minlength=n_bins)
        p_commit = np.divide(p_react, n_count, out=np.zeros_like(p_react), where=n_count > 0)
        p = W / "p_commit.npz"
        np.savez_compressed(p, r_bins=bins, p_commit=p_commit, n_samples=n_count)
        written.append(("p_commit.npz", p))

    if on("transition_matrix") and "trans_matrix" in sd:
        p = W / "transition_matrix.npz"
        np.savez_compressed(p, bins=sd["trans_bins"], counts=sd["trans_matrix"])
        written.append(("transition_matrix.npz", p))

    if on("energetics") and "energy_steps" in sd and len(sd["energy_steps"]) > 0:
        p = W / "energetics.npz"
        np.savez_compressed(p, data=np.vstack(sd["energy_steps"]),
                            columns=np.array(["traj_id", "step", "fx", "fy", "fz", "dt"]))
        written.append(("energetics.npz", p))

    if on("pose_clusters") and "encounter_q" in sd and len(sd["encounter_q"]) > 5:
        eq = np.asarray(sd["encounter_q"])
        angle = 2.0 * np.arccos(np.clip(np.abs(eq[:, 0]), 0, 1))  # rotation angle of the reaction pose
        n_clusters = min(8, len(eq))
        labels = np.clip(np.digitize(angle, np.linspace(0, np.pi, n_clusters + 1)) - 1, 0, n_clusters - 1)
        cols = [_col("%d", np.asarray(sd["encounter_traj"]).astype(np.int64)), _col("%d", labels),
                _col("%.6f", angle)] + [_col("%.6f", eq[:, k]) for k in range(4)]
        p = W / "pose_clusters.csv"
        _write_rows(p, "traj_id,cluster,angle_rad,q0,q1,q2,q3\n", cols)
        written.append(("pose_clusters.csv", p))

    if verbose and written:
        print(f"\n  Output files ({len(written)})")
        for name, fp in written:
            size = fp.stat().st_size
            txt = f"{size / 1e6:.1f} MB" if size > 1e6 else f"{size / 1e3:.1f} KB" if size > 1e3 else f"{size} B"
            print(f"  {name:<30s}  {txt}")
    return written
