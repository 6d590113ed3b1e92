"""Generate golden vectors by running the UNMODIFIED reference on seeded synthetic inputs.

Run where a checkout of the reference exists, naming its path with ``--reference``
or the ``PYSTARC_REFERENCE`` environment variable:

    python tests/golden/make_golden.py --reference <path to the PySTARC checkout>

The reference's batched engine and stepper import ``cupy``; this script puts
``oracle/cupy_standin`` first on ``sys.path`` so they run on NumPy, with the
single CUDA kernel they launch restated by ``oracle.forces``.  The K1 arithmetic
is pinned independently by ``DXGrid.batch_interpolate`` / ``batch_gradient``
(reference code with the same +-h/2 central difference).

Outputs (small .npz files next to this script) hold the inputs that are cheap
to store, SHA-256 digests of the grids (rebuilt deterministically from
``pystarc_b200.synth`` by the tests) and the reference's outputs.
"""

from __future__ import annotations

import argparse
import contextlib
import hashlib
import io
import json
import math
import os
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]


def grid_digest(grids):
    h = hashlib.sha256()
    for g in grids:
        h.update(np.ascontiguousarray(np.asarray(g.data, dtype=np.float32)).tobytes())
        h.update(np.asarray(g.origin, dtype=np.float64).tobytes())
        h.update(np.asarray(g.delta, dtype=np.float64).tobytes())
    return h.hexdigest()


def system_digest(s):
    return grid_digest(list(s.elec_grids) + list(s.born_grids) + list(s.lig_born_grids))


def quiet():
    return contextlib.redirect_stdout(io.StringIO())


def ref_grid(DXGrid, g):
    return DXGrid(np.asarray(g.origin, dtype=float), np.asarray(g.delta, dtype=float),
                  np.asarray(g.data, dtype=np.float64))


def ref_molecules(mod, s):
    Atom, Molecule = mod.Atom, mod.Molecule

    def mk(name, pos, q, r):
        return Molecule(name, [Atom(index=i + 1, name="A", x=float(p[0]), y=float(p[1]), z=float(p[2]),
                                    charge=float(c), radius=float(rr)) for i, (p, c, rr) in enumerate(zip(pos, q, r))])

    return mk("receptor", s.rec_pos, s.rec_q, s.rec_r), mk("ligand", s.lig_pos, s.lig_q, s.lig_r)


def make_engine(ref, s, multipole=True, use_lj=False):
    from pystarc.forces.gpu_batch_engine import GPUBatchForceEngine
    from pystarc.forces.multipole_farfield import MultipoleExpansion
    from pystarc.forces.electrostatic.grid_force import DXGrid

    mp = MultipoleExpansion(s.rec_pos, s.rec_q, debye_length=s.debye, sdie=s.sdie) if multipole else None
    with quiet():
        eng = GPUBatchForceEngine(
            elec_grids=[ref_grid(DXGrid, g) for g in s.elec_grids],
            born_grids=[ref_grid(DXGrid, g) for g in s.born_grids], alpha=s.alpha,
            receptor_charge=float(np.sum(s.rec_q)), debye_length=s.debye, sdie=s.sdie,
            lig_born_grids=[ref_grid(DXGrid, g) for g in s.lig_born_grids] or None,
            rec_positions=s.rec_pos, rec_charges=s.rec_q, multipole_expansion=mp,
            rec_radii=s.rec_r if use_lj else None, lig_radii=s.lig_r if use_lj else None, use_lj=use_lj)
    return eng


def random_poses(n, rmin, rmax, rng):
    v = rng.standard_normal((n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    c = v * rng.uniform(rmin, rmax, size=(n, 1))
    u = rng.random((n, 3))
    q = np.stack([np.sqrt(1 - u[:, 0]) * np.sin(2 * np.pi * u[:, 1]), np.sqrt(1 - u[:, 0]) * np.cos(2 * np.pi * u[:, 1]),
                  np.sqrt(u[:, 0]) * np.sin(2 * np.pi * u[:, 2]), np.sqrt(u[:, 0]) * np.cos(2 * np.pi * u[:, 2])], 1)
    return c, q


def gen_k1(out):
    from pystarc.forces.electrostatic.grid_force import DXGrid

    rng = np.random.default_rng(7)
    nx, ny, nz = 24, 20, 28
    X, Y, Z = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    data = (np.sin(0.3 * X) * np.cos(0.2 * Y) + 0.05 * Z + 0.01 * rng.standard_normal((nx, ny, nz))).astype(np.float32)
    origin = np.array([-3.0, 1.5, -7.25])
    sp = np.array([0.5, 0.6, 0.4])
    g = DXGrid(origin, np.diag(sp), data.astype(np.float64))
    lo = origin + 0.6 * sp
    hi = origin + (np.array([nx, ny, nz]) - 1.6) * sp
    pts = lo + (hi - lo) * rng.random((400, 3))
    edge = np.array([origin + 0.49 * sp, origin + (np.array([nx, ny, nz]) - 1.51) * sp, origin - 5.0,
                     origin + (np.array([nx, ny, nz]) + 3) * sp, origin + np.array([2.0, 3.0, 4.0]) * sp])
    pts = np.vstack([pts, edge])
    out["k1"] = dict(data=data, origin=origin, sp=sp, points=pts, phi=g.batch_interpolate(pts),
                     grad=g.batch_gradient(pts))


def gen_engine(out, name, s, n_poses, rmin, rmax, seed):
    import pystarc.forces.gpu_batch_engine as gbe
    from pystarc.simulation.gpu_batch_simulator import GPUBatchSimulator

    eng = make_engine(None, s)
    rng = np.random.default_rng(seed)
    c, q = random_poses(n_poses, rmin, rmax, rng)
    sim = GPUBatchSimulator.__new__(GPUBatchSimulator)
    R = sim._quats_to_rotmats(q)
    body = s.lig_pos - s.lig_pos.mean(axis=0)
    pos = np.einsum("nij,kj->nki", R, body) + c[:, None, :]
    with quiet():
        F, T, E = eng(pos, s.lig_q.astype(np.float64), R_matrices=R, centroids=c)
    out[name] = dict(digest=system_digest(s), centroids=c, quats=q, R=R, positions=pos, F=F, T=T, E=E,
                     V_factor=eng._V_factor, has_yukawa=eng._has_yukawa, n_elec=len(eng._elec_grids_gpu),
                     n_born=len(eng._born_grids_gpu), n_lig_born=len(eng._lig_born_grids_gpu))


def gen_engine_wca(out, name, s, n_poses, rmin, rmax, seed):
    """The engine with WCA contact forces on (use_lj=True), at centroids around the activation
    radius: the totals and the contact term alone (``_wca_forces_gpu``)."""
    from pystarc.simulation.gpu_batch_simulator import GPUBatchSimulator

    eng = make_engine(None, s, use_lj=True)
    rng = np.random.default_rng(seed)
    c, q = random_poses(n_poses, rmin, rmax, rng)
    sim = GPUBatchSimulator.__new__(GPUBatchSimulator)
    R = sim._quats_to_rotmats(q)
    body = s.lig_pos - s.lig_pos.mean(axis=0)
    pos = np.einsum("nij,kj->nki", R, body) + c[:, None, :]
    with quiet():
        F, T, E = eng(pos, s.lig_q.astype(np.float64), R_matrices=R, centroids=c)
        F_wca = eng._wca_forces_gpu(pos, c)
    out[name] = dict(digest=system_digest(s), centroids=c, quats=q, R=R, positions=pos, F=F, T=T, E=E, F_wca=F_wca,
                     activation=eng._lj_activation, epsilon=eng._lj_epsilon)


def gen_physics(out):
    from pystarc.hydrodynamics import rotne_prager as rp
    from pystarc.simulation.gpu_batch_simulator import GPUBatchSimulator, GPUBatchResult
    from pystarc.forces.multipole_farfield import MultipoleExpansion

    rng = np.random.default_rng(11)
    radii = np.array([1.0, 1.005, 5.0, 17.5, 20.0, 25.375])
    out["stokes"] = dict(radii=radii, Dt=np.array([rp.stokes_translational_diffusion(r) for r in radii]),
                         Dr=np.array([rp.stokes_rotational_diffusion(r) for r in radii]),
                         Dt_089=np.array([rp.stokes_translational_diffusion(r, eta=0.89e-3) for r in radii]),
                         Dr_089=np.array([rp.stokes_rotational_diffusion(r, eta=0.89e-3) for r in radii]))
    rs = np.array([0.5, 2.0, 5.0, 20.0, 30.0, 33.9, 34.1, 50.0, 120.0])
    rpy = []
    for r in rs:
        v = np.array([r, 0.3 * r, -0.2 * r]) / math.sqrt(1 + 0.09 + 0.04)
        rpy.append(rp.rpy_offdiagonal(v, 17.5, 16.5, 0.0123, 0.0131))
    out["rpy"] = dict(r=rs, M=np.array(rpy))
    sim = GPUBatchSimulator.__new__(GPUBatchSimulator)
    q = rng.standard_normal((50, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    om = rng.standard_normal((50, 3)) * np.array([[1.0]] * 25 + [[1e-12]] * 25)
    out["quat"] = dict(q=q, omega=om, R=sim._quats_to_rotmats(q), q_new=sim._apply_rotation_gpu(q, om),
                       shoemake=sim._random_quaternions_gpu(20, np.random.default_rng(5)),
                       shoemake_u=np.random.default_rng(5).random((20, 3)))
    cis = []
    cases = [(500, 500), (50, 950), (2, 998), (0, 1000), (1000, 0), (4479, 5521), (1, 2)]
    for nr, ne in cases:
        res = GPUBatchResult(nr + ne, nr, ne, 0, {}, 50.0, 100.0, 0.2, 1.0, 1.0)
        cis.append([res.reaction_probability, *res.reaction_probability_ci(0.95), *res.reaction_probability_ci(0.9),
                    res.rate_constant(0.06, 57.449), res.rate_constant(0.06, 0.0), *res.rate_constant_ci(0.06, 57.449)])
    out["wilson"] = dict(cases=np.array(cases), values=np.array(cis))
    pos = rng.standard_normal((30, 3)) * 8
    qq = rng.normal(0, 0.4, 30)
    mp = MultipoleExpansion(pos, qq, debye_length=7.85, sdie=78.5)
    pts = rng.standard_normal((12, 3)) * 40
    out["multipole"] = dict(pos=pos, q=qq, Q=mp.Q, dipole=mp.dipole, quad=mp.quadrupole, fpe=mp.four_pi_eps,
                            pts=pts, V=np.array([mp.potential(p) for p in pts]))


def gen_bradius(out):
    """GPUBatchSimulator._compute_bradius_cover (it reads no instance state) on a grid of b-sphere
    radii, charge pairs and Debye lengths, with the reference's dielectric 78 * 0.000142."""
    from pystarc.simulation.gpu_batch_simulator import GPUBatchSimulator

    rows, vals = [], []
    for b in (10.0, 26.0, 50.0, 60.0, 80.0, 120.0):
        for q_rec, q_lig in ((8.0, 1.0), (8.0, -1.0), (2.0, -6.0), (5.0, -5.0), (1.0, -1.0), (-3.0, -2.0), (0.5, 0.1)):
            for debye in (3.0, 7.828, 7.858, 15.0):
                rows.append((b, q_rec, q_lig, debye))
                vals.append(GPUBatchSimulator._compute_bradius_cover(None, b, q_rec, q_lig, 78.0 * 0.000142, debye,
                                                                     0.05))
    out["bradius"] = dict(inputs=np.array(rows), cover=np.array(vals))


def build_sim(s, n_traj, seed, max_steps, work, sm=None, use_lj=False):
    from pystarc.simulation.gpu_batch_simulator import GPUBatchSimulator
    from pystarc.simulation.nam_simulator import NAMParameters
    from pystarc.hydrodynamics.rotne_prager import MobilityTensor
    from pystarc.structures.molecules import ContactPair, ReactionCriteria
    from pystarc.pathways.reaction_interface import ReactionInterface, PathwaySet
    import pystarc.structures.molecules as mols

    mol1, mol2 = ref_molecules(mols, s)
    mob = MobilityTensor.from_radii(s.r_hydro_rec, s.r_hydro_lig, eta=s.eta, T=s.temperature)
    pairs = [ContactPair(int(a), int(b), float(c)) for a, b, c in s.pairs]
    ps = PathwaySet([ReactionInterface("stage_0", ReactionCriteria("stage_0", pairs, n_needed=s.n_needed))])
    if sm is not None:
        rx = []
        for name, before, after, (a, b, c) in sm["reactions"]:
            crit = ReactionCriteria(name, [ContactPair(int(a), int(b), float(c))], n_needed=1, state_before=before,
                                    state_after=after)
            rx.append(ReactionInterface(name, crit, state_before=before, state_after=after))
        ps = PathwaySet(rx, first_state=sm["first_state"])
    params = NAMParameters(n_trajectories=n_traj, max_steps=max_steps, r_start=s.r_start, r_escape=s.r_escape,
                           seed=seed, hydrodynamic_interactions=s.hi)
    params.max_dt = s.max_dt
    params.checkpoint_interval = 0
    params.convergence_interval = 0
    params._work_dir = str(work)
    params._kT_scale = s.temperature / 298.15
    params._overlap_check = s.overlap
    if sm is not None:
        params.minimum_core_reaction_dt = sm["min_core_rxn_dt"]
    eng = make_engine(None, s, multipole=s.multipole, use_lj=use_lj)
    with quiet():
        sim = GPUBatchSimulator(mol1, mol2, mob, ps, params, eng)
    return sim, mob


def gen_run(out, name, s, n_traj, seed, max_steps, use_lj=False, trace_steps=None):
    """A reference run: tallies, per-trajectory outcomes and statistics; with ``trace_steps`` also the
    path and energy rows the reference records every save_interval steps, for steps below it."""
    with tempfile.TemporaryDirectory() as work:
        sim, mob = build_sim(s, n_traj, seed, max_steps, work, use_lj=use_lj)
        with quiet():
            res = sim.run()
    sd = res.sim_data
    traces = {}
    if trace_steps is not None:
        for key, ncol in (("path_steps", 8), ("energy_steps", 6)):
            rows = np.vstack(sd[key]) if len(sd[key]) else np.zeros((0, ncol))
            traces[f"sd_{key}"] = rows[rows[:, 1] < trace_steps]
    out[name] = dict(digest=system_digest(s), n_traj=n_traj, seed=seed, max_steps=max_steps,
                     n_reacted=res.n_reacted, n_escaped=res.n_escaped, n_max_steps=res.n_max_steps,
                     total_steps=int(round(res.steps_per_sec * res.elapsed_sec)), outcome=sd["outcome"],
                     n_steps=sd["n_steps"], n_returns=sd["n_returns"], return_prob=sim._return_prob, k_b=sim._k_b,
                     D_t=mob.relative_translational_diffusion(), D_r=mob.relative_rotational_diffusion(),
                     ci=np.array(res.reaction_probability_ci(0.95)),
                     **{f"sd_{k}": np.asarray(sd[k]) for k in (
                         "start_pos", "start_q", "min_dist", "step_at_min", "total_time_ps", "bb_triggered",
                         "encounter_traj", "encounter_step", "encounter_pos", "encounter_q", "near_miss_traj",
                         "near_miss_pos", "near_miss_dist", "radial_counts", "angular_counts", "milestone_flux_out",
                         "milestone_flux_in", "contact_pair_counts", "contact_total_steps", "trans_matrix")},
                     **traces)


WRITER_FILES = ("results.json", "trajectories.csv", "encounters.csv", "near_misses.csv", "paths.npz",
                "radial_density.csv", "angular_map.npz", "fpt_distribution.csv", "contact_frequency.csv",
                "milestone_flux.csv", "p_commit.npz", "transition_matrix.npz", "energetics.npz", "pose_clusters.csv")


def gen_writer(out, name, s, n_traj, seed, max_steps, save_interval):
    """The reference's output files (pipeline/output_writer.py:15-304) for one reference run: the run's
    sim_data and result fields (the writer's inputs) and the content of every file written."""
    from pystarc.pipeline.input_parser import OutputConfig
    from pystarc.pipeline.output_writer import write_all

    with tempfile.TemporaryDirectory() as work:
        sim, mob = build_sim(s, n_traj, seed, max_steps, work)
        cfg = OutputConfig(save_interval=save_interval)
        sim.params._output_cfg = cfg
        with quiet():
            res = sim.run()
            sd = res.sim_data
            D_rel = mob.relative_translational_diffusion()
            written = write_all(Path(work) / "out", res, sd, cfg, sim._k_b, D_rel, 0.95)
        rec = {}
        for fname, path in written:
            if fname.endswith(".npz"):
                with np.load(path) as z:
                    for k in z.files:
                        rec[f"file:{fname}:{k}"] = z[k]
            else:
                rec[f"file:{fname}"] = np.array(Path(path).read_text())
    arrays = {f"sd:{k}": (np.vstack(v) if len(v) else np.zeros((0, 8 if k == "path_steps" else 6)))
              if isinstance(v, list) else np.asarray(v) for k, v in sd.items() if k != "completed_reactions"}
    fields = {f"res:{k}": np.asarray(getattr(res, k)) for k in (
        "n_trajectories", "n_reacted", "n_escaped", "n_max_steps", "r_start", "r_escape", "elapsed_sec",
        "steps_per_sec", "dt")}
    out[name] = dict(digest=system_digest(s), n_traj=n_traj, seed=seed, max_steps=max_steps,
                     save_interval=save_interval, k_b=sim._k_b, D_rel=D_rel,
                     written=np.array([f for f, _ in written]), **arrays, **fields, **rec)


# State-machine reaction sets: (name, state_before, state_after, (receptor atom, ligand atom, cutoff)).
SM_TWO_SPHERE = {"first_state": "b_surface", "min_core_rxn_dt": 0.0,
                 "reactions": [("b_6", "b_surface", "6", (1, 1, 6.0)), ("6_3", "6", "3", (1, 1, 3.0))]}
SM_C2 = {"first_state": "A", "min_core_rxn_dt": 0.05,
         "reactions": [("A_B", "A", "B", (29, 0, 15.0)), ("B_C", "B", "C", (1, 1, 14.0)), ("B_A", "B", "A", (3, 2, 12.0))]}


def gen_run_sm(out, name, s, sm, n_traj, seed, max_steps):
    """A reference run with state-machine reactions: outcomes, step and return counts, per-reaction
    fire counts (discrete test and Brownian bridge) and the completed_reactions record."""
    with tempfile.TemporaryDirectory() as work:
        sim, mob = build_sim(s, n_traj, seed, max_steps, work, sm=sm)
        with quiet():
            res = sim.run()
    sd = res.sim_data
    rx = sm["reactions"]
    out[name] = dict(digest=system_digest(s), n_traj=n_traj, seed=seed, max_steps=max_steps,
                     n_reacted=res.n_reacted, n_escaped=res.n_escaped, n_max_steps=res.n_max_steps,
                     outcome=sd["outcome"], n_steps=sd["n_steps"], n_returns=sd["n_returns"],
                     return_prob=sim._return_prob, k_b=sim._k_b,
                     fires_discrete=np.asarray(sim._sm_rxn_fire_counts_discrete),
                     fires_bridge=np.asarray(sim._sm_rxn_fire_counts_bridge),
                     n_fired=np.array([r["n_fired"] for r in sd["completed_reactions"]]),
                     state_index_before=np.asarray(sim._sm_rxn_state_before_idx),
                     state_index_after=np.asarray(sim._sm_rxn_state_after_idx),
                     state_terminal=np.asarray(sim._sm_state_is_terminal),
                     rx_names=np.array([r[0] for r in rx]), rx_before=np.array([r[1] for r in rx]),
                     rx_after=np.array([r[2] for r in rx]), rx_pairs=np.array([r[3] for r in rx], dtype=float),
                     first_state=sm["first_state"], min_core_rxn_dt=sm["min_core_rxn_dt"])


PIPE_DIR = HERE / "pipeline"

PIPE_INPUT = """<?xml version="1.0" encoding="UTF-8"?>
<pystarc>
  <receptor_pqr>rec.pqr</receptor_pqr>
  <ligand_pqr>lig.pqr</ligand_pqr>
  <rxns_xml>rxns_sm.xml</rxns_xml>
  <work_dir>work</work_dir>
  <bd_milestone_radius>12.5</bd_milestone_radius>
  <bd_milestone_radius_inner> 4.0 </bd_milestone_radius_inner>
  <debye_length> 9.5 </debye_length>
  <sdie>80</sdie>
  <desolvation_alpha></desolvation_alpha>
  <hydrodynamic_interactions>yes</hydrodynamic_interactions>
  <overlap_check>0</overlap_check>
  <lj_forces>1</lj_forces>
  <multipole_fallback>False</multipole_fallback>
  <n_trajectories>321</n_trajectories>
  <max_steps>4321</max_steps>
  <seed>99</seed>
  <r_hydro_rec>2.25</r_hydro_rec>
  <minimum_core_reaction_dt>0.05</minimum_core_reaction_dt>
  <state_machine_reactions>TRUE</state_machine_reactions>
  <ghost_atoms>auto</ghost_atoms>
  <temperature>310.0</temperature>
  <outputs>
    <save_interval>5</save_interval>
    <p_commit>false</p_commit>
    <energetics>no</energetics>
  </outputs>
</pystarc>
"""

PIPE_REC = """REMARK synthetic receptor: chain column, element column, a 4-letter residue
ATOM      1  N   ALA A   1      11.104   6.134  -6.504 -0.3000 1.8240
ATOM      2  CA  ALA A   1      11.639   6.071  -5.147  0.0337 1.9080 C
ATOM      3  CB  NTHR    2       9.000   1.000   2.000  0.1000 1.5000
HETATM    4  O1  LIG     3      -2.345  -7.890  10.000 -0.5000 1.6612
ATOM      5  C   ALA A   4       1.250  -3.500   0.750  0.6500 1.7000
END
"""

PIPE_LIG = """ATOM      1  C1  BEN     1       0.500   0.250  -0.125  0.2500 1.7000
ATOM      2  C2  BEN     1      -0.500   1.250   0.875 -0.1250 1.7000
ATOM      3  N1  BEN     1       1.500  -1.000   0.000  0.8750 1.5500
"""

PIPE_RXNS_FLAT = """<?xml version="1.0"?>
<roottag>
  <reactions>
    <reaction>
      <n>first</n>
      <criterion>
        <n_needed>2</n_needed>
        <pair><atoms>1 2</atoms><distance>5.5</distance></pair>
        <pair><atom1>3 -0.5 6.25</atom1><atom2>1 0.2</atom2></pair>
      </criterion>
    </reaction>
    <reaction>
      <n>second</n>
      <criterion>
        <pair><atom1>5</atom1><atom2>3</atom2></pair>
        <pair><atoms>4 4</atoms><distance>3.0</distance></pair>
      </criterion>
    </reaction>
  </reactions>
</roottag>
"""

PIPE_RXNS_SM = """<?xml version="1.0"?>
<roottag>
  <first_state> outer </first_state>
  <reactions>
    <reaction>
      <n> outer_mid </n>
      <state_before> outer </state_before>
      <state_after> mid </state_after>
      <criterion><n_needed>1</n_needed><pair><atoms>6 4</atoms><distance>9.0</distance></pair></criterion>
    </reaction>
    <reaction>
      <n> empty </n>
      <state_before> mid </state_before>
      <state_after> nowhere </state_after>
      <criterion><n_needed>1</n_needed></criterion>
    </reaction>
    <reaction>
      <n> mid_in </n>
      <state_before> mid </state_before>
      <state_after> inner </state_after>
      <criterion><pair><atoms>6 4</atoms><distance>4.0</distance></pair></criterion>
    </reaction>
    <reaction>
      <n> mid_back </n>
      <state_before> mid </state_before>
      <state_after></state_after>
      <criterion><pair><atoms>1 1</atoms><distance>7.5</distance></pair></criterion>
    </reaction>
  </reactions>
</roottag>
"""


def gen_pipeline(out):
    """Input files of the pipeline tests (synthetic, written here) and what the reference's
    input parser, PQR reader/writer, GHO injection, rxns parsers and hydrodynamic-radius cache make
    of them."""
    import os
    import dataclasses
    from pystarc.pipeline import input_parser, geometry
    from pystarc.pipeline import prepare_bd_surface as pbs
    from pystarc.structures.pqr_io import parse_pqr_records

    PIPE_DIR.mkdir(exist_ok=True)
    files = {"input.xml": PIPE_INPUT, "rec.pqr": PIPE_REC, "lig.pqr": PIPE_LIG, "rxns_flat.xml": PIPE_RXNS_FLAT,
             "rxns_sm.xml": PIPE_RXNS_SM}
    for k, v in files.items():
        (PIPE_DIR / k).write_text(v)
    ref = {}
    cwd = os.getcwd()
    with tempfile.TemporaryDirectory() as tmp:
        os.chdir(tmp)  # the reference parser creates its work_dir relative to the working directory
        try:
            with quiet():
                cfg = input_parser.parse(PIPE_DIR / "input.xml")
        finally:
            os.chdir(cwd)
        ref["config"] = {f.name: (str(getattr(cfg, f.name)) if isinstance(getattr(cfg, f.name), Path)
                                  else getattr(cfg, f.name))
                         for f in dataclasses.fields(cfg) if f.name != "outputs"}
        ref["outputs"] = dataclasses.asdict(cfg.outputs)
        for name in ("rec.pqr", "lig.pqr"):
            recs = parse_pqr_records(PIPE_DIR / name)
            ref[name] = [[r.serial, r.name, r.resname, r.resid, r.x, r.y, r.z, r.charge, r.radius] for r in recs]
            atoms = pbs.centre_at_origin(pbs.read_pqr(PIPE_DIR / name))
            atoms = pbs.inject_gho(atoms)
            w = Path(tmp) / name
            pbs.write_pqr(atoms, w)
            ref[name + ".written"] = w.read_text()
            with quiet():
                g = geometry.analyse_molecule(w, srad=1.5)
            cache = sorted(Path(tmp).glob(name + ".r_hydro_*.cache"))
            ref[name + ".cache"] = [cache[0].name, cache[0].read_text()] if cache else None
            ref[name + ".r_hydro"] = g.hydrodynamic_r
        for name in ("rxns_flat.xml", "rxns_sm.xml"):
            pairs, nn = geometry._parse_rxns_xml_criteria(PIPE_DIR / name)
            ref[name + ".flat"] = [[[p.rec_index, p.lig_index, p.cutoff] for p in pairs], nn]
            groups, first = geometry._parse_rxns_xml_reaction_groups(PIPE_DIR / name)
            ref[name + ".groups"] = [[[g.name, g.state_before, g.state_after,
                                       [[p.rec_index, p.lig_index, p.cutoff] for p in g.pairs], g.n_needed]
                                      for g in groups], first]
    (HERE / "pipeline_ref.json").write_text(json.dumps(ref, indent=1, sort_keys=True) + "\n")


def two_sphere_example():
    """The reference's two-charged-spheres example (examples/two_charged_spheres) on a synthetic grid."""
    from pystarc_b200.synth import BDSystem, sphere_dh_grid

    rec_pos, lig_pos = np.zeros((2, 3)), np.zeros((2, 3))
    q_r, q_l = np.array([1.0, 0.0]), np.array([-1.0, 0.0])
    r_r = np.array([1.0, 0.0])
    g = sphere_dh_grid(1.0, 1.0, (33, 33, 33), 1.0, 7.828, 78.0 * 0.000142)
    return BDSystem("two_sphere_example", rec_pos, q_r, r_r, lig_pos, q_l, r_r.copy(), [g], [], [], [(0, 0, 2.5)], 1,
                    r_start=10.0, r_escape=20.0, r_hydro_rec=1.005, r_hydro_lig=1.005, debye=7.828, sdie=78.0,
                    eta=1.002e-3, alpha=0.0, hi=False, overlap=False)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("PYSTARC_REFERENCE"),
                    help="path of the PySTARC checkout (default: $PYSTARC_REFERENCE)")
    ap.add_argument("--only", nargs="*", help="regenerate only these fixtures (the manifest keeps the others)")
    args = ap.parse_args()
    if not args.reference:
        ap.error("name the reference checkout with --reference or PYSTARC_REFERENCE")
    sys.path.insert(0, str(REPO / "oracle" / "cupy_standin"))
    sys.path.insert(0, str(REPO))
    sys.path.insert(1, args.reference)
    from pystarc_b200 import synth

    out = {}
    c2 = synth.config2(scale=0.3)
    c3 = synth.config3(scale=0.25)
    jobs = {
        "k1": lambda: gen_k1(out),
        "physics": lambda: gen_physics(out),
        "bradius": lambda: gen_bradius(out),
        "engine_c2": lambda: gen_engine(out, "engine_c2", c2, 96, 3.0, 40.0, 21),
        "engine_c3": lambda: gen_engine(out, "engine_c3", c3, 64, 4.0, 40.0, 22),
        "engine_wca_c2": lambda: gen_engine_wca(out, "engine_wca_c2", c2, 64, 5.0, 11.0, 23),
        "engine_wca_c3": lambda: gen_engine_wca(out, "engine_wca_c3", c3, 48, 5.0, 11.0, 24),
        "run_two_sphere": lambda: gen_run(out, "run_two_sphere", two_sphere_example(), 2000, 11111113, 1_000_000),
        "run_c2": lambda: gen_run(out, "run_c2", c2, 160, 424242, 400, trace_steps=100),
        "run_c3": lambda: gen_run(out, "run_c3", c3, 64, 515151, 150, trace_steps=150),
        "run_lj_c2": lambda: gen_run(out, "run_lj_c2", c2, 160, 424242, 400, use_lj=True),
        "writer_two_sphere": lambda: gen_writer(out, "writer_two_sphere", two_sphere_example(), 300, 20261205,
                                                1_000_000, 100),
        "run_sm_two_sphere": lambda: gen_run_sm(out, "run_sm_two_sphere", two_sphere_example(), SM_TWO_SPHERE, 1000,
                                                31337, 1_000_000),
        "run_sm_c2": lambda: gen_run_sm(out, "run_sm_c2", c2, SM_C2, 160, 434343, 600),
    }
    jobs["pipeline"] = lambda: gen_pipeline(out)
    for k, job in jobs.items():
        if not args.only or k in args.only:
            job()
    manifest = HERE / "MANIFEST.json"
    meta = json.loads(manifest.read_text()) if args.only and manifest.exists() else {}
    for k, v in out.items():
        np.savez_compressed(HERE / f"{k}.npz", **{kk: np.asarray(vv) for kk, vv in v.items()})
        meta[k] = sorted(v.keys())
    manifest.write_text(json.dumps(meta, indent=1, sort_keys=True) + "\n")
    print("wrote", ", ".join(sorted(out)))


if __name__ == "__main__":
    main()
