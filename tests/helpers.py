"""Shared test helpers: build oracle objects and engine inputs from a synthetic system."""

from __future__ import annotations

import hashlib
from pathlib import Path

import numpy as np

from oracle.forces import FarField, OracleForceEngine, OracleGrid, multipole_moments
from oracle.stepper import StepParams, StepSystem, n_needed_of
from pystarc_b200 import synth
from pystarc_b200.simulator import zuk_kT_eta

GOLDEN = Path(__file__).resolve().parent / "golden"


def golden(name):
    return dict(np.load(GOLDEN / f"{name}.npz", allow_pickle=False))


def grid_digest(grids):
    h = hashlib.sha256()
    for g in grids:
        h.update(np.ascontiguousarray(np.asarray(g.data, dtype=np.float32)).tobytes())
        h.update(np.asarray(g.origin, dtype=np.float64).tobytes())
        h.update(np.asarray(g.delta, dtype=np.float64).tobytes())
    return h.hexdigest()


def system_digest(s):
    return grid_digest(list(s.elec_grids) + list(s.born_grids) + list(s.lig_born_grids))


def two_sphere_example():
    rec_pos, lig_pos = np.zeros((2, 3)), np.zeros((2, 3))
    g = synth.sphere_dh_grid(1.0, 1.0, (33, 33, 33), 1.0, 7.828, 78.0 * 0.000142)
    return synth.BDSystem("two_sphere_example", rec_pos, np.array([1.0, 0.0]), np.array([1.0, 0.0]), lig_pos,
                          np.array([-1.0, 0.0]), np.array([1.0, 0.0]), [g], [], [], [(0, 0, 2.5)], 1,
                          r_start=10.0, r_escape=20.0, r_hydro_rec=1.005, r_hydro_lig=1.005, debye=7.828,
                          sdie=78.0, eta=1.002e-3, alpha=0.0, hi=False, overlap=False)


_CACHE = {}


def system(name):
    """Small synthetic systems used by the golden fixtures (cached per process)."""
    if name not in _CACHE:
        if name == "c2":
            _CACHE[name] = synth.config2(scale=0.3)
        elif name == "c3":
            _CACHE[name] = synth.config3(scale=0.25)
        elif name == "two_sphere":
            _CACHE[name] = two_sphere_example()
        else:
            raise KeyError(name)
    return _CACHE[name]


def oracle_engine(s, multipole=True, born_chunk_skip=True, use_lj=False):
    if multipole and s.multipole:
        dip, quad = multipole_moments(s.rec_pos, s.rec_q)
        ff = FarField(float(np.sum(s.rec_q)), s.debye, s.sdie, dip, quad, 4.0 * np.pi * (s.sdie * 0.000142))
    else:
        ff = FarField(float(np.sum(s.rec_q)), s.debye, s.sdie)
    return OracleForceEngine([OracleGrid.from_dx(g) for g in s.elec_grids],
                             [OracleGrid.from_dx(g) for g in s.born_grids], s.alpha, ff,
                             [OracleGrid.from_dx(g) for g in s.lig_born_grids] or None, s.rec_pos, s.rec_q,
                             born_chunk_skip=born_chunk_skip, rec_radii=s.rec_r, lig_radii=s.lig_r, use_lj=use_lj)


def step_system(s, engine=None):
    mob = s.mobility()
    body = s.lig_pos - s.lig_pos.mean(axis=0)
    P = len(s.pairs)
    return StepSystem(lig_body=body, lig_q=np.asarray(s.lig_q, dtype=float), rec_pos=np.asarray(s.rec_pos, float),
                      engine=engine or oracle_engine(s),
                      rxn_rec_pos=np.asarray([s.rec_pos[a] for a, _, _ in s.pairs], dtype=float).reshape(P, 3),
                      rxn_lig_idx=np.asarray([b for _, b, _ in s.pairs], dtype=np.int64),
                      rxn_cutoff=np.asarray([c for _, _, c in s.pairs], dtype=float),
                      n_needed=n_needed_of(s.n_needed, P), D_t=mob.relative_translational_diffusion(),
                      D_r=mob.relative_rotational_diffusion(), r_h_rec=s.r_hydro_rec, r_h_lig=s.r_hydro_lig,
                      # Molecule.total_charge sums atom by atom (pystarc/structures/molecules.py:69-70)
                      q_rec_total=sum(float(v) for v in s.rec_q), q_lig_total=sum(float(v) for v in s.lig_q),
                      debye=s.debye, hi_kT_eta=zuk_kT_eta(mob))


def sm_spec(g):
    """State-machine reaction set of a golden run: names, source and destination labels, pairs, first state."""
    pairs = [(int(a), int(b), float(c)) for a, b, c in np.asarray(g["rx_pairs"])]
    return ([str(x) for x in g["rx_names"]], [str(x) for x in g["rx_before"]], [str(x) for x in g["rx_after"]],
            pairs, str(g["first_state"]))


def sm_step_system(s, g, engine=None):
    """Oracle stepper system with the state-machine reactions of golden run ``g``."""
    from oracle.stepper import sm_tables

    names, sb, sa, pairs, first = sm_spec(g)
    ss = step_system(s, engine)
    P = len(pairs)
    ss.rxn_rec_pos = np.asarray([s.rec_pos[a] for a, _, _ in pairs], dtype=float).reshape(P, 3)
    ss.rxn_lig_idx = np.asarray([b for _, b, _ in pairs], dtype=np.int64)
    ss.rxn_cutoff = np.asarray([c for _, _, c in pairs], dtype=float)
    ss.n_needed = n_needed_of(1, P)
    ss.sm_before, ss.sm_after, ss.sm_terminal = sm_tables(sb, sa, first)
    return ss


def sm_pathway(g):
    """The same reaction set as a PathwaySet of labelled reactions (the drop-in's input)."""
    from pystarc_b200 import structures as st

    names, sb, sa, pairs, first = sm_spec(g)
    rx = []
    for name, b, a, (i, j, c) in zip(names, sb, sa, pairs):
        crit = st.ReactionCriteria(name, [st.ContactPair(i, j, c)], n_needed=1, state_before=b, state_after=a)
        rx.append(st.ReactionInterface(name, crit, state_before=b, state_after=a))
    return st.PathwaySet(rx, first_state=first)


def step_params(s, n_traj, seed, max_steps, hi_mode="reference_gpu"):
    return StepParams(n_traj=n_traj, seed=seed, r_b=s.r_start, r_esc=s.r_escape, max_steps=max_steps,
                      max_dt=s.max_dt, use_hi=s.hi, overlap=s.overlap, kT_scale=s.temperature / 298.15,
                      hi_mode=hi_mode)
