"""The BD stage of ``run_pystarc.py input.xml`` on the B200 engine.

The reference's pipeline (pystarc/pipeline/pipeline.py:57-457) runs six steps:
PDB extraction, ligand parameterisation, PQR building, APBS grids, geometry and
reactions, and the BD run.  Steps 1-4 need AmberTools and APBS and are not
part of the trajectory engine.  This module reads the same ``input.xml`` and a
work directory in which they have already run (the PQR files and the
``receptor[0-9].dx``, ``receptor[0-9]_born.dx`` and ``ligand[0-9]_born.dx`` grids
APBS wrote; the reference skips APBS when they are present, run_apbs.py:342-349).
It does steps 5-6 with ``B200ForceEngine`` and ``B200BatchSimulator``:

* ``parse_input``        -- input_parser.parse (input_parser.py:139-268): same tags,
                            defaults and casts
* ``read_pqr`` / ``write_pqr`` / ``centre_and_inject_gho``
                         -- the PQR step 3b (pipeline.py:127-147,
                            prepare_bd_surface.py:199-291)
* ``hydrodynamic_radius`` -- compute_geometry's radii (geometry.py:242-313): the
                            XML value when > 0, else the reference's cached
                            Monte-Carlo value next to the PQR (the MC itself is not
                            rebuilt here)
* ``reaction_pathway``   -- auto_detect_reactions and the state-machine parser
                            (geometry.py:321-621, pipeline.py:225-291)
* ``build`` / ``run``    -- the GPU branch of step 6 (pipeline.py:292-351) and the
                            output files of output_writer.write_all (:15-304),
                            written by ``pystarc_b200.output``

Engine-only options may sit in a ``<b200>`` block of the same file, which the
reference's parser ignores: ``precision`` (fp64 | mixed), ``torque_mode`` (zero |
centroid), ``hi_mode`` (reference_gpu | zuk), ``termination`` (reference |
complete), ``steps_per_launch``, ``launches_per_poll``, ``slots``, ``device``,
``layout`` and ``verbose``.  An unknown key or value is an error.

Usage: ``python -m pystarc_b200.pipeline input.xml``.
"""

from __future__ import annotations

import re
import shutil
import sys
import xml.etree.ElementTree as ET
from dataclasses import dataclass, field
from pathlib import Path
from typing import List, Optional

import numpy as np

from . import hostphys
from . import structures as st
from .dx import DXGrid

# (tag, default, cast) of every scalar field of the reference's PySTARCConfig
_FIELDS = [
    ("pdb", None, str), ("desolvation_alpha", 0.07957747, float), ("debye_length", 7.858, float),
    ("max_steps", 1000000, int), ("ligand_resname", None, str), ("ligand_charge", 0, int),
    ("work_dir", "bd_sims", str), ("protein_ff", "ff14SB", str), ("ligand_ff", "gaff", str),
    ("apbs_grid_spacing", 0.5, float), ("apbs_coarse_spacing", 2.0, float), ("n_trajectories", 10000, int),
    ("n_threads", 24, int), ("gpu", True, bool), ("seed", 1523, int), ("confidence_interval", 0.95, float),
    ("bd_milestone_radius", 30.0, float), ("bd_milestone_radius_inner", 0.0, float),
    ("state_machine_reactions", False, bool), ("ghost_atoms", "auto", str), ("rxns_xml", "", str),
    ("receptor_pqr", "", str), ("ligand_pqr", "", str), ("ion_concentration", 0.150, float),
    ("ion_radius_pos", 0.95, float), ("ion_radius_neg", 1.81, float), ("apbs_cglen", 0.0, float),
    ("apbs_fglen", 0.0, float), ("apbs_dime", 129, int), ("apbs_coarse_dime", 0, int), ("apbs_fine_dime", 0, int),
    ("gpu_force_batch", 0, int), ("pdie", 4.0, float), ("sdie", 78.0, float), ("srad", 1.5, float),
    ("temperature", 298.15, float), ("dt", 0.2, float), ("hydrodynamic_interactions", False, bool),
    ("r_hydro_rec", 0.0, float), ("r_hydro_lig", 0.0, float), ("minimum_core_dt", 0.0, float),
    ("minimum_core_reaction_dt", 0.0, float), ("max_dt", 0.0, float), ("overlap_check", True, bool),
    ("multipole_fallback", True, bool), ("lj_forces", False, bool), ("checkpoint_interval", 0, int),
    ("convergence_interval", 10, int), ("convergence_check", True, bool), ("convergence_tol", 0.05, float),
]
_OUTPUT_FLAGS = ["results_json", "trajectories_csv", "encounters_csv", "near_misses_csv", "full_paths",
                 "radial_density", "angular_map", "fpt_distribution", "contact_frequency", "milestone_flux",
                 "p_commit", "transition_matrix", "energetics", "pose_clusters"]
# engine-only keys of an optional <b200> block (no reference counterpart; the reference's tags stay as
# they are): tag -> (cast, allowed values or None)
_B200_KEYS = {
    "precision": (str, ("fp64", "mixed")), "torque_mode": (str, ("zero", "centroid")),
    "hi_mode": (str, ("reference_gpu", "zuk")), "termination": (str, ("reference", "complete")),
    "steps_per_launch": (int, None), "launches_per_poll": (int, None), "slots": (int, None),
    "device": (int, None), "layout": (int, None), "verbose": (bool, None),
}


@dataclass
class OutputConfig:
    """Which output files a run writes (input_parser.py:16-36); every flag defaults to on."""

    results_json: bool = True
    trajectories_csv: bool = True
    encounters_csv: bool = True
    near_misses_csv: bool = True
    full_paths: bool = True
    radial_density: bool = True
    angular_map: bool = True
    fpt_distribution: bool = True
    contact_frequency: bool = True
    milestone_flux: bool = True
    p_commit: bool = True
    transition_matrix: bool = True
    energetics: bool = True
    pose_clusters: bool = True
    save_interval: int = 10


@dataclass
class RunConfig:
    """The reference's PySTARCConfig fields, plus the directory of the XML file (relative paths)."""

    values: dict
    outputs: OutputConfig = field(default_factory=OutputConfig)
    xml_dir: Path = Path(".")
    b200: dict = field(default_factory=dict)  # the keys the <b200> block sets

    def __getattr__(self, name):
        try:
            return self.__dict__["values"][name]
        except KeyError:
            raise AttributeError(name) from None

    @property
    def work_path(self) -> Path:
        w = Path(self.values["work_dir"])
        return w if w.is_absolute() else self.xml_dir / w


def _cast(text, default, cast):
    if text is None:
        return default
    t = text.strip()
    if cast is bool:
        return t.lower() in ("true", "1", "yes")
    return cast(t)


def parse_input(xml_path) -> RunConfig:
    """Parse ``input.xml`` like the reference (input_parser.py:139-268).  A missing or empty tag
    takes the default; booleans are true for "true", "1" or "yes"."""
    xml_path = Path(xml_path)
    root = ET.parse(xml_path).getroot()
    vals = {}
    for tag, default, cast in _FIELDS:
        el = root.find(tag)
        vals[tag] = _cast(None if el is None else el.text, default, cast)
    outputs = OutputConfig()
    out_el = root.find("outputs")
    if out_el is not None:
        for flag in _OUTPUT_FLAGS:
            el = out_el.find(flag)
            setattr(outputs, flag, _cast(None if el is None else el.text, True, bool))
        el = out_el.find("save_interval")
        outputs.save_interval = _cast(None if el is None else el.text, 10, int)
    b200 = {}
    b_el = root.find("b200")
    if b_el is not None:
        for child in b_el:
            if child.tag not in _B200_KEYS:
                raise ValueError(f"<b200>: unknown key <{child.tag}>; known: {', '.join(sorted(_B200_KEYS))}")
            cast, allowed = _B200_KEYS[child.tag]
            try:
                v = _cast(child.text, None, cast)
            except ValueError:
                raise ValueError(f"<b200><{child.tag}>: {child.text!r} is not an integer") from None
            if v is None or (allowed is not None and v not in allowed):
                raise ValueError(f"<b200><{child.tag}>: {child.text!r} is not one of {allowed}" if allowed else
                                 f"<b200><{child.tag}>: no value")
            b200[child.tag] = v
    has_pqrs = bool(vals["receptor_pqr"] and vals["ligand_pqr"])
    if not has_pqrs and vals["pdb"] is None:
        raise ValueError("Either <pdb> or both <receptor_pqr> and <ligand_pqr> must be specified")
    if vals["n_trajectories"] < 1:
        raise ValueError("n_trajectories must be >= 1")
    return RunConfig(vals, outputs, xml_path.resolve().parent, b200)


# ----------------------------------------------------------------------------
# PQR files
# ----------------------------------------------------------------------------
@dataclass
class PQRAtom:
    serial: int
    name: str
    resname: str
    resid: int
    x: float
    y: float
    z: float
    charge: float
    radius: float


_FLOAT = re.compile(r"[-+]?(?:\d+\.\d*|\.\d+)(?:[eE][-+]?\d+)?")


def read_pqr(path) -> List[PQRAtom]:
    """ATOM/HETATM records of a PQR file.  The five decimal numbers ending the record are
    x, y, z, charge and radius, so a chain column, a trailing element symbol and numbers
    run together without a space ("-12.345-67.890") all parse."""
    atoms = []
    with open(path) as fh:
        for line in fh:
            if not (line.startswith("ATOM") or line.startswith("HETATM")):
                continue
            head = line[:6].strip()
            rest = line[len(head):]
            tok = rest.split()
            nums = _FLOAT.findall(rest)
            if len(tok) < 4 or len(nums) < 5:
                continue
            try:
                serial = int(tok[0])
                name, resname = tok[1], tok[2]
                # the residue number is the last integer token before the coordinates
                resid = 0
                for t in tok[3:]:
                    if re.fullmatch(r"[-+]?\d+", t):
                        resid = int(t)
                        break
                x, y, z, q, r = (float(v) for v in nums[-5:])
            except ValueError:
                continue
            atoms.append(PQRAtom(serial, name, resname, resid, x, y, z, q, r))
    return atoms


def write_pqr(atoms, path):
    """HETATM records in the column layout of the reference's PQRAtom.to_pqr_line
    (prepare_bd_surface.py:211-219), then END."""
    with open(path, "w") as f:
        for a in atoms:
            f.write(f"HETATM{a.serial:5d}  {a.name:<4s} {a.resname:<4s}{a.resid:5d}    "
                    f"{a.x:8.3f}{a.y:8.3f}{a.z:8.3f}  {a.charge:7.4f}  {a.radius:6.4f}\n")
        f.write("END\n")


def centre_and_inject_gho(atoms):
    """Move the centroid of the non-GHO atoms to the origin and append a GHO atom there
    (charge 0, radius 0, next serial and residue number), unless a GHO atom exists
    (pipeline.py:139-147, prepare_bd_surface.py:254-291).  Returns (atoms, changed)."""
    if any(a.name.strip().upper() == "GHO" for a in atoms):
        return atoms, False
    ctr = np.array([[a.x, a.y, a.z] for a in atoms if a.name != "GHO"]).mean(axis=0)
    for a in atoms:
        a.x -= ctr[0]
        a.y -= ctr[1]
        a.z -= ctr[2]
    atoms.append(PQRAtom(max(a.serial for a in atoms) + 1, "GHO", "GHO", max(a.resid for a in atoms) + 1,
                         0.0, 0.0, 0.0, 0.0, 0.0))
    return atoms, True


def molecule(name, atoms) -> st.Molecule:
    return st.Molecule(name, [st.Atom(index=i + 1, name=a.name, residue_name=a.resname, residue_index=a.resid,
                                      x=a.x, y=a.y, z=a.z, charge=a.charge, radius=a.radius)
                              for i, a in enumerate(atoms)])


def _resolve(path_text, *bases) -> Path:
    p = Path(path_text.strip())
    if p.is_absolute():
        return p
    for b in bases:
        if (Path(b) / p).exists():
            return Path(b) / p
    return Path(bases[0]) / p if bases else p


def prepare_molecules(cfg: RunConfig):
    """Copy the receptor and ligand PQR files into the work directory as receptor.pqr and
    ligand.pqr, centred with a GHO atom, and return them as Molecules (pipeline.py:81-147)."""
    if not (cfg.receptor_pqr and cfg.ligand_pqr):
        raise ValueError("this engine starts from receptor_pqr and ligand_pqr (PDB extraction and "
                         "AmberTools parameterisation are not part of it)")
    W = cfg.work_path
    W.mkdir(parents=True, exist_ok=True)
    out = []
    for tag, dst in (("receptor_pqr", "receptor.pqr"), ("ligand_pqr", "ligand.pqr")):
        src = _resolve(getattr(cfg, tag), cfg.xml_dir, Path.cwd())
        if not src.exists():
            raise FileNotFoundError(f"{tag} not found: {src}")
        target = W / dst
        if src.resolve() != target.resolve():
            shutil.copy(src, target)
        atoms, changed = centre_and_inject_gho(read_pqr(target))
        if changed:
            write_pqr(atoms, target)
        # the run reads the file back, with the written precision (pipeline.py:185-186)
        out.append(molecule(dst[:-4], read_pqr(target)))
    return out[0], out[1]


# ----------------------------------------------------------------------------
# Grids, geometry, reactions
# ----------------------------------------------------------------------------
def load_grids(work_dir, prefix, suffix):
    """DX grids named <prefix><digit><suffix> in the work directory, in name order (pipeline.py:312-315)."""
    return [DXGrid.from_file(p) for p in sorted(Path(work_dir).glob(f"{prefix}[0-9]{suffix}"))]


def _mc_grid_spacing(atoms, srad):
    coords = np.array([[a.x, a.y, a.z] for a in atoms])
    radii = np.array([a.radius for a in atoms])
    rb = radii + srad if srad > 0.0 else radii
    bbox = float(np.max(np.max(coords + rb[:, None], axis=0) - np.min(coords - rb[:, None], axis=0)))
    return max(0.02, min(1.0, bbox / 100.0))


def hydrodynamic_radius(pqr_path, atoms, xml_value, srad):
    """The XML value when > 0; else the Monte-Carlo radius the reference cached next to the PQR file
    (``<pqr>.r_hydro_s<spacing>_p<srad>.cache``, geometry.py:182-214)."""
    if xml_value > 0:
        return float(xml_value)
    spacing = _mc_grid_spacing(atoms, srad)
    cache = Path(str(pqr_path) + f".r_hydro_s{spacing}_p{srad:.4g}.cache")
    if cache.exists():
        return float(cache.read_text().split()[0])
    raise FileNotFoundError(f"no hydrodynamic radius for {Path(pqr_path).name}: set r_hydro_rec / r_hydro_lig in "
                            f"the input XML, or provide the reference's cached Monte-Carlo value {cache.name}")


@dataclass
class ReactionGroup:
    name: str
    state_before: Optional[str]
    state_after: Optional[str]
    pairs: list  # (receptor index, ligand index, cutoff), 0-based
    n_needed: int = -1


def _pair_of(pair_node):
    """(rec, lig, cutoff), 0-based, from <atom1>/<atom2> or <atoms>/<distance>; None if malformed."""
    a1, a2 = pair_node.find("atom1"), pair_node.find("atom2")
    try:
        if a1 is not None and a2 is not None:
            p1, p2 = a1.text.strip().split(), a2.text.strip().split()
            return int(p1[0]) - 1, int(p2[0]) - 1, float(p1[2]) if len(p1) >= 3 else 5.0
        at, dist = pair_node.find("atoms"), pair_node.find("distance")
        if at is not None and dist is not None:
            idx = at.text.strip().split()
            return int(idx[0]) - 1, int(idx[1]) - 1, float(dist.text.strip())
    except (ValueError, IndexError, AttributeError):
        return None
    return None


def parse_rxns(path):
    """Every reaction of a rxns XML file with its state labels, pairs and n_needed, and the
    <first_state> (geometry.py:321-389, :502-621).  Reactions without pairs are dropped; a file
    that does not parse gives no reactions, as in the reference."""
    try:
        root = ET.parse(str(path)).getroot()
    except (ET.ParseError, OSError):
        return [], None
    fs = root.find(".//first_state")
    first = fs.text.strip() if fs is not None and fs.text else None
    groups = []
    for rx in root.iter("reaction"):
        crit = rx.find("criterion")
        if crit is None:
            continue

        def label(tag):
            n = rx.find(tag)
            return n.text.strip() if n is not None and n.text else None

        nn = -1
        nn_node = crit.find("n_needed")
        if nn_node is not None and nn_node.text:
            try:
                nn = int(nn_node.text.strip())
            except ValueError:
                pass
        pairs = [p for p in (_pair_of(n) for n in crit.findall("pair")) if p is not None]
        if pairs:
            groups.append(ReactionGroup(label("n") or "", label("state_before"), label("state_after"), pairs, nn))
    return groups, first


def flattened_pairs(path):
    """All pairs of all reactions, and the n_needed of the last reaction that states one
    (the reference keeps overwriting it, geometry.py:337-345)."""
    try:
        root = ET.parse(str(path)).getroot()
    except (ET.ParseError, OSError):
        return [], -1
    pairs, n_needed = [], -1
    for rx in root.iter("reaction"):
        crit = rx.find("criterion")
        if crit is None:
            continue
        nn_node = crit.find("n_needed")
        if nn_node is not None:
            try:
                n_needed = int(nn_node.text.strip())
            except (ValueError, AttributeError):
                pass
        pairs += [p for p in (_pair_of(n) for n in crit.findall("pair")) if p is not None]
    return pairs, n_needed


def check_reaction_indices(pathway, n_rec, n_lig, where):
    """Reaction atom indices (0-based) must name atoms of the prepared molecules (GHO atom
    included).  The reference indexes its position arrays with them, so an index past the end
    raises IndexError when its simulator is built; this raises the same error, naming the
    reaction source, before any grid is uploaded.  Negative indices keep NumPy's meaning (from
    the end), as in the reference."""
    k = 0
    for rxn in pathway.reactions:
        for p in rxn.criteria.pairs:
            k += 1
            for idx, n, mol in ((p.mol1_atom_index, n_rec, "receptor"), (p.mol2_atom_index, n_lig, "ligand")):
                if not -n <= int(idx) < n:
                    raise IndexError(f"{where}: reaction pair {k} names {mol} atom {int(idx) + 1} (1-based), "
                                     f"but the {mol} has {n} atoms")


def reaction_pathway(cfg: RunConfig, rec_atoms, lig_atoms) -> st.PathwaySet:
    """The PathwaySet of step 6 (pipeline.py:225-291 with auto_detect_reactions, geometry.py:391-482)."""
    rxns = _resolve(cfg.rxns_xml, cfg.xml_dir, Path.cwd()) if cfg.rxns_xml and cfg.rxns_xml.strip() else None
    if cfg.state_machine_reactions and rxns is not None and rxns.exists():
        groups, first = parse_rxns(rxns)
        if groups:
            reactions = []
            for g in groups:
                crit = st.ReactionCriteria(g.name or "reaction", [st.ContactPair(*p) for p in g.pairs],
                                           n_needed=g.n_needed, state_before=g.state_before,
                                           state_after=g.state_after)
                reactions.append(st.ReactionInterface(g.name or "reaction", crit, state_before=g.state_before,
                                                      state_after=g.state_after))
            return st.PathwaySet(reactions, first_state=first)
    pairs, n_needed = None, -1
    if rxns is not None and rxns.exists():
        pairs, n_needed = flattened_pairs(rxns)
        pairs = pairs or None
    if pairs is None and cfg.ghost_atoms.strip().lower() != "auto":
        pairs = []
        for line in cfg.ghost_atoms.strip().splitlines():
            line = line.strip()
            if not line:
                continue
            parts = line.split(",")
            if len(parts) != 3:
                raise ValueError(f"ghost_atoms line must be 'rec_idx,lig_idx,cutoff': {line!r}")
            pairs.append((int(parts[0]), int(parts[1]), float(parts[2])))
        n_needed = -1
    if pairs is None:
        rg = [i for i, a in enumerate(rec_atoms) if a.name.strip().upper() == "GHO"]
        lg = [i for i, a in enumerate(lig_atoms) if a.name.strip().upper() == "GHO"]
        if not (rg and lg):
            raise RuntimeError("no reaction criterion: no rxns_xml pairs, no ghost_atoms and no GHO atoms")
        cut = cfg.bd_milestone_radius_inner if cfg.bd_milestone_radius_inner > 0 else cfg.bd_milestone_radius
        pairs, n_needed = [(rg[0], lg[0], cut)], 1
    crit = st.ReactionCriteria("stage_0", [st.ContactPair(*p) for p in pairs], n_needed=n_needed)
    return st.PathwaySet([st.ReactionInterface("stage_0", crit)])


class _Multipole:
    def __init__(self, positions, charges, sdie):
        _, self.dipole, self.quadrupole, self.four_pi_eps = hostphys.multipole(positions, charges, sdie)


# ----------------------------------------------------------------------------
# Step 6
# ----------------------------------------------------------------------------
@dataclass
class Prepared:
    cfg: RunConfig
    engine: object
    simulator: object
    mobility: object
    D_rel: float


def engine_options(cfg: RunConfig, **explicit) -> dict:
    """Engine and stepper options of a run: keyword arguments given (not None) first, then the
    input file's <b200> block, then the defaults (FP64, zero torque, device 0)."""
    opts = {"precision": "fp64", "torque_mode": "zero", "device": 0}
    opts.update(cfg.b200)
    opts.update({k: v for k, v in explicit.items() if v is not None})
    return opts


def build(xml_path, *, precision=None, torque_mode=None, device=None, **sim_options) -> Prepared:
    """Engine and stepper for ``input.xml`` from its prepared work directory (pipeline.py:292-351).
    Options come from the keyword arguments, else from the file's <b200> block (``engine_options``)."""
    from .engine import B200ForceEngine
    from .simulator import B200BatchSimulator

    cfg = parse_input(xml_path)
    opts = engine_options(cfg, precision=precision, torque_mode=torque_mode, device=device, **sim_options)
    precision, torque_mode, device = opts.pop("precision"), opts.pop("torque_mode"), opts.pop("device")
    layout = opts.pop("layout", None)
    sim_options = opts
    W = cfg.work_path
    mol_rec, mol_lig = prepare_molecules(cfg)
    rec_atoms, lig_atoms = read_pqr(W / "receptor.pqr"), read_pqr(W / "ligand.pqr")
    r_rec = hydrodynamic_radius(W / "receptor.pqr", rec_atoms, cfg.r_hydro_rec, cfg.srad)
    r_lig = hydrodynamic_radius(W / "ligand.pqr", lig_atoms, cfg.r_hydro_lig, cfg.srad)
    elec = load_grids(W, "receptor", ".dx")
    if not elec:
        raise FileNotFoundError(f"no receptor[0-9].dx grids in {W}: run the APBS step of the reference pipeline "
                                f"first (this engine reads its DX files)")
    born = load_grids(W, "receptor", "_born.dx")
    lig_born = load_grids(W, "ligand", "_born.dx")
    mob = st.MobilityTensor.from_radii(r_rec, r_lig, use_rpy=True, T=cfg.temperature)
    pathway = reaction_pathway(cfg, rec_atoms, lig_atoms)
    check_reaction_indices(pathway, len(rec_atoms), len(lig_atoms), cfg.rxns_xml or "ghost_atoms")
    r_start = cfg.bd_milestone_radius
    params = st.NAMParameters(n_trajectories=cfg.n_trajectories, dt=cfg.dt, dt_rxn=cfg.minimum_core_reaction_dt,
                              max_steps=cfg.max_steps, r_start=r_start, r_escape=2.0 * r_start, seed=cfg.seed,
                              n_threads=cfg.n_threads, hydrodynamic_interactions=cfg.hydrodynamic_interactions,
                              use_hard_sphere=True, verbose=True, minimum_core_dt=cfg.minimum_core_dt,
                              minimum_core_reaction_dt=cfg.minimum_core_reaction_dt)
    mp = _Multipole(mol_rec.positions_array(), mol_rec.charges_array(), cfg.sdie) if cfg.multipole_fallback else None
    engine = B200ForceEngine(elec_grids=elec, born_grids=born, alpha=cfg.desolvation_alpha,
                             receptor_charge=float(mol_rec.total_charge()), debye_length=cfg.debye_length,
                             sdie=cfg.sdie, lig_born_grids=lig_born, rec_positions=mol_rec.positions_array(),
                             rec_charges=mol_rec.charges_array(), multipole_expansion=mp,
                             rec_radii=mol_rec.radii_array() if cfg.lj_forces else None,
                             lig_radii=mol_lig.radii_array() if cfg.lj_forces else None, use_lj=cfg.lj_forces,
                             precision=precision, torque_mode=torque_mode, device=device, layout=layout)
    params._output_cfg = cfg.outputs
    params.max_dt = cfg.max_dt
    params.checkpoint_interval = cfg.checkpoint_interval
    params.convergence_interval = cfg.convergence_interval
    params._work_dir = str(W)
    params._kT_scale = cfg.temperature / 298.15
    params._overlap_check = cfg.overlap_check
    sim = B200BatchSimulator(mol_rec, mol_lig, mob, pathway, params, engine, **sim_options)
    return Prepared(cfg, engine, sim, mob, float(mob.relative_translational_diffusion()))


def run(xml_path, **options):
    """Build, run every trajectory and write the reference's output files (results.json,
    trajectories.csv, ... energetics.npz) plus sim_data.npz (the per-trajectory and histogram
    arrays under the reference's sim_data keys) into the work directory."""
    from .output import write_all

    prep = build(xml_path, **options)
    result = prep.simulator.run()
    sd = result.sim_data
    W = prep.cfg.work_path
    write_all(W, result, sd, prep.cfg.outputs, prep.simulator._k_b, prep.D_rel, prep.cfg.confidence_interval,
              verbose=False)
    arrays = {k: np.asarray(v) for k, v in sd.items() if k != "completed_reactions" and not isinstance(v, list)}
    np.savez_compressed(W / "sim_data.npz", **arrays)
    return prep, result


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    if not argv or argv[0] in ("-h", "--help"):
        print(__doc__)
        return 0
    # the reference's console reports while the BD stage runs, unless the <b200> block says otherwise
    extra = {} if "verbose" in parse_input(argv[0]).b200 else {"verbose": True}
    prep, result = run(argv[0], **extra)
    print(result.summary(prep.D_rel, prep.simulator._k_b, prep.cfg.confidence_interval))
    return 0


if __name__ == "__main__":
    sys.exit(main())
