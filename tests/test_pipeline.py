"""The input.xml path (pystarc_b200.pipeline) against what the reference's pipeline helpers make of the
same input files (tests/golden/pipeline_ref.json, written by tests/golden/make_golden.py)."""

import json
import shutil
from pathlib import Path

import numpy as np
import pytest

from pystarc_b200 import pipeline as pl

HERE = Path(__file__).resolve().parent
PIPE = HERE / "golden" / "pipeline"


@pytest.fixture(scope="module")
def ref():
    return json.loads((HERE / "golden" / "pipeline_ref.json").read_text())


def test_parse_input_matches_reference(ref):
    cfg = pl.parse_input(PIPE / "input.xml")
    for k, v in ref["config"].items():
        assert getattr(cfg, k) == v, k
    assert set(ref["config"]) == {t for t, _, _ in pl._FIELDS}
    for k, v in ref["outputs"].items():
        assert getattr(cfg.outputs, k) == v, k
    assert cfg.work_path == PIPE / "work"


def test_parse_input_requires_structures(tmp_path):
    p = tmp_path / "in.xml"
    p.write_text("<pystarc><n_trajectories>10</n_trajectories></pystarc>")
    with pytest.raises(ValueError):
        pl.parse_input(p)
    p.write_text("<pystarc><receptor_pqr>a</receptor_pqr><ligand_pqr>b</ligand_pqr>"
                 "<n_trajectories>0</n_trajectories></pystarc>")
    with pytest.raises(ValueError):
        pl.parse_input(p)


@pytest.mark.parametrize("name", ["rec.pqr", "lig.pqr"])
def test_read_pqr_matches_reference(ref, name):
    got = [[a.serial, a.name, a.resname, a.resid, a.x, a.y, a.z, a.charge, a.radius]
           for a in pl.read_pqr(PIPE / name)]
    assert got == ref[name]


@pytest.mark.parametrize("name", ["rec.pqr", "lig.pqr"])
def test_gho_injection_writes_the_reference_file(ref, tmp_path, name):
    atoms, changed = pl.centre_and_inject_gho(pl.read_pqr(PIPE / name))
    assert changed
    pl.write_pqr(atoms, tmp_path / name)
    assert (tmp_path / name).read_text() == ref[name + ".written"]
    # a file that already has its GHO atom is left alone
    again, changed = pl.centre_and_inject_gho(pl.read_pqr(tmp_path / name))
    assert not changed and len(again) == len(atoms)


@pytest.mark.parametrize("name", ["rxns_flat.xml", "rxns_sm.xml"])
def test_rxns_parsers_match_reference(ref, name):
    pairs, nn = pl.flattened_pairs(PIPE / name)
    assert [[a, b, c] for a, b, c in pairs] == ref[name + ".flat"][0] and nn == ref[name + ".flat"][1]
    groups, first = pl.parse_rxns(PIPE / name)
    want, want_first = ref[name + ".groups"]
    assert first == want_first
    assert [[g.name, g.state_before, g.state_after, [list(p) for p in g.pairs], g.n_needed] for g in groups] == want


def test_unparsable_rxns_gives_no_reactions(tmp_path):
    p = tmp_path / "bad.xml"
    p.write_text("<roottag><reaction>")
    assert pl.flattened_pairs(p) == ([], -1)
    assert pl.parse_rxns(p) == ([], None)


@pytest.mark.parametrize("name", ["rec.pqr", "lig.pqr"])
def test_hydrodynamic_radius_from_xml_or_reference_cache(ref, tmp_path, name):
    path = tmp_path / name
    path.write_text(ref[name + ".written"])
    atoms = pl.read_pqr(path)
    with pytest.raises(FileNotFoundError):
        pl.hydrodynamic_radius(path, atoms, 0.0, 1.5)
    cache_name, text = ref[name + ".cache"]
    (tmp_path / cache_name).write_text(text)
    assert pl.hydrodynamic_radius(path, atoms, 0.0, 1.5) == pytest.approx(ref[name + ".r_hydro"], rel=1e-8)
    assert pl.hydrodynamic_radius(path, atoms, 2.5, 1.5) == 2.5


def _cfg(**over):
    cfg = pl.parse_input(PIPE / "input.xml")
    cfg.values.update(over)
    return cfg


def test_reaction_pathway_state_machine_flattened_and_gho():
    rec = pl.read_pqr(PIPE / "rec.pqr")
    lig = pl.read_pqr(PIPE / "lig.pqr")
    ps = pl.reaction_pathway(_cfg(), rec, lig)
    assert ps.first_state == "outer"
    assert [(r.name, r.state_before, r.state_after) for r in ps.reactions] == [
        ("outer_mid", "outer", "mid"), ("mid_in", "mid", "inner"), ("mid_back", "mid", None)]
    assert [(p.mol1_atom_index, p.mol2_atom_index, p.distance_cutoff) for r in ps.reactions
            for p in r.criteria.pairs] == [(5, 3, 9.0), (5, 3, 4.0), (0, 0, 7.5)]
    flat = pl.reaction_pathway(_cfg(state_machine_reactions=False), rec, lig)
    assert len(flat.reactions) == 1 and flat.reactions[0].state_before is None
    assert flat.reactions[0].criteria.n_needed == 1 and len(flat.reactions[0].criteria.pairs) == 3
    manual = pl.reaction_pathway(_cfg(state_machine_reactions=False, rxns_xml="", ghost_atoms="1,2,3.5\n0,0,4"),
                                 rec, lig)
    assert [(p.mol1_atom_index, p.mol2_atom_index, p.distance_cutoff)
            for p in manual.reactions[0].criteria.pairs] == [(1, 2, 3.5), (0, 0, 4.0)]
    assert manual.reactions[0].criteria.n_needed == -1
    rec_g, _ = pl.centre_and_inject_gho(pl.read_pqr(PIPE / "rec.pqr"))
    lig_g, _ = pl.centre_and_inject_gho(pl.read_pqr(PIPE / "lig.pqr"))
    auto = pl.reaction_pathway(_cfg(state_machine_reactions=False, rxns_xml=""), rec_g, lig_g)
    p = auto.reactions[0].criteria.pairs[0]
    assert (p.mol1_atom_index, p.mol2_atom_index, p.distance_cutoff) == (len(rec_g) - 1, len(lig_g) - 1, 4.0)
    with pytest.raises(RuntimeError):
        pl.reaction_pathway(_cfg(state_machine_reactions=False, rxns_xml=""), rec, lig)


def test_reaction_index_past_the_molecule_is_an_index_error(tmp_path):
    """A reaction atom that the prepared molecule does not have stops the run before any grid is
    uploaded, with the IndexError the reference raises when it builds its simulator."""
    rec, _ = pl.centre_and_inject_gho(pl.read_pqr(PIPE / "rec.pqr"))
    lig, _ = pl.centre_and_inject_gho(pl.read_pqr(PIPE / "lig.pqr"))
    for sm in (True, False):  # both reaction files' pairs are in range once the GHO atoms are there
        pl.check_reaction_indices(pl.reaction_pathway(_cfg(state_machine_reactions=sm), rec, lig), len(rec),
                                  len(lig), "rxns")
    bad = tmp_path / "rxns_bad.xml"
    bad.write_text((PIPE / "rxns_flat.xml").read_text().replace("<atom1>5</atom1>", f"<atom1>{len(rec) + 1}</atom1>"))
    pw = pl.reaction_pathway(_cfg(state_machine_reactions=False, rxns_xml=str(bad)), rec, lig)
    with pytest.raises(IndexError, match="reaction pair 3 names receptor atom"):
        pl.check_reaction_indices(pw, len(rec), len(lig), bad.name)
    pw = pl.reaction_pathway(_cfg(state_machine_reactions=False, rxns_xml="", ghost_atoms=f"0,{len(lig)},4"), rec, lig)
    with pytest.raises(IndexError, match="ligand atom"):
        pl.check_reaction_indices(pw, len(rec), len(lig), "ghost_atoms")
    # the last atom, and NumPy's -1 as the reference reads it
    pw = pl.reaction_pathway(_cfg(state_machine_reactions=False, rxns_xml="", ghost_atoms=f"{len(rec) - 1},-1,4"),
                             rec, lig)
    pl.check_reaction_indices(pw, len(rec), len(lig), "ghost_atoms")


def test_prepare_molecules_copies_centres_and_reads_back(ref, tmp_path):
    for f in ("rec.pqr", "lig.pqr", "input.xml"):
        shutil.copy(PIPE / f, tmp_path / f)
    cfg = pl.parse_input(tmp_path / "input.xml")
    mol_rec, mol_lig = pl.prepare_molecules(cfg)
    assert (tmp_path / "work" / "receptor.pqr").read_text() == ref["rec.pqr.written"]
    assert (tmp_path / "work" / "ligand.pqr").read_text() == ref["lig.pqr.written"]
    assert mol_rec.atoms[-1].name == "GHO" and len(mol_lig) == 4
    np.testing.assert_allclose(mol_rec.positions_array()[0], [4.974, 5.771, -6.724])


def test_missing_grids_or_radii_name_the_missing_step(tmp_path):
    """Without APBS's DX files, or without a hydrodynamic radius, the run stops before any GPU work."""
    for f in ("rec.pqr", "lig.pqr", "rxns_sm.xml"):
        shutil.copy(PIPE / f, tmp_path / f)
    xml = (PIPE / "input.xml").read_text()
    (tmp_path / "input.xml").write_text(xml.replace("<r_hydro_rec>2.25</r_hydro_rec>",
                                                    "<r_hydro_rec>2.25</r_hydro_rec><r_hydro_lig>1.5</r_hydro_lig>"))
    with pytest.raises(FileNotFoundError, match="APBS"):
        pl.build(tmp_path / "input.xml")
    (tmp_path / "input.xml").write_text(xml)  # no ligand radius and no cached Monte-Carlo value
    with pytest.raises(FileNotFoundError, match="r_hydro"):
        pl.build(tmp_path / "input.xml")


def test_main_prints_usage(capsys):
    assert pl.main(["--help"]) == 0
    assert "input.xml" in capsys.readouterr().out


def test_b200_block_sets_engine_options(tmp_path):
    """Engine-only keys in a <b200> block; keyword arguments override them, unknown keys and values fail."""
    xml = (PIPE / "input.xml").read_text()
    close = xml.rstrip().rsplit("</", 1)
    block = ("<b200><precision>mixed</precision><hi_mode>zuk</hi_mode><steps_per_launch>32</steps_per_launch>"
             "<verbose>false</verbose><layout>58</layout></b200>")
    p = tmp_path / "input.xml"
    p.write_text(close[0] + block + "</" + close[1])
    cfg = pl.parse_input(p)
    assert cfg.b200 == {"precision": "mixed", "hi_mode": "zuk", "steps_per_launch": 32, "verbose": False,
                        "layout": 58}
    assert cfg.n_trajectories == pl.parse_input(PIPE / "input.xml").n_trajectories  # reference tags unchanged
    opts = pl.engine_options(cfg, precision=None, termination="complete")
    assert opts == {"precision": "mixed", "torque_mode": "zero", "device": 0, "hi_mode": "zuk",
                    "steps_per_launch": 32, "verbose": False, "layout": 58, "termination": "complete"}
    assert pl.engine_options(cfg, precision="fp64")["precision"] == "fp64"
    assert pl.engine_options(pl.parse_input(PIPE / "input.xml")) == {"precision": "fp64", "torque_mode": "zero",
                                                                    "device": 0}
    for bad, msg in (("<b200><precision>half</precision></b200>", "not one of"),
                     ("<b200><warp_size>64</warp_size></b200>", "unknown key"),
                     ("<b200><slots>many</slots></b200>", "not an integer")):
        p.write_text(close[0] + bad + "</" + close[1])
        with pytest.raises(ValueError, match=msg):
            pl.parse_input(p)
