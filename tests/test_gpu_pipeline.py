"""input.xml end to end on the GPU: a work directory prepared as the reference's steps 1-4 leave it
(PQR files, APBS-named DX grids), run through pystarc_b200.pipeline, against the same system built
directly."""

import json

import numpy as np
import pytest

from tests.helpers import system

pytestmark = pytest.mark.gpu

INPUT = """<?xml version="1.0"?>
<pystarc>
  <receptor_pqr>receptor_in.pqr</receptor_pqr>
  <ligand_pqr>ligand_in.pqr</ligand_pqr>
  <rxns_xml>rxns.xml</rxns_xml>
  <work_dir>bd_sims</work_dir>
  <bd_milestone_radius>10.0</bd_milestone_radius>
  <r_hydro_rec>1.005</r_hydro_rec>
  <r_hydro_lig>1.005</r_hydro_lig>
  <debye_length>7.828</debye_length>
  <sdie>78.0</sdie>
  <desolvation_alpha>0.0</desolvation_alpha>
  <overlap_check>false</overlap_check>
  <multipole_fallback>true</multipole_fallback>
  <n_trajectories>3000</n_trajectories>
  <max_steps>1000000</max_steps>
  <seed>{seed}</seed>
  <state_machine_reactions>{sm}</state_machine_reactions>
</pystarc>
"""

RXNS = """<?xml version="1.0"?>
<top>
  <first_state> b_surface </first_state>
  <reactions>
    <reaction>
      <n> association </n>
      <state_before> b_surface </state_before>
      <state_after> contact </state_after>
      <criterion>
        <n_needed> 1 </n_needed>
        <pair><atoms> 1 1 </atoms><distance> 2.5 </distance></pair>
      </criterion>
    </reaction>
  </reactions>
</top>
"""


def _work(tmp_path, sm):
    s = system("two_sphere")
    (tmp_path / "receptor_in.pqr").write_text(
        "ATOM      1  U   FOO    1       0.000   0.000   0.000  1.0000  1.0000\n")
    (tmp_path / "ligand_in.pqr").write_text(
        "ATOM      1  U   FOO    1       0.000   0.000   0.000 -1.0000  1.0000\n")
    (tmp_path / "rxns.xml").write_text(RXNS)
    (tmp_path / "input.xml").write_text(INPUT.format(seed=s.seed, sm="true" if sm else "false"))
    (tmp_path / "bd_sims").mkdir()
    s.elec_grids[0].write(tmp_path / "bd_sims" / "receptor0.dx")  # the name APBS gives the grid
    return s


@pytest.mark.parametrize("sm", [False, True])
def test_input_xml_run_matches_the_directly_built_system(tmp_path, sm):
    """Both reaction modes give the single-reaction example the same fates as the direct build."""
    from pystarc_b200 import pipeline
    from pystarc_b200.engine import B200ForceEngine
    from pystarc_b200.simulator import B200BatchSimulator

    s = _work(tmp_path, sm)
    prep, res = pipeline.run(tmp_path / "input.xml", termination="complete")
    assert prep.simulator._sm_active == sm
    W = tmp_path / "bd_sims"
    rec = json.loads((W / "results.json").read_text())
    assert rec["n_reacted"] == res.n_reacted and rec["n_trajectories"] == 3000
    assert rec["r_start"] == 10.0 and rec["r_escape"] == 20.0 and rec["k_on"] > 0
    assert ("completed_reactions" in rec) == sm
    sd = np.load(W / "sim_data.npz")
    assert sd["outcome"].shape == (3000,) and "radial_counts" in sd.files
    # the reference's output files (pipeline/output_writer.py:15-304); pose clusters need > 5 reactions
    for name in ("results.json", "trajectories.csv", "encounters.csv", "near_misses.csv", "paths.npz",
                 "radial_density.csv", "angular_map.npz", "fpt_distribution.csv", "contact_frequency.csv",
                 "milestone_flux.csv", "p_commit.npz", "transition_matrix.npz", "energetics.npz",
                 "pose_clusters.csv"):
        assert (W / name).exists(), name
    assert len((W / "trajectories.csv").read_text().splitlines()) == 3001
    paths = np.load(W / "paths.npz")["data"]
    assert paths.shape[1] == 8 and np.all(paths[:, 1] % 10 == 0)
    st_a, steps_a, rets_a = prep.simulator.outcomes()
    # the same system built directly from the synthetic arrays
    eng = B200ForceEngine(**s.engine_kwargs())
    mol1, mol2 = s.molecules()
    pathway = s.pathway_set()
    if sm:
        from pystarc_b200 import structures as st

        crit = st.ReactionCriteria("association", [st.ContactPair(0, 0, 2.5)], n_needed=1, state_before="b_surface",
                                   state_after="contact")
        pathway = st.PathwaySet([st.ReactionInterface("association", crit, state_before="b_surface",
                                                      state_after="contact")], first_state="b_surface")
    direct = B200BatchSimulator(mol1, mol2, s.mobility(), pathway,
                                s.params(n_traj=3000, max_steps=1000000, seed=s.seed), eng, termination="complete")
    res_b = direct.run()
    st_b, steps_b, rets_b = direct.outcomes()
    np.testing.assert_array_equal(st_a, st_b)
    np.testing.assert_array_equal(steps_a, steps_b)
    np.testing.assert_array_equal(rets_a, rets_b)
    assert prep.simulator._k_b == direct._k_b and prep.D_rel == direct.mob.relative_translational_diffusion()
    assert res.n_reacted == res_b.n_reacted and res.n_reacted > 0
    if sm:
        assert rec["completed_reactions"][0]["n_fired"] == res.n_reacted


def test_missing_grids_name_the_apbs_step(tmp_path):
    from pystarc_b200 import pipeline

    _work(tmp_path, False)
    (tmp_path / "bd_sims" / "receptor0.dx").unlink()
    with pytest.raises(FileNotFoundError, match="APBS"):
        pipeline.build(tmp_path / "input.xml")
