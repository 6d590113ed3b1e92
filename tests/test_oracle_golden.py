"""The oracle against golden vectors produced by the unmodified reference (CPU only)."""

import math

import numpy as np
import pytest

from oracle import physics as oph
from oracle import stepper as ost
from oracle.forces import k1_batch_force, _interp, multipole_moments, yukawa_forces, FarField
from oracle.philox import philox4x32_10, KeyedDraws
from tests.helpers import golden, system, system_digest, oracle_engine, step_system, step_params


def test_k1_matches_reference_dxgrid():
    g = golden("k1")
    data = g["data"].astype(np.float64)
    pts = g["points"]
    inv = 1.0 / g["sp"]
    phi = _interp(data, g["origin"], inv, pts[:, 0], pts[:, 1], pts[:, 2])
    np.testing.assert_allclose(phi, g["phi"], rtol=0, atol=1e-13)
    # F = -q grad phi with q = -1 gives grad phi
    f, e = k1_batch_force(pts, -np.ones(len(pts)), data, g["origin"], g["sp"], 0.0, False)
    np.testing.assert_allclose(f, g["grad"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(e, -g["phi"], rtol=0, atol=1e-13)


def test_k1_zero_charge_and_born_coefficients():
    g = golden("k1")
    data = g["data"].astype(np.float64)
    pts = g["points"][:10]
    f0, e0 = k1_batch_force(pts, np.full(10, 5e-10), data, g["origin"], g["sp"], 0.3, True)
    assert np.all(f0 == 0) and np.all(e0 == 0)
    fb, eb = k1_batch_force(pts, np.full(10, 0.5), data, g["origin"], g["sp"], 0.3, True)
    fe, ee = k1_batch_force(pts, np.full(10, 1.0), data, g["origin"], g["sp"], 0.0, False)
    np.testing.assert_allclose(fb, 0.3 * 0.25 * fe, rtol=1e-14)
    np.testing.assert_allclose(eb, 0.3 * 0.25 * ee, rtol=1e-14)


@pytest.mark.parametrize("name,sysname", [("engine_c2", "c2"), ("engine_c3", "c3")])
def test_engine_matches_reference(name, sysname):
    g = golden(name)
    s = system(sysname)
    assert system_digest(s) == str(g["digest"]), "synthetic system drifted from the golden fixture"
    eng = oracle_engine(s)
    assert len(eng.elec) == int(g["n_elec"]) and len(eng.born) == int(g["n_born"])
    assert len(eng.lig_born) == int(g["n_lig_born"])
    F, T, E = eng(g["positions"], s.lig_q, R_matrices=g["R"], centroids=g["centroids"])
    scale = np.abs(g["F"]).max()
    np.testing.assert_allclose(F, g["F"], rtol=1e-11, atol=1e-13 * scale)
    np.testing.assert_allclose(E, g["E"], rtol=1e-11, atol=1e-12 * np.abs(g["E"]).max())
    assert np.all(T == 0) and np.all(g["T"] == 0)
    assert np.isclose(eng.ff.V_factor, float(g["V_factor"]), rtol=1e-15)


@pytest.mark.parametrize("name,sysname", [("engine_wca_c2", "c2"), ("engine_wca_c3", "c3")])
def test_contact_forces_match_reference(name, sysname):
    """WCA contact forces (use_lj=True): the totals and the contact term alone, at centroids on both
    sides of the activation radius."""
    from oracle.forces import WCA_EPSILON, wca_activation, wca_forces

    g = golden(name)
    s = system(sysname)
    assert system_digest(s) == str(g["digest"])
    assert wca_activation(s.rec_r, s.lig_r) == float(g["activation"]) and WCA_EPSILON == float(g["epsilon"])
    fa, fw = wca_forces(g["positions"], g["centroids"], s.rec_pos, s.rec_r, s.lig_r)
    scale = np.linalg.norm(fa, axis=2).sum(axis=1)
    np.testing.assert_allclose(fw, g["F_wca"], rtol=1e-12, atol=1e-14 * scale.max())
    inactive = np.linalg.norm(g["centroids"], axis=1) >= float(g["activation"])
    assert inactive.any() and (~inactive).any()
    assert np.all(g["F_wca"][inactive] == 0) and np.all(fw[inactive] == 0)
    eng = oracle_engine(s, use_lj=True)
    F, T, E = eng(g["positions"], s.lig_q, R_matrices=g["R"], centroids=g["centroids"])
    np.testing.assert_allclose(F, g["F"], rtol=1e-11, atol=1e-13 * np.abs(g["F"]).max())
    np.testing.assert_allclose(E, g["E"], rtol=1e-11, atol=1e-12 * np.abs(g["E"]).max())
    assert np.all(T == 0) and np.all(g["T"] == 0)


def test_contact_force_cutoff_and_sign():
    """One receptor and one ligand atom on the x axis: repulsive below 1.122462 sigma, zero from it on."""
    from oracle.forces import wca_forces

    sig = 3.0
    for x, nonzero in ((2.5, True), (3.0, True), (3.3673, True), (3.3674, False), (4.0, False)):
        pos = np.array([[[x, 0.0, 0.0]]])
        fa, fw = wca_forces(pos, np.zeros((1, 3)), np.zeros((1, 3)), [1.0], [2.0], activation=10.0)
        assert (fw[0, 0] > 0) == nonzero and fw[0, 1] == 0 and fw[0, 2] == 0, (x, fw)
    # beyond the activation radius nothing is evaluated
    fa, fw = wca_forces(np.array([[[2.5, 0, 0]]]), np.array([[10.0, 0, 0]]), np.zeros((1, 3)), [1.0], [2.0],
                        activation=10.0)
    assert np.all(fw == 0)


def test_torque_centroid_is_consistent():
    s = system("c2")
    g = golden("engine_c2")
    eng = oracle_engine(s)
    F, T, E = eng(g["positions"], s.lig_q, g["R"], g["centroids"], torque_mode="centroid")
    # a rigid translation of every atom by a about the same centre leaves the torque unchanged
    assert np.all(np.isfinite(T)) and np.any(T != 0)
    F2, T2, _ = eng(g["positions"], s.lig_q, g["R"], g["centroids"], torque_mode="zero")
    np.testing.assert_array_equal(F, F2)
    assert np.all(T2 == 0)


def test_physics_constants():
    g = golden("stokes")
    for i, r in enumerate(g["radii"]):
        assert math.isclose(oph.stokes_translational(r), g["Dt"][i], rel_tol=1e-15)
        assert math.isclose(oph.stokes_rotational(r), g["Dr"][i], rel_tol=1e-15)
        assert math.isclose(oph.stokes_translational(r, eta=0.89e-3), g["Dt_089"][i], rel_tol=1e-15)
        assert math.isclose(oph.stokes_rotational(r, eta=0.89e-3), g["Dr_089"][i], rel_tol=1e-15)
    g = golden("rpy")
    for i, r in enumerate(g["r"]):
        v = np.array([r, 0.3 * r, -0.2 * r]) / math.sqrt(1 + 0.09 + 0.04)
        np.testing.assert_allclose(oph.rpy_offdiagonal(v, 17.5, 16.5, 0.0123, 0.0131), g["M"][i], rtol=1e-13,
                                   atol=1e-18)


def test_zuk_relative_diffusion_is_the_rpy_trace_form():
    """The oracle stepper's Zuk D(r) equals D_t1 + D_t2 - (2/3) tr M12(r) of the RPY tensor pinned
    above (MobilityTensor.relative_translational_diffusion, rotne_prager.py:177-200) in all three
    regimes: far field (r > a + b), partial overlap (|a - b| < r <= a + b), one sphere inside the
    other (r <= |a - b|)."""
    a, b = 17.5, 16.5
    Da, Db = oph.stokes_translational(a, eta=0.89e-3), oph.stokes_translational(b, eta=0.89e-3)
    kT_eta = math.sqrt(Da * 6 * math.pi * a * Db * 6 * math.pi * b)
    rs = np.array([0.2, 0.7, 1.0, 1.5, 5.0, 20.0, 33.9, 34.0, 34.1, 40.0, 80.0, 200.0])
    D = ost.zuk_diffusion(rs, a, b, kT_eta, Da + Db)
    for r, d in zip(rs, D):
        v = np.array([r, 0.3 * r, -0.2 * r]) / math.sqrt(1 + 0.09 + 0.04)
        ref = max(Da + Db - (2.0 / 3.0) * np.trace(oph.rpy_offdiagonal(v, a, b, Da, Db)), 1e-12)
        assert math.isclose(d, ref, rel_tol=1e-13), (r, d, ref)
    assert np.all(np.diff(D[rs > 34.0]) > 0)  # the coupling fades with distance
    assert ost.zuk_diffusion(np.array([0.0]), a, b, kT_eta, Da + Db)[0] == Da + Db


def test_quaternion_conventions():
    g = golden("quat")
    np.testing.assert_array_equal(ost.rotmats(g["q"]), g["R"])
    np.testing.assert_array_equal(ost.apply_rotation(g["q"], g["omega"]), g["q_new"])
    np.testing.assert_array_equal(ost.shoemake(g["shoemake_u"]), g["shoemake"])


def test_wilson_and_rate_constant():
    g = golden("wilson")
    for (nr, ne), v in zip(g["cases"], g["values"]):
        n = nr + ne
        P = nr / n if n else 0.0
        assert P == v[0]
        lo, hi = oph.wilson_ci(int(nr), int(ne), 0.95)
        assert math.isclose(lo, v[1], rel_tol=1e-12, abs_tol=1e-15) and math.isclose(hi, v[2], rel_tol=1e-12)
        lo, hi = oph.wilson_ci(int(nr), int(ne), 0.90)
        assert math.isclose(lo, v[3], rel_tol=1e-12, abs_tol=1e-15) and math.isclose(hi, v[4], rel_tol=1e-12)
        assert math.isclose(oph.rate_constant(P, 0.06, 57.449, 50.0, 100.0), v[5], rel_tol=1e-14)
        assert math.isclose(oph.rate_constant(P, 0.06, 0.0, 50.0, 100.0), v[6], rel_tol=1e-14)


def test_multipole_moments_and_farfield_potential():
    g = golden("multipole")
    dip, quad = multipole_moments(g["pos"], g["q"])
    np.testing.assert_allclose(dip, g["dipole"], rtol=1e-13, atol=1e-13)
    np.testing.assert_allclose(quad, g["quad"], rtol=1e-13, atol=1e-12)
    ff = FarField(float(g["Q"]), 7.85, 78.5, dip, quad, float(g["fpe"]))
    _, e = yukawa_forces(g["pts"], np.ones(len(g["pts"])), ff)
    # the reference potential() uses r itself; the far-field uses max(r, 1): same for these points
    np.testing.assert_allclose(e, g["V"], rtol=1e-12)


def test_reference_known_answers():
    """Known-answer values from the reference's own test suite (tests/test_pystarc.py)."""
    eps = 78.0 * 0.000142
    V = 1.0 * -1.0 / (4 * math.pi * eps)
    assert abs(V - (-7.1847)) < 0.01  # :4027-4029
    assert abs(V * math.exp(-10.0 / 7.828) / 10.0 - (-0.200268)) < 0.001  # :4031-4034
    D = 1.0 / (6 * math.pi * 0.243 * 1.0)
    assert abs(D - 0.21803) < 0.001  # :3988-3990
    rp, kb = oph.return_prob_and_kb(10.0, 20.1, 1.0, -1.0, 7.828, 0.43371)
    assert abs(kb - 57.5) < 1.0 and abs(rp - 0.52) < 0.03  # :4246-4263
    assert abs(oph.CONV - 6.022e8) / 6.022e8 < 1e-3  # :4322-4325
    assert abs(math.sqrt(2 * 0.43371 * 0.2) - 0.4169) < 0.001  # :4147-4151
    lo, hi = oph.wilson_ci(50, 950)
    assert 0 <= lo < 0.05 < hi <= 1


def test_reference_known_answers_grid_and_farfield():
    """The reference suite's known answers for trilinear grids and the multipole far-field
    (tests/test_pystarc.py:935-960, :4505-4566), applied to the oracle's K1 and far-field."""
    data = np.zeros((5, 5, 5))
    for i in range(5):
        data[i] = float(i)  # potential rises along x
    o, sp = np.zeros(3), np.ones(3)
    pts = np.array([[2.0, 2.0, 2.0], [1.5, 1.0, 1.0], [100.0, 0.0, 0.0]])
    f, e = k1_batch_force(pts, np.ones(3), data, o, sp, 0.0, False)  # q = 1: E = phi, F = -grad phi
    assert abs(e[0] - 2.0) < 1e-12 and abs(e[1] - 1.5) < 1e-12 and e[2] == 0.0  # :941-954
    assert abs(-f[0, 0] - 1.0) < 1e-12 and abs(f[0, 1]) < 1e-12 and abs(f[0, 2]) < 1e-12  # :956-960
    assert np.all(f[2] == 0.0)
    # monopole of +3 e at the origin, lambda = 7.86, eps = 78 * 0.000142 (:4511-4520)
    ff = FarField(3.0, 7.86, 78.0)
    r = 20.0
    V_exact = 3.0 / (4 * math.pi * 78.0 * 0.000142 * r) * math.exp(-r / 7.86)
    _, V = yukawa_forces(np.array([[r, 0.0, 0.0]]), np.ones(1), ff)
    assert abs(V[0] - V_exact) / abs(V_exact) < 1e-12
    # F = -grad V by central differences (:4552-4566)
    rv = np.array([15.0, 3.0, -2.0])
    F, _ = yukawa_forces(rv[None], np.ones(1), ff)
    h = 1e-4
    for i in range(3):
        d = np.zeros(3)
        d[i] = h
        _, vp = yukawa_forces((rv + d)[None], np.ones(1), ff)
        _, vm = yukawa_forces((rv - d)[None], np.ones(1), ff)
        F_num = -(vp[0] - vm[0]) / (2 * h)
        assert abs(F[0, i] - F_num) < 1e-6 * max(abs(F_num), 1e-10)
    # two opposite charges: no monopole, dipole magnitude 10 (:4522-4531)
    dip, quad = multipole_moments(np.array([[5.0, 0, 0], [-5.0, 0, 0]]), np.array([1.0, -1.0]))
    assert abs(np.linalg.norm(dip) - 10.0) < 1e-12


def test_philox_known_answers():
    """Random123 known-answer vectors for philox4x32-10."""
    out = philox4x32_10(0, 0, 0, 0, 0, 0)
    assert [int(x) for x in out] == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    out = philox4x32_10(0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF)
    assert [int(x) for x in out] == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    out = philox4x32_10(0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344, 0xA4093822, 0x299F31D0)
    assert [int(x) for x in out] == [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


def test_keyed_draw_statistics():
    d = KeyedDraws(99)
    ids = np.arange(200000)
    xi_t, xi_r = d.step_normals(np.full(ids.shape, 3), ids)
    for x in (xi_t, xi_r):
        assert abs(x.mean()) < 0.01 and abs(x.std() - 1) < 0.01
    u = d.u_escape(np.zeros_like(ids), ids)
    assert 0 <= u.min() and u.max() < 1 and abs(u.mean() - 0.5) < 0.005


@pytest.mark.parametrize("name,sysname", [("run_two_sphere", "two_sphere"), ("run_c2", "c2"), ("run_c3", "c3")])
def test_stepper_reproduces_reference_run_exactly(name, sysname):
    g = golden(name)
    s = system(sysname)
    assert system_digest(s) == str(g["digest"])
    ss = step_system(s)
    assert math.isclose(ss.D_t, float(g["D_t"]), rel_tol=1e-15)
    assert math.isclose(ss.D_r, float(g["D_r"]), rel_tol=1e-15)
    res = ost.run(ss, step_params(s, int(g["n_traj"]), int(g["seed"]), int(g["max_steps"])), noise="pcg64")
    assert res.return_prob == float(g["return_prob"]) and res.k_b == float(g["k_b"])
    assert (res.n_reacted, res.n_escaped, res.n_max_steps) == (int(g["n_reacted"]), int(g["n_escaped"]),
                                                              int(g["n_max_steps"]))
    assert abs(res.total_steps - int(g["total_steps"])) <= 1  # reference reports steps/s x elapsed
    np.testing.assert_array_equal(res.n_steps, g["n_steps"])
    np.testing.assert_array_equal(res.n_returns, g["n_returns"])
    ref_outcome = g["outcome"].copy()
    ref_outcome[ref_outcome == 0] = 3
    np.testing.assert_array_equal(res.status, ref_outcome)


def test_stepper_with_contact_forces_reproduces_reference_run_exactly():
    """use_lj=True in the stepper: the reference run with WCA contact forces, trajectory for trajectory."""
    g = golden("run_lj_c2")
    s = system("c2")
    assert system_digest(s) == str(g["digest"])
    res = ost.run(step_system(s, oracle_engine(s, use_lj=True)),
                  step_params(s, int(g["n_traj"]), int(g["seed"]), int(g["max_steps"])), noise="pcg64")
    assert (res.n_reacted, res.n_escaped, res.n_max_steps) == (int(g["n_reacted"]), int(g["n_escaped"]),
                                                              int(g["n_max_steps"]))
    np.testing.assert_array_equal(res.n_steps, g["n_steps"])
    np.testing.assert_array_equal(res.n_returns, g["n_returns"])
    ref_outcome = g["outcome"].copy()
    ref_outcome[ref_outcome == 0] = 3
    np.testing.assert_array_equal(res.status, ref_outcome)
    # the same seed without the contact term takes other paths
    plain = golden("run_c2")
    assert np.any(plain["n_steps"] != g["n_steps"])


@pytest.mark.parametrize("name,sysname", [("run_sm_two_sphere", "two_sphere"), ("run_sm_c2", "c2")])
def test_state_machine_run_reproduces_reference_exactly(name, sysname):
    """State-machine reactions: state numbering, every trajectory's fate and step count, and the
    per-reaction fire counts of the discrete test and the Brownian bridge."""
    from dataclasses import replace

    from oracle.stepper import sm_tables
    from tests.helpers import sm_spec, sm_step_system

    g = golden(name)
    s = system(sysname)
    assert system_digest(s) == str(g["digest"])
    _, sb, sa, _, first = sm_spec(g)
    before, after, terminal = sm_tables(sb, sa, first)
    np.testing.assert_array_equal(before, g["state_index_before"])
    np.testing.assert_array_equal(after, g["state_index_after"])
    np.testing.assert_array_equal(terminal, g["state_terminal"])
    ss = sm_step_system(s, g)
    prm = replace(step_params(s, int(g["n_traj"]), int(g["seed"]), int(g["max_steps"])),
                  min_core_rxn_dt=float(g["min_core_rxn_dt"]))
    res = ost.run(ss, prm, noise="pcg64")
    assert res.return_prob == float(g["return_prob"]) and res.k_b == float(g["k_b"])
    assert (res.n_reacted, res.n_escaped, res.n_max_steps) == (int(g["n_reacted"]), int(g["n_escaped"]),
                                                              int(g["n_max_steps"]))
    np.testing.assert_array_equal(res.n_steps, g["n_steps"])
    np.testing.assert_array_equal(res.n_returns, g["n_returns"])
    ref_outcome = g["outcome"].copy()
    ref_outcome[ref_outcome == 0] = 3
    np.testing.assert_array_equal(res.status, ref_outcome)
    np.testing.assert_array_equal(res.sm_fires_discrete, g["fires_discrete"])
    np.testing.assert_array_equal(res.sm_fires_bridge, g["fires_bridge"])
    np.testing.assert_array_equal(res.sm_fires_discrete + res.sm_fires_bridge, g["n_fired"])


def test_state_machine_tables_of_the_drop_in():
    """pystarc_b200.simulator.state_machine numbers states as the reference does, labels unset included."""
    from oracle.stepper import sm_tables
    from pystarc_b200.simulator import state_machine
    from tests.helpers import sm_pathway, sm_spec

    for name in ("run_sm_two_sphere", "run_sm_c2"):
        g = golden(name)
        sm = state_machine(sm_pathway(g))
        np.testing.assert_array_equal(sm["before"], g["state_index_before"])
        np.testing.assert_array_equal(sm["after"], g["state_index_after"])
        np.testing.assert_array_equal(sm["terminal"], g["state_terminal"])
        assert sm["names"] == sm_spec(g)[0]
    # a destination without a label is -1; the first state defaults to the first reaction's source
    b, a, t = sm_tables(["x", "y"], ["y", None])
    assert list(b) == [0, 1] and list(a) == [1, -1] and list(t) == [False, False]


@pytest.mark.parametrize("name,sysname", [("run_two_sphere", "two_sphere"), ("run_c2", "c2"), ("run_c3", "c3")])
def test_stepper_statistics_match_reference(name, sysname):
    """The per-step statistics the reference collects for its output files (gpu_batch_simulator.py:1255-1317)."""
    g = golden(name)
    s = system(sysname)
    res = ost.run(step_system(s), step_params(s, int(g["n_traj"]), int(g["seed"]), int(g["max_steps"])), noise="pcg64")
    st = res.stats
    np.testing.assert_array_equal(st.start_pos, g["sd_start_pos"])
    np.testing.assert_array_equal(st.start_q, g["sd_start_q"])
    np.testing.assert_array_equal(st.min_dist, g["sd_min_dist"])
    np.testing.assert_array_equal(st.step_at_min, g["sd_step_at_min"])
    np.testing.assert_allclose(st.total_time, g["sd_total_time_ps"], rtol=1e-12)
    np.testing.assert_array_equal(st.bridge, g["sd_bb_triggered"])
    for k, mine in [("radial_counts", st.rad_counts), ("angular_counts", st.ang_counts),
                    ("milestone_flux_out", st.ms_out), ("milestone_flux_in", st.ms_in), ("trans_matrix", st.trans)]:
        np.testing.assert_array_equal(mine, g[f"sd_{k}"], err_msg=k)
    P = len(s.pairs)
    np.testing.assert_array_equal(st.contact[:P], g["sd_contact_pair_counts"][:P])
    assert st.contact_total == int(g["sd_contact_total_steps"])
    et = g["sd_encounter_traj"]
    np.testing.assert_array_equal(st.enc_step[et], g["sd_encounter_step"])
    np.testing.assert_array_equal(st.enc_pos[et], g["sd_encounter_pos"])
    np.testing.assert_array_equal(st.enc_q[et], g["sd_encounter_q"])
    nt = g["sd_near_miss_traj"]
    np.testing.assert_array_equal(st.nm_pos[nt], g["sd_near_miss_pos"])
    np.testing.assert_array_equal(st.min_dist[nt], g["sd_near_miss_dist"])


@pytest.mark.parametrize("name,sysname", [("run_c2", "c2"), ("run_c3", "c3")])
def test_stepper_path_and_energy_traces_match_reference(name, sysname):
    """Path rows [traj, step, x, y, z, q0, q1, q2] and energy rows [traj, step, fx, fy, fz, dt] recorded
    every save_interval (10) steps, as the reference run recorded them (gpu_batch_simulator.py:1319-1340)."""
    g = golden(name)
    s = system(sysname)
    res = ost.run(step_system(s), step_params(s, int(g["n_traj"]), int(g["seed"]), int(g["max_steps"])), noise="pcg64")
    for key, mine in (("path_steps", res.stats.path_steps), ("energy_steps", res.stats.energy_steps)):
        ref = g[f"sd_{key}"]
        rows = np.vstack(mine)
        rows = rows[rows[:, 1] <= ref[:, 1].max()]
        assert rows.shape == ref.shape, (key, rows.shape, ref.shape)
        np.testing.assert_array_equal(rows[:, :2], ref[:, :2])
        np.testing.assert_allclose(rows[:, 2:], ref[:, 2:], rtol=1e-13, atol=1e-13, err_msg=key)
