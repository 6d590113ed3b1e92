"""Host-side logic of the product (no GPU): setup physics, data types, synthetic inputs, DX I/O."""

import math

import numpy as np
import pytest

from pystarc_b200 import hostphys, structures as st, synth
from pystarc_b200.dx import DXGrid
from pystarc_b200.simulator import B200BatchResult, flatten_pairs
from tests.helpers import golden, system


def test_return_prob_matches_reference_runs():
    for name, sysname in [("run_two_sphere", "two_sphere"), ("run_c2", "c2"), ("run_c3", "c3")]:
        g = golden(name)
        s = system(sysname)
        mob = s.mobility()
        D_t = mob.relative_translational_diffusion()
        rp, kb = hostphys.return_prob_and_kb(s.r_start, s.r_escape, float(np.sum(s.rec_q)), float(np.sum(s.lig_q)),
                                             s.debye, D_t, s.hi, s.r_hydro_rec, s.r_hydro_lig)
        assert rp == float(g["return_prob"]) and kb == float(g["k_b"])


def test_bradius_cover_matches_reference():
    """The cover-zone boundary (gpu_batch_simulator.py:406-460), bit for bit on the reference's fixture."""
    g = golden("bradius")
    for (b, q_rec, q_lig, debye), want in zip(g["inputs"], g["cover"]):
        assert hostphys.bradius_cover(float(b), float(q_rec), float(q_lig), float(debye)) == float(want)


def test_mobility_mirror_matches_reference():
    g = golden("stokes")
    for i, r in enumerate(g["radii"]):
        assert st.stokes_translational_diffusion(r) == g["Dt"][i]
        assert st.stokes_rotational_diffusion(r, eta=0.89e-3) == g["Dr_089"][i]
    g = golden("rpy")
    for i, r in enumerate(g["r"]):
        v = np.array([r, 0.3 * r, -0.2 * r]) / math.sqrt(1 + 0.09 + 0.04)
        np.testing.assert_allclose(st.rpy_offdiagonal(v, 17.5, 16.5, 0.0123, 0.0131), g["M"][i], rtol=1e-13,
                                   atol=1e-18)


def test_result_api_matches_reference_wilson():
    g = golden("wilson")
    for (nr, ne), v in zip(g["cases"], g["values"]):
        r = B200BatchResult(int(nr + ne), int(nr), int(ne), 0, {}, 50.0, 100.0, 0.2, 1.0, 1.0)
        lo, hi = r.reaction_probability_ci(0.95)
        assert math.isclose(lo, v[1], rel_tol=1e-12, abs_tol=1e-15) and math.isclose(hi, v[2], rel_tol=1e-12)
        assert math.isclose(r.rate_constant(0.06, 57.449), v[5], rel_tol=1e-14)
        assert math.isclose(r.rate_constant(0.06, 0.0), v[6], rel_tol=1e-14)
        lo, hi = r.rate_constant_ci(0.06, 57.449)
        assert math.isclose(lo, v[7], rel_tol=1e-12, abs_tol=1e-6) and math.isclose(hi, v[8], rel_tol=1e-12)
    assert "k_on" in B200BatchResult(10, 4, 6, 0, {}, 50, 100, 0.2, 1.0, 1.0).summary(0.06, 57.4)


def test_multipole_matches_reference():
    g = golden("multipole")
    Q, dip, quad, fpe = hostphys.multipole(g["pos"], g["q"], 78.5)
    assert math.isclose(Q, float(g["Q"]), rel_tol=1e-13)
    np.testing.assert_allclose(dip, g["dipole"], rtol=1e-13, atol=1e-13)
    np.testing.assert_allclose(quad, g["quad"], rtol=1e-13, atol=1e-12)
    assert fpe == float(g["fpe"])


def test_flatten_pairs_n_needed_rules():
    pairs = [st.ContactPair(1, 2, 4.0), st.ContactPair(3, 4, 5.0)]
    for nn, want in [(-1, 2), (1, 1), (5, 2), (0, 0)]:
        ps = st.PathwaySet([st.ReactionInterface("r", st.ReactionCriteria("r", pairs, n_needed=nn))])
        assert flatten_pairs(ps)[3] == want
    assert flatten_pairs(st.PathwaySet([]))[3] == 1


def test_bridge_deff_matches_oracle_formula():
    s = system("c2")
    mob = s.mobility()
    D_t = mob.relative_translational_diffusion()
    from tests.helpers import step_system
    from oracle.stepper import bridge_D_eff

    ss = step_system(s)
    rec = np.array([s.rec_pos[a] for a, _, _ in s.pairs])
    body = s.lig_pos - s.lig_pos.mean(0)
    lig = np.array([body[b] for _, b, _ in s.pairs])
    np.testing.assert_array_equal(hostphys.bridge_d_eff(D_t, s.r_hydro_rec, s.r_hydro_lig, rec, lig),
                                  bridge_D_eff(ss))


def test_synthetic_configs_have_stated_shapes():
    s = synth.config2(scale=0.3)
    assert len(s.lig_q) == 19 and abs(np.sum(s.lig_q) - 1.0) < 1e-12
    assert s.lig_q[-1] == 0 and np.allclose(s.lig_pos[-1], s.lig_pos[:-1].mean(0), atol=1e-12)
    d = np.linalg.norm(s.rec_pos[:-1, None] - s.rec_pos[None, :-1], axis=2) + np.eye(len(s.rec_pos) - 1) * 99
    assert d.min() >= 1.2
    assert len(s.elec_grids) == 2 and s.elec_grids[0].data.dtype == np.float32
    s1 = synth.config1(grid_dims=33, n_traj=10)
    assert s1.pairs == [(0, 0, 26.0)] and s1.alpha == 0.0


def test_dx_roundtrip(tmp_path):
    g = synth.sphere_dh_grid(2.0, 3.0, (9, 10, 11), 0.7, 7.85, 78.5 * 0.000142)
    p = tmp_path / "g.dx"
    g.write(p)
    h = DXGrid.from_file(p)
    assert h.data.shape == (9, 10, 11)
    np.testing.assert_allclose(h.data, g.data, rtol=1e-8)
    np.testing.assert_allclose(h.origin, g.origin, atol=1e-6)
    bad = tmp_path / "bad.dx"
    bad.write_text(p.read_text().replace("object 3 class array", "object 3 class array") + "")
    txt = p.read_text().splitlines()
    txt = [t if not t[:1].isdigit() and not t[:1] == "-" else t for t in txt]
    (tmp_path / "short.dx").write_text("\n".join(txt[:-3]) + "\n")
    with pytest.raises(ValueError):
        DXGrid.from_file(tmp_path / "short.dx")


def test_dx_reader_matches_reference_fixture(tmp_path):
    # the DX text of the reference's own DXGrid test (tests/test_pystarc.py:971-991)
    txt = ("# APBS generated potential\nobject 1 class gridpositions counts 3 3 3\norigin 0.000 0.000 0.000\n"
           "delta 1.000 0.000 0.000\ndelta 0.000 1.000 0.000\ndelta 0.000 0.000 1.000\n"
           "object 2 class gridconnections counts 3 3 3\n"
           "object 3 class array type double rank 0 items 27 data follows\n"
           "0.0 1.0 2.0 1.0 2.0 3.0 2.0 3.0 4.0\n1.0 2.0 3.0 2.0 3.0 4.0 3.0 4.0 5.0\n"
           "2.0 3.0 4.0 3.0 4.0 5.0 4.0 5.0 6.0\nobject 4 class field\n")
    p = tmp_path / "t.dx"
    p.write_text(txt)
    g = DXGrid.from_file(p)
    assert g.data.shape == (3, 3, 3) and g.data[0, 0, 0] == 0.0 and g.data[2, 2, 2] == 6.0
    assert g.data[1, 0, 2] == 3.0  # z fastest


def test_nan_grid_rejected(tmp_path):
    g = synth.sphere_dh_grid(2.0, 3.0, (8, 8, 8), 0.7, 7.85, 78.5 * 0.000142)
    g.data[3, 3, 3] = np.nan
    g.write(tmp_path / "n.dx")
    with pytest.raises(ValueError):
        DXGrid.from_file(tmp_path / "n.dx")


def test_reference_known_answers_on_the_host_physics():
    """The reference suite's known answers (tests/test_pystarc.py) on this package's host physics:
    Romberg integrals (:4290-4307), CONV (:4322-4325), Wilson bounds at small P (:5318-5330)."""
    for n in range(6):
        assert abs(hostphys.romberg(lambda x, n=n: x ** n, 0.0, 1.0) - 1.0 / (n + 1)) < 1e-8
    assert abs(hostphys.romberg(math.sin, 0.0, math.pi) - 2.0) < 1e-8
    assert abs(hostphys.CONV - 6.022e8) / 6.022e8 < 1e-12
    for nr, ne in ((50, 950), (2, 998), (0, 1000), (1000, 0)):
        r = B200BatchResult(nr + ne, nr, ne, 0, {}, 50.0, 100.0, 0.2, 1.0, 1.0)
        lo, hi = r.reaction_probability_ci()
        assert 0.0 <= lo and hi <= 1.0 + 1e-15  # the bounds the reference tests
        if 0 < nr < nr + ne:
            assert lo < r.reaction_probability < hi
    # k_b of two +-1 e spheres at b = 10 A (:4246-4249) and its k_on(P) table (:4333-4341) without the
    # return-probability correction
    _, kb = hostphys.return_prob_and_kb(10.0, 20.1, 1.0, -1.0, 7.828, 0.43371)
    assert abs(kb - 57.5) < 1.0
    for P, k in ((0.1, 3.46e9), (0.2, 6.93e9), (0.3, 1.04e10), (0.4, 1.39e10), (0.5, 1.73e10)):
        assert abs(hostphys.CONV * 57.5 * P - k) / k < 0.02
