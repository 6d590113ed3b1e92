"""CUDA force kernels against the reference's outputs and the FP64 oracle on identical poses."""

import numpy as np
import pytest

from oracle.forces import force_error
from oracle.stepper import rotmats
from tests.helpers import golden, oracle_engine, system, system_digest

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-9   # error metric of oracle.forces.force_error, FP64 engine
MIXED_TOL = 1e-4  # FP32 force arithmetic, FP64 geometry and sums (the bound required of mixed precision)


class _MP:
    def __init__(self, s):
        self.dipole, self.quadrupole, self.four_pi_eps = s.multipole_moments()


def make_engine(s, precision="fp64", torque="zero", layout=None, use_lj=False):
    from pystarc_b200.engine import B200ForceEngine

    lj = dict(rec_radii=s.rec_r, lig_radii=s.lig_r, use_lj=True) if use_lj else {}
    eng = B200ForceEngine(**s.engine_kwargs(), multipole_expansion=_MP(s) if s.multipole else None,
                          precision=precision, torque_mode=torque, layout=layout, **lj)
    eng.set_ligand(s.lig_pos - s.lig_pos.mean(axis=0), s.lig_q)
    return eng


def random_poses(n, rmin, rmax, seed):
    rng = np.random.default_rng(seed)
    v = rng.standard_normal((n, 3))
    c = v / np.linalg.norm(v, axis=1, keepdims=True) * rng.uniform(rmin, rmax, (n, 1))
    q = rng.standard_normal((n, 4))
    return c, q / np.linalg.norm(q, axis=1, keepdims=True)


@pytest.mark.parametrize("name,sysname", [("engine_c2", "c2"), ("engine_c3", "c3")])
@pytest.mark.parametrize("path", ["atoms", "poses"])
def test_fp64_matches_reference_outputs(name, sysname, path):
    g = golden(name)
    s = system(sysname)
    assert system_digest(s) == str(g["digest"])
    eng = make_engine(s)
    if path == "atoms":
        F, T, E = eng(g["positions"], s.lig_q, g["R"], g["centroids"])
    else:
        F, T, E = eng.eval_poses(g["centroids"], g["quats"])
    _, _, _, scale = oracle_engine(s)(g["positions"], s.lig_q, g["R"], g["centroids"], return_scale=True)
    err = force_error(F, g["F"], scale)
    assert err.max() < FP64_TOL, err.max()
    np.testing.assert_allclose(E, g["E"], rtol=1e-9, atol=1e-12 * np.abs(g["E"]).max())
    assert np.all(T == 0)
    eng.close()


@pytest.mark.parametrize("sysname", ["c2", "c3", "two_sphere"])
@pytest.mark.parametrize("precision,tol", [("fp64", FP64_TOL), ("mixed", MIXED_TOL)])
def test_random_poses_against_oracle(sysname, precision, tol):
    s = system(sysname)
    eng = make_engine(s, precision, "centroid")
    rmax = {"c2": 30.0, "c3": 40.0, "two_sphere": 22.0}[sysname]
    c, q = random_poses(3000, 0.5, rmax, 17)
    F, T, E = eng.eval_poses(c, q)
    R = rotmats(q)
    body = s.lig_pos - s.lig_pos.mean(axis=0)
    pos = np.einsum("nij,kj->nki", R, body) + c[:, None, :]
    o = oracle_engine(s, born_chunk_skip=False)
    Fo, To, Eo, scale = o(pos, s.lig_q, R, c, torque_mode="centroid", return_scale=True)
    err = force_error(F, Fo, scale)
    assert err.max() < tol, (err.max(), np.percentile(err, 99))
    lever = np.max(np.linalg.norm(body, axis=1)) + 1e-12
    terr = force_error(T, To, scale * lever)
    assert terr.max() < tol, terr.max()
    escale = np.maximum(np.abs(Eo), 1e-3 * np.abs(Eo).max() + 1e-300)
    assert np.max(np.abs(E - Eo) / escale) < max(tol, 1e-9) * 10
    eng.close()


@pytest.mark.parametrize("sysname", ["c2", "c3"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_grid_windows_give_identical_forces(sysname, precision):
    """Window copies, cube copies (vector loads) and plain scalar loads feed the same values to the same
    arithmetic."""
    from pystarc_b200 import _lib

    s = system(sysname)
    c, q = random_poses(2000, 0.5, 35.0, 5)
    out = []
    for layout in (0, _lib.LAYOUT_WINDOWS_1, _lib.LAYOUT_WINDOWS_2, _lib.LAYOUT_DEFAULT, _lib.LAYOUT_CUBES_1,
                   _lib.LAYOUT_CUBES_1 | _lib.LAYOUT_WINDOWS_1, _lib.LAYOUT_DEFAULT & ~_lib.LAYOUT_XY_1,
                   _lib.LAYOUT_DEFAULT & ~_lib.LAYOUT_ZTEX_1, _lib.LAYOUT_DEFAULT | _lib.LAYOUT_XYTEX_1,
                   _lib.LAYOUT_DEFAULT | _lib.LAYOUT_PTEX_2):
        eng = make_engine(s, precision, "centroid", layout=layout)
        out.append(eng.eval_poses(c, q))
        eng.close()
    for other in out[1:]:
        for x, y in zip(out[0], other):
            np.testing.assert_array_equal(x, y)


@pytest.mark.parametrize("group", [1, 4, 8, 16, 32, 64, 65])
def test_launch_shape_does_not_change_results(group):
    s = system("c2")
    eng = make_engine(s, "fp64", "centroid")
    c, q = random_poses(500, 1.0, 25.0, 5)
    F0, T0, E0 = eng.eval_poses(c, q)
    eng.handle.call("bd_set_launch", group, 64)
    F1, T1, E1 = eng.eval_poses(c, q)
    np.testing.assert_allclose(F1, F0, rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(T1, T0, rtol=1e-12, atol=1e-15)
    eng.close()


def test_no_yukawa_uses_every_grid_finest_first():
    """With zero receptor charge the reference keeps all elec grids and has no far-field (:186-193, :356-366)."""
    import copy

    s = copy.copy(system("c2"))
    charged = np.abs(s.rec_q) > 0
    s.rec_q = s.rec_q - s.rec_q.sum() / charged.sum() * charged
    assert abs(s.rec_q.sum()) < 1e-9
    eng = make_engine(s, "fp64")
    assert len(eng._elec_grids_gpu) == 2 and not eng._has_yukawa
    c, q = random_poses(800, 5.0, 75.0, 9)
    F, T, E = eng.eval_poses(c, q)
    R = rotmats(q)
    body = s.lig_pos - s.lig_pos.mean(axis=0)
    pos = np.einsum("nij,kj->nki", R, body) + c[:, None, :]
    o = oracle_engine(s, born_chunk_skip=False)
    assert len(o.elec) == 2
    Fo, _, Eo, scale = o(pos, s.lig_q, R, c, return_scale=True)
    assert force_error(F, Fo, scale).max() < FP64_TOL
    eng.close()


def test_empty_batch_and_bad_arguments():
    from pystarc_b200 import _lib

    s = system("two_sphere")
    eng = make_engine(s)
    F, T, E = eng.eval_poses(np.zeros((0, 3)), np.zeros((0, 4)))
    assert F.shape == (0, 3)
    with pytest.raises(_lib.BdError):
        eng.handle.call("bd_eval_forces", 1, None, None, 0, None, None, None, 0, 0, None)
    with pytest.raises(_lib.BdError):
        eng.handle.call("bd_set_launch", 3, 64)
    bad = np.array([[np.nan, 0, 0]])
    with pytest.raises(_lib.BdError):
        eng.set_ligand(bad, np.array([1.0]))
    eng.close()


def test_reference_chunk_skip_quirk_only_when_batch_is_far():
    """The reference zeroes Born direction 2 for a whole batch whose closest centroid is beyond the
    receptor radius plus the ligand grid's x half-width (gpu_batch_engine.py:635-639); the engine culls
    per atom exactly.  On batches with any near pose the two agree."""
    s = system("c2")
    g = golden("engine_c2")
    o_skip = oracle_engine(s, born_chunk_skip=True)
    o_exact = oracle_engine(s, born_chunk_skip=False)
    a = o_skip(g["positions"], s.lig_q, g["R"], g["centroids"])[0]
    b = o_exact(g["positions"], s.lig_q, g["R"], g["centroids"])[0]
    np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("sysname", ["c2", "c3"])
def test_force_terms_add_up(sysname):
    """bd_set_terms: grid + far-field + reverse Born evaluated apart sum to the full force."""
    from pystarc_b200 import _lib

    s = system(sysname)
    eng = make_engine(s, "fp64", "centroid")
    c, q = random_poses(1500, 0.5, 60.0, 23)
    F, T, E = eng.eval_poses(c, q)
    parts = [eng.eval_poses(c, q, terms=t) for t in (_lib.TERM_GRID, _lib.TERM_FARFIELD, _lib.TERM_REV_BORN)]
    Fs = sum(p[0] for p in parts)
    Ts = sum(p[1] for p in parts)
    np.testing.assert_allclose(Fs, F, rtol=1e-9, atol=1e-12 * np.abs(F).max())
    np.testing.assert_allclose(Ts, T, rtol=1e-9, atol=1e-12 * np.abs(T).max())
    # the mask is restored after each call
    F2, _, _ = eng.eval_poses(c, q)
    np.testing.assert_array_equal(F2, F)
    eng.close()


# ---- WCA contact forces (use_lj=True) ---------------------------------------------------------

@pytest.mark.parametrize("name,sysname", [("engine_wca_c2", "c2"), ("engine_wca_c3", "c3")])
@pytest.mark.parametrize("path", ["atoms", "poses"])
@pytest.mark.parametrize("precision,tol", [("fp64", FP64_TOL), ("mixed", MIXED_TOL)])
def test_contact_forces_match_reference_outputs(name, sysname, path, precision, tol):
    from oracle.forces import wca_forces
    from pystarc_b200 import _lib

    g = golden(name)
    s = system(sysname)
    assert system_digest(s) == str(g["digest"])
    eng = make_engine(s, precision, use_lj=True)
    assert eng._lj_activation == float(g["activation"]) and eng._lj_epsilon == float(g["epsilon"])
    if path == "atoms":
        F, T, E = eng(g["positions"], s.lig_q, g["R"], g["centroids"])
    else:
        F, T, E = eng.eval_poses(g["centroids"], g["quats"])
    _, _, _, scale = oracle_engine(s, use_lj=True)(g["positions"], s.lig_q, g["R"], g["centroids"],
                                                    return_scale=True)
    err = force_error(F, g["F"], scale)
    assert err.max() < tol, err.max()
    assert np.all(T == 0)
    # the contact term alone, against the reference's _wca_forces_gpu
    Fw, _, Ew = eng.eval_poses(g["centroids"], g["quats"], terms=_lib.TERM_CONTACT)
    fa, _ = wca_forces(g["positions"], g["centroids"], s.rec_pos, s.rec_r, s.lig_r)
    werr = force_error(Fw, g["F_wca"], np.linalg.norm(fa, axis=2).sum(axis=1))
    assert werr.max() < FP64_TOL, werr.max()
    inactive = np.linalg.norm(g["centroids"], axis=1) >= eng._lj_activation
    assert np.all(Fw[inactive] == 0) and np.all(Ew == 0)
    eng.close()


@pytest.mark.parametrize("sysname", ["c2", "c3"])
@pytest.mark.parametrize("precision,tol", [("fp64", FP64_TOL), ("mixed", MIXED_TOL)])
@pytest.mark.parametrize("group", [None, 1, 8])
def test_contact_random_poses_against_oracle(sysname, precision, tol, group):
    """Poses from deep overlap to beyond the activation radius, with the torque about the centroid."""
    s = system(sysname)
    eng = make_engine(s, precision, "centroid", use_lj=True)
    if group is not None:
        eng.handle.call("bd_set_launch", group, 64)
    c, q = random_poses(600, 0.5, 1.3 * eng._lj_activation, 29)
    F, T, E = eng.eval_poses(c, q)
    R = rotmats(q)
    body = s.lig_pos - s.lig_pos.mean(axis=0)
    pos = np.einsum("nij,kj->nki", R, body) + c[:, None, :]
    o = oracle_engine(s, born_chunk_skip=False, use_lj=True)
    Fo, To, Eo, scale = o(pos, s.lig_q, R, c, torque_mode="centroid", return_scale=True)
    err = force_error(F, Fo, scale)
    assert err.max() < tol, (err.max(), np.percentile(err, 99))
    lever = np.max(np.linalg.norm(body, axis=1)) + 1e-12
    terr = force_error(T, To, scale * lever)
    assert terr.max() < tol, terr.max()
    eng.close()


def test_contact_term_adds_up_and_is_off_without_radii():
    from pystarc_b200 import _lib

    s = system("c2")
    eng = make_engine(s, "fp64", "centroid", use_lj=True)
    c, q = random_poses(800, 0.5, 14.0, 31)
    F, T, E = eng.eval_poses(c, q)
    parts = [eng.eval_poses(c, q, terms=t)
             for t in (_lib.TERM_GRID, _lib.TERM_FARFIELD, _lib.TERM_REV_BORN, _lib.TERM_CONTACT)]
    np.testing.assert_allclose(sum(p[0] for p in parts), F, rtol=1e-9, atol=1e-12 * np.abs(F).max())
    np.testing.assert_allclose(sum(p[1] for p in parts), T, rtol=1e-9, atol=1e-12 * np.abs(T).max())
    assert np.any(parts[3][0] != 0)
    plain = make_engine(s, "fp64", "centroid")
    F0, T0, E0 = plain.eval_poses(c, q)
    np.testing.assert_allclose(F0, F - parts[3][0], rtol=1e-9, atol=1e-12 * np.abs(F).max())
    np.testing.assert_array_equal(E0, E)
    # use_lj without radii evaluates no contact term (gpu_batch_engine.py:233-236)
    from pystarc_b200.engine import B200ForceEngine

    e2 = B200ForceEngine(**s.engine_kwargs(), multipole_expansion=_MP(s), torque_mode="centroid", use_lj=True)
    e2.set_ligand(s.lig_pos - s.lig_pos.mean(axis=0), s.lig_q)
    np.testing.assert_array_equal(e2.eval_poses(c, q)[0], F0)
    for e in (eng, plain, e2):
        e.close()
