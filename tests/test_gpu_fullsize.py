"""The benchmark configurations at their stated sizes, against the FP64 oracle.

* Forces, torques and energies on 320 identical poses per configuration, from inside contact
  to beyond the finest grid, in FP64 and in mixed precision (reference:
  ``GPUBatchForceEngine.__call__``, pystarc/forces/gpu_batch_engine.py:531-605).
* FP64 trajectories from contact poses, 96 steps each, against the oracle stepper with the
  same keyed draws: identical fates, step and return counts, and poses that agree to
  rounding (pystarc/simulation/gpu_batch_simulator.py:783-1254).
* Two charged spheres (config 1) as specified, 1e5 trajectories: the reaction probability's
  Wilson 95 % interval holds the exact Smoluchowski value.
"""

import numpy as np
import pytest

from tests import fullsize as fs

pytestmark = pytest.mark.gpu

# Bounds on oracle.forces.force_error (per pose: ||F - F_ref|| over max(||F_ref||, 1e-3 sum_i ||F_ref,i||))
FP64_TOL = 1e-9
MIXED_TOL = 1e-4
# Plain relative force error ||F - F_ref|| / ||F_ref||, 99th percentile over the poses
FP64_PLAIN_P99 = 1e-9
MIXED_PLAIN_P99 = 1e-4


@pytest.mark.parametrize("name", fs.NAMES)
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_force_error_at_full_size(name, precision):
    r = fs.force_report(name, precision)
    print(r)
    tol = FP64_TOL if precision == "fp64" else MIXED_TOL
    assert r["force_metric"]["max"] < tol, r
    assert r["torque_metric"]["max"] < tol, r
    assert r["force_plain"]["p99"] < (FP64_PLAIN_P99 if precision == "fp64" else MIXED_PLAIN_P99), r
    assert r["energy_plain"]["p99"] < (1e-9 if precision == "fp64" else 1e-3), r


@pytest.mark.parametrize("name,hi_mode", [(n, "reference_gpu") for n in fs.NAMES] + [("c3", "zuk")])
def test_fp64_trajectories_at_full_size(name, hi_mode):
    """Same fates, step and return counts as the oracle; final poses within 1e-8 A, except for
    trajectories whose dynamics amplify rounding: those the oracle itself moves by more than
    1e-6 A when its forces change by 1 part in 1e13 (the large-ligand c5 system near contact)."""
    r = fs.identity_run(name, hi_mode=hi_mode)
    g, o = r["gpu"], r["oracle"]
    np.testing.assert_array_equal(g[0], o[0])
    np.testing.assert_array_equal(g[1], o[1])
    np.testing.assert_array_equal(g[2], o[2])
    far = r["pose_diff_per_trajectory"] > 1e-8
    if far.any():
        sens = fs.oracle_sensitivity(name, r["start"], 96, hi_mode=hi_mode)
        print(f"{name}: {int(far.sum())} of {len(far)} poses differ by > 1e-8 A; oracle sensitivity there "
              f"{np.round(sens[far], 6)}")
        assert np.all(sens[far] > 1e-6), (r["pose_diff_per_trajectory"][far], sens[far])
        assert (~far).sum() >= len(far) // 2
    else:
        assert r["max_quat_diff"] < 1e-9, r


def _two_sphere_run(max_dt):
    from pystarc_b200.engine import B200ForceEngine
    from pystarc_b200.simulator import B200BatchSimulator

    s = fs.system("c1")
    eng = B200ForceEngine(**s.engine_kwargs(), precision="fp64")
    mol1, mol2 = s.molecules()
    params = s.params()
    params.max_dt = max_dt
    sim = B200BatchSimulator(mol1, mol2, s.mobility(), s.pathway_set(), params, eng, termination="complete")
    res = sim.run()
    eng.close()
    assert res.n_trajectories == 100_000 and res.n_max_steps == 0
    return res, fs.analytic_p_rxn(s, sim._return_prob)


def test_two_spheres_reaction_probability_is_the_exact_solution():
    """Config 1 (+5/-5 e, 1e5 trajectories) against the exact Smoluchowski P_rxn.

    As specified (no max_dt) the reference's adaptive dt takes 0.005 r^2 / D, about 55 ps and
    4.5 A per step at the 26 A reaction surface, where the potential is -11.5 kT: that
    discretisation lowers P_rxn by about 1.5 % of its value.  With max_dt = 2 ps the steps are
    5x to 25x shorter there and the exact value lies inside the Wilson 95 % interval.
    """
    res, exact = _two_sphere_run(0.0)
    p = res.reaction_probability
    print(f"as specified: P_rxn {p:.5f} {res.reaction_probability_ci()}, exact {exact:.5f}")
    assert abs(p - exact) < 0.02 * exact
    res, exact = _two_sphere_run(2.0)
    lo, hi = res.reaction_probability_ci()
    print(f"max_dt 2 ps: P_rxn {res.reaction_probability:.5f} [{lo:.5f}, {hi:.5f}], exact {exact:.5f}")
    assert lo <= exact <= hi
