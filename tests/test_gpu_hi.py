"""Hydrodynamic interactions of the stepper: D(r) in both modes against the oracle, and FP64
trajectories with the Zuk three-regime RPY coupling against the oracle stepper.

Reference: the GPU stepper's line-of-centres D(r) (pystarc/simulation/gpu_batch_simulator.py:741-751,
:1074-1084) and MobilityTensor.relative_translational_diffusion with the Zuk et al. (2014) tensor
(pystarc/hydrodynamics/rotne_prager.py:67-124, :177-200).
"""

import numpy as np
import pytest

from oracle import stepper as ost
from tests.helpers import oracle_engine, step_params, step_system, system

pytestmark = pytest.mark.gpu

# separations covering the three Zuk regimes of the c3 radii (17.5 + 16.5 A): one sphere inside the
# other (r <= 1 A), partial overlap (1 < r <= 34 A), far field
R = np.array([0.3, 0.9, 1.0, 1.2, 3.0, 10.0, 20.0, 30.0, 33.99, 34.0, 34.01, 40.0, 60.0, 80.0, 160.0])


def _sim(s, precision, hi_mode, n_traj=64, max_steps=100, **kw):
    from tests.test_gpu_stepper import make_sim

    kw.setdefault("steps_per_launch", 16)
    kw.setdefault("launches_per_poll", 4)
    return make_sim(s, n_traj, max_steps, precision, "centroid", hi_mode=hi_mode, **kw)


@pytest.mark.parametrize("hi_mode", ["reference_gpu", "zuk"])
@pytest.mark.parametrize("precision,rtol", [("fp64", 1e-13), ("mixed", 2e-5)])
def test_diffusion_of_separation_matches_oracle(hi_mode, precision, rtol):
    from pystarc_b200 import _lib, synth

    s = synth.config3(scale=0.25)
    s.r_hydro_rec, s.r_hydro_lig = 17.5, 16.5  # the full-size radii: all three regimes within 0-160 A
    sim = _sim(s, precision, hi_mode)
    sim._setup()
    D = np.zeros_like(R)
    sim.engine.handle.call("bd_sim_hi_diffusion", len(R), _lib.ptr(np.ascontiguousarray(R)), _lib.ptr(D))
    ss = step_system(s)
    prm = step_params(s, 1, 1, 1, hi_mode=hi_mode)
    Do = ost.hi_diffusion(R, ss, prm)
    np.testing.assert_allclose(D, Do, rtol=rtol)
    assert len(np.unique(np.round(D, 12))) > 5  # D(r) varies
    sim.engine.close()


def test_fp64_trajectories_with_zuk_hi_match_oracle_exactly():
    """Protein-protein shape (scaled), HI in the Zuk mode: same fates, step and return counts."""
    s = system("c3")
    n, max_steps = 32, 80
    sim = _sim(s, "fp64", "zuk", n_traj=n, max_steps=max_steps)
    res = sim.run()
    st, steps, rets = sim.outcomes()
    eng = oracle_engine(s, born_chunk_skip=False)
    fn = lambda *a, **k: eng(*a, torque_mode="centroid", **k)
    o = ost.run(step_system(s, fn), step_params(s, n, s.seed, max_steps, hi_mode="zuk"), noise="philox",
                termination="complete")
    np.testing.assert_array_equal(st, o.status)
    np.testing.assert_array_equal(steps, o.n_steps)
    np.testing.assert_array_equal(rets, o.n_returns)
    assert res.total_steps == o.total_steps

