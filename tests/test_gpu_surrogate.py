"""Stepper with the learned surrogate: plumbing against the exact stepper, training, k_on."""

import numpy as np
import pytest

from tests.helpers import system

pytestmark = pytest.mark.gpu


class _MP:
    def __init__(self, s):
        self.dipole, self.quadrupole, self.four_pi_eps = s.multipole_moments()


def make_sim(s, n_traj, max_steps, precision="fp64", seed=None, surrogate=None, **kw):
    from pystarc_b200.engine import B200ForceEngine
    from pystarc_b200.simulator import B200BatchSimulator

    eng = B200ForceEngine(**s.engine_kwargs(), multipole_expansion=_MP(s) if s.multipole else None,
                          precision=precision)
    mol1, mol2 = s.molecules()
    kw.setdefault("termination", "complete")
    return B200BatchSimulator(mol1, mol2, s.mobility(), s.pathway_set(),
                              s.params(n_traj=n_traj, max_steps=max_steps, seed=seed), eng, surrogate=surrogate, **kw)


def _spec(**kw):
    from pystarc_b200.surrogate import SurrogateSpec

    return SurrogateSpec(**kw)


def _ens(members=2, seed=3):
    from pystarc_b200.surrogate import MLPEnsemble

    return MLPEnsemble(n_members=members, seed=seed)


@pytest.mark.parametrize("terms", [6, 7])
def test_forced_fallback_reproduces_the_exact_stepper(terms):
    """threshold 0: every trusted pose falls back to the exact terms the surrogate replaces (far-field
    + reverse Born, or those and the grid terms: the total force)."""
    s = system("c2")
    ens = _ens()
    spec = _spec(r_min=0.0, r_max=1e9, threshold=0.0, force_floor=1.0, terms=terms)
    a = make_sim(s, 400, 300, "fp64", steps_per_launch=8, surrogate=(ens, spec))
    ra = a.run()
    b = make_sim(s, 400, 300, "fp64", steps_per_launch=8)
    rb = b.run()
    sa, na, _ = a.outcomes()
    sb, nb, _ = b.outcomes()
    same = (sa == sb) & (na == nb)
    assert same.mean() >= 0.98, same.mean()
    c = ra.counters
    assert c["surrogate_evals"] > 0 and c["surrogate_fallbacks"] == c["surrogate_evals"]
    assert c["steps"] == int(na.sum())
    assert abs(ra.n_reacted - rb.n_reacted) <= 8
    ens.close()


def test_untrusted_region_never_calls_the_surrogate():
    s = system("c2")
    ens = _ens()
    spec = _spec(r_min=1e8, r_max=1e9, threshold=1e9)
    sim = make_sim(s, 300, 200, "mixed", steps_per_launch=8, surrogate=(ens, spec))
    res = sim.run()
    assert res.counters["surrogate_evals"] == 0
    ref = make_sim(s, 300, 200, "mixed", steps_per_launch=8)
    ref.run()
    np.testing.assert_array_equal(sim.outcomes()[0], ref.outcomes()[0])
    ens.close()


def test_trained_surrogate_gains_over_omitting_it_and_keeps_k_on():
    from pystarc_b200 import surrogate as sg

    s = system("c2")
    ens = sg.MLPEnsemble(n_members=3, seed=11)
    spec = sg.SurrogateSpec()
    spec.r_min = sg.contact_distance(s.rec_pos, s.lig_pos) + 8.0
    spec.r_max = 80.0
    sampler = make_sim(s, 20000, 100000, "mixed", steps_per_launch=16)
    c, q = sg.sample_poses(sampler, 60000, r_lo=spec.r_min - 2.0, r_hi=80.0)
    eng = sampler.engine
    lig = s.lig_pos - s.lig_pos.mean(axis=0)
    eng.set_ligand(lig, s.lig_q)
    T = sg.exact_targets(eng, c, q)
    n_tr = 50000
    rep = sg.fit(ens, spec, c[:n_tr], q[:n_tr], T[:n_tr], steps=4000, batch=4096, lr=1e-3)
    err = sg.heldout_error(ens, spec, c[n_tr:], q[n_tr:], T[n_tr:])
    # what the trained network gains: its error against leaving the two terms out
    assert err["median"] < 0.2 * err["without_surrogate_median"], err
    sim = make_sim(s, 20000, 100000, "mixed", seed=77, steps_per_launch=16, surrogate=(ens, spec),
                   termination="reference")
    res = sim.run()
    ref = make_sim(s, 20000, 100000, "mixed", seed=77, steps_per_launch=16, termination="reference")
    rr = ref.run()
    lo, hi = res.reaction_probability_ci()
    rlo, rhi = rr.reaction_probability_ci()
    assert lo <= rhi and rlo <= hi, ((lo, hi), (rlo, rhi), err, rep.final_loss)
    assert res.counters["surrogate_evals"] > 0
    ens.close()
