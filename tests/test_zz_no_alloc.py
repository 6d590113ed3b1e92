"""bd_sim_run_noalloc, the stepper entry point that allocates no device memory.

It is for callers that cannot call cudaMalloc when they run trajectories (an
application whose allocator already holds the GPU memory, or a process under a
device-memory quota).  Through the C
ABI it must give every trajectory the same outcome, step count and return count as
the regular stepper, and the same counters, on two calls in a row: the calls share
one static scratch array, so the second call also shows that each call clears what
it uses.  This file is collected last so that a run stopping at the first failure
has already run every other test.
"""

import ctypes as C

import numpy as np
import pytest

from tests.helpers import system

pytestmark = pytest.mark.gpu


def _params(sim, slots):
    from pystarc_b200 import _lib

    p = sim.params
    mob = sim.mob
    sp = _lib.BdSimParams()
    sp.n_traj = int(p.n_trajectories)
    sp.seed = int(p.seed)
    sp.r_start = float(p.r_start)
    sp.r_escape = float(p.r_escape)
    sp.return_prob = float(sim._return_prob)
    sp.max_steps = int(p.max_steps)
    sp.max_dt = float(p.max_dt)
    sp.min_core_dt = float(getattr(p, "minimum_core_dt", 0.0))
    sp.use_hi = int(bool(p.hydrodynamic_interactions))
    sp.overlap = int(bool(p._overlap_check))
    sp.D_t = float(mob.relative_translational_diffusion())
    sp.D_r = float(mob.relative_rotational_diffusion())
    sp.q_rec_total = float(sim.mol1.total_charge())
    sp.q_lig_total = float(sim.mol2.total_charge())
    sp.adt_debye = float(sim.engine._debye)
    sp.r_hydro_rec = float(mob.radius1)
    sp.r_hydro_lig = float(mob.radius2)
    sp.precision = _lib.PREC_MIXED
    sp.torque_mode = _lib.TORQUE_ZERO
    sp.slots = slots
    sp.id_offset = 0
    return sp


def test_noalloc_run_matches_regular_stepper_on_two_calls():
    import torch

    from pystarc_b200 import _lib
    from tests.test_gpu_stepper import make_sim

    s = system("c2")
    N, max_steps, slots = 3000, 300, 2048
    sim = make_sim(s, N, max_steps, "mixed", slots=slots, steps_per_launch=16)
    res = sim.run()
    st_ref, steps_ref, rets_ref = sim.outcomes()
    assert set(np.unique(st_ref)) <= {1, 2, 3}
    sp = _params(sim, slots)
    h = sim.engine.handle
    dev = torch.device("cuda", h.device)
    out_st = torch.empty(N, dtype=torch.int8, device=dev)
    out_steps = torch.empty(N, dtype=torch.int32, device=dev)
    out_rets = torch.empty(N, dtype=torch.int32, device=dev)
    ctr = torch.empty(_lib.N_CTR, dtype=torch.int64, device=dev)
    for call in range(2):
        for t in (out_st, out_steps, out_rets, ctr):
            t.fill_(-7)  # the call must overwrite every entry
        torch.cuda.synchronize()
        h.call("bd_sim_run_noalloc", C.byref(sp), _lib.P(out_st.data_ptr()), _lib.P(out_steps.data_ptr()),
               _lib.P(out_rets.data_ptr()), _lib.P(ctr.data_ptr()), 16, 100_000, None)
        np.testing.assert_array_equal(out_st.cpu().numpy(), st_ref, err_msg=f"call {call}")
        np.testing.assert_array_equal(out_steps.cpu().numpy(), steps_ref, err_msg=f"call {call}")
        np.testing.assert_array_equal(out_rets.cpu().numpy(), rets_ref, err_msg=f"call {call}")
        c = dict(zip(_lib.CTR_NAMES, (int(v) for v in ctr.cpu().numpy())))
        for k in ("started", "reacted", "escaped", "max_steps", "steps", "returns", "overlap", "bridge"):
            assert c[k] == res.counters[k], (call, k, c[k], res.counters[k])


def test_noalloc_rejects_more_slots_than_the_array_holds():
    import torch

    from pystarc_b200 import _lib
    from tests.test_gpu_stepper import make_sim

    s = system("c2")
    sim = make_sim(s, 200, 50, "mixed", steps_per_launch=16)
    sim.run()
    sp = _params(sim, 65537)
    h = sim.engine.handle
    out = torch.empty(1024, dtype=torch.int32, device="cuda")
    with pytest.raises(_lib.BdError, match="at most 65536"):
        h.call("bd_sim_run_noalloc", C.byref(sp), _lib.P(out.data_ptr()), _lib.P(out.data_ptr()),
               _lib.P(out.data_ptr()), _lib.P(out.data_ptr()), 16, 10, None)


def test_noalloc_rejects_a_handle_with_a_surrogate():
    """The entry point runs only the exact-force stepper; a handle carrying a surrogate is refused
    instead of silently ignoring it."""
    import torch

    from pystarc_b200 import _lib
    from pystarc_b200.surrogate import MLPEnsemble, SurrogateSpec
    from tests.test_gpu_stepper import make_sim

    s = system("c2")
    sim = make_sim(s, 200, 50, "mixed", steps_per_launch=16)
    sim.run()
    ens = MLPEnsemble(n_members=2, seed=3)
    spec = SurrogateSpec(r_min=0.0, r_max=1e9, threshold=0.0, force_floor=1.0)
    h = sim.engine.handle
    h.call("bd_sim_set_surrogate", ens.h, C.byref(spec.c_params()))
    sp = _params(sim, 256)
    out = torch.empty(1024, dtype=torch.int32, device="cuda")
    with pytest.raises(_lib.BdError, match="exact-force stepper only"):
        h.call("bd_sim_run_noalloc", C.byref(sp), _lib.P(out.data_ptr()), _lib.P(out.data_ptr()),
               _lib.P(out.data_ptr()), _lib.P(out.data_ptr()), 16, 10, None)
    h.call("bd_sim_set_surrogate", None, None)
    ens.close()
