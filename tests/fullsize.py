"""Full-size configurations: force/torque error against the FP64 oracle and FP64 trajectory identity.

Shared by ``tests/test_gpu_fullsize.py`` (which asserts the bounds) and by
``python -m tests.fullsize`` (which prints the measured errors per
configuration as one JSON line; it needs a GPU).

Systems are built at the sizes of the benchmark configurations, with their
grids filled on the GPU:

* ``c1``   two charged spheres (+5/-5 e, 129^3 at 1.0 A, 1e5 trajectories);
* ``c2``   protein + small ligand (3,200/18 atoms, 193^3 + 129^3 elec and Born grids, 65^3 ligand Born grid);
* ``c3``   protein-protein (1,700/1,400 atoms, three 161^3 grids at 0.6 A, HI);
* ``c5_NN`` systems of the heterogeneous batch: 10 has the largest grid (225^3), 7 the largest
  receptor (6,344 atoms), 12 the largest ligand (1,828 atoms).

The reference force is ``GPUBatchForceEngine.__call__`` (pystarc/forces/gpu_batch_engine.py:531-605),
restated by ``oracle.forces.OracleForceEngine``; trajectories follow the reference step loop
(pystarc/simulation/gpu_batch_simulator.py:783-1254) restated by ``oracle.stepper.run`` with the
engine's keyed Philox draws.
"""

from __future__ import annotations

import json
import math

import numpy as np

from oracle import stepper as ost
from oracle.forces import force_error
from tests.helpers import oracle_engine, step_params, step_system

NAMES = ("c1", "c2", "c3", "c5_10", "c5_07", "c5_12")
_SYS = {}


def system(name):
    """Full-size system ``name`` (grids filled on cuda:0), cached per process."""
    from pystarc_b200 import synth

    if name not in _SYS:
        if name == "c1":
            _SYS[name] = synth.config1()
        elif name == "c2":
            _SYS[name] = synth.config2(scale=1.0, device="cuda")
        elif name == "c3":
            _SYS[name] = synth.config3(scale=1.0, device="cuda")
        elif name.startswith("c5_"):
            _SYS[name] = synth.config5(int(name[3:]), device="cuda")
        else:
            raise KeyError(name)
    return _SYS[name]


class _MP:
    def __init__(self, s):
        self.dipole, self.quadrupole, self.four_pi_eps = s.multipole_moments()


def engine(s, precision, torque="centroid"):
    from pystarc_b200.engine import B200ForceEngine

    eng = B200ForceEngine(**s.engine_kwargs(), multipole_expansion=_MP(s) if s.multipole else None,
                          precision=precision, torque_mode=torque)
    eng.set_ligand(s.lig_pos - s.lig_pos.mean(axis=0), s.lig_q)
    return eng


def extents(s):
    """(receptor radius, ligand radius, half-width of the finest elec grid) in A."""
    r_rec = float(np.max(np.linalg.norm(s.rec_pos, axis=1)))
    body = s.lig_pos - s.lig_pos.mean(axis=0)
    r_lig = float(np.max(np.linalg.norm(body, axis=1)))
    g = min(s.elec_grids, key=lambda g: float(np.asarray(g.delta)[0, 0]))
    half = 0.5 * (np.asarray(g.data).shape[0] - 1) * float(np.asarray(g.delta)[0, 0])
    return r_rec, r_lig, half


def force_poses(s, n, seed=11):
    """Poses from inside contact to beyond the finest grid: |c| uniform on
    [0.6 (r_rec + r_lig), half-width + r_lig + 10 A] (two spheres: from the reaction distance),
    directions and orientations uniform."""
    r_rec, r_lig, half = extents(s)
    lo = 0.6 * (r_rec + r_lig) if len(s.rec_pos) > 2 else s.pairs[0][2] * 0.9
    hi = half + r_lig + 10.0
    rng = np.random.default_rng(seed)
    v = rng.standard_normal((n, 3))
    c = v / np.linalg.norm(v, axis=1, keepdims=True) * rng.uniform(lo, hi, (n, 1))
    q = rng.standard_normal((n, 4))
    return c, q / np.linalg.norm(q, axis=1, keepdims=True)


def _stats(x):
    x = np.asarray(x, dtype=float)
    return {"max": float(np.max(x)), "p99": float(np.percentile(x, 99)), "median": float(np.median(x))}


def force_report(name, precision, n=320, seed=11, s=None):
    """Errors of the CUDA engine against the FP64 oracle on ``n`` identical poses.

    ``plain`` is ||F - F_ref|| / ||F_ref|| (torque likewise); ``metric`` is the
    tested metric ``oracle.forces.force_error``, whose denominator is at least
    1e-3 of the summed per-atom force sizes.  Poses whose reference force is
    below 1e-6 of the median are left out of the plain relative error (the
    ratio is not defined there); their count is reported.
    """
    from oracle.stepper import rotmats

    s = s or system(name)
    c, q = force_poses(s, n, seed)
    eng = engine(s, precision)
    F, T, E = eng.eval_poses(c, q)
    eng.close()
    R = rotmats(q)
    body = s.lig_pos - s.lig_pos.mean(axis=0)
    pos = np.einsum("nij,kj->nki", R, body) + c[:, None, :]
    Fo, To, Eo, scale = oracle_engine(s, born_chunk_skip=False)(pos, s.lig_q, R, c, torque_mode="centroid",
                                                                 return_scale=True)
    nf = np.linalg.norm(Fo, axis=1)
    nt = np.linalg.norm(To, axis=1)
    okf = nf > 1e-6 * np.median(nf)
    okt = nt > 1e-6 * max(np.median(nt), 1e-300)
    lever = float(np.max(np.linalg.norm(body, axis=1))) + 1e-12
    out = {
        "config": name, "precision": precision, "poses": int(n),
        "radii_A": [round(float(np.min(np.linalg.norm(c, axis=1))), 2),
                    round(float(np.max(np.linalg.norm(c, axis=1))), 2)],
        "force_plain": _stats(np.linalg.norm(F - Fo, axis=1)[okf] / nf[okf]),
        "force_metric": _stats(force_error(F, Fo, scale)),
        "force_plain_excluded": int((~okf).sum()),
        "energy_plain": _stats(np.abs(E - Eo) / np.maximum(np.abs(Eo), 1e-300)),
    }
    if okt.any():
        out["torque_plain"] = _stats(np.linalg.norm(T - To, axis=1)[okt] / nt[okt])
        out["torque_plain_excluded"] = int((~okt).sum())
    out["torque_metric"] = _stats(force_error(T, To, scale * lever))
    return out


def contact_poses(s, n, seed=5):
    """Start poses near contact with no receptor atom within 1.5 A of the centroid: |c| uniform on
    [r_rec - 2, r_rec + r_lig + 4] A (two spheres: 27-45 A from the centre)."""
    r_rec, r_lig, _ = extents(s)
    lo, hi = (r_rec - 2.0, r_rec + r_lig + 4.0) if len(s.rec_pos) > 2 else (27.0, 45.0)
    rng = np.random.default_rng(seed)
    c = np.zeros((0, 3))
    while c.shape[0] < n:
        v = rng.standard_normal((4 * n, 3))
        cand = v / np.linalg.norm(v, axis=1, keepdims=True) * rng.uniform(lo, hi, (4 * n, 1))
        d = np.min(np.linalg.norm(cand[:, None, :] - np.asarray(s.rec_pos)[None, :, :], axis=2), axis=1)
        c = np.vstack([c, cand[d >= 1.6]])
    q = rng.standard_normal((n, 4))
    return c[:n], q / np.linalg.norm(q, axis=1, keepdims=True)


def identity_run(name, n=32, launches=6, K=16, torque=None, s=None, hi_mode="reference_gpu"):
    """FP64 trajectories from the same start poses, engine vs oracle with the same keyed draws.

    Every trajectory runs ``launches * K`` steps or until it ends.  Returns a dict of
    (gpu, oracle) outcome arrays and the largest pose difference of the trajectories
    still running at the end.
    """
    from pystarc_b200 import _lib
    from pystarc_b200.simulator import B200BatchSimulator

    s = s or system(name)
    torque = torque or ("centroid" if len(s.lig_q) > 100 else "zero")
    c0, q0 = contact_poses(s, n)
    M = launches * K
    eng = engine(s, "fp64", torque)
    mol1, mol2 = s.molecules()
    params = s.params(n_traj=n, max_steps=10 * M)
    sim = B200BatchSimulator(mol1, mol2, s.mobility(), s.pathway_set(), params, eng, slots=n,
                             termination="complete", steps_per_launch=K, hi_mode=hi_mode)
    sim._setup()
    h = eng.handle
    h.call("bd_sim_reset", None)
    cap = _lib.C.c_int32()
    h.call("bd_sim_capacity", _lib.C.byref(cap))
    C = cap.value
    assert C == n, (C, n)
    cc = np.ascontiguousarray(c0.T.reshape(-1))
    qq = np.ascontiguousarray(q0.T.reshape(-1))
    ids = np.arange(n, dtype=np.int32)
    zi = np.zeros(n, dtype=np.int32)
    z8 = np.zeros(n, dtype=np.int8)
    ctr = np.zeros(_lib.N_CTR, dtype=np.uint64)
    ctr[_lib.CTR_NAMES.index("started")] = n
    h.call("bd_sim_restore", _lib.ptr(cc), _lib.ptr(qq), _lib.ptr(ids, _lib.C.c_int32), _lib.ptr(zi, _lib.C.c_int32),
           _lib.ptr(zi, _lib.C.c_int32), _lib.ptr(z8, _lib.C.c_int8), n, _lib.ptr(ctr, _lib.C.c_uint64),
           _lib.ptr(z8, _lib.C.c_int8), _lib.ptr(zi, _lib.C.c_int32), _lib.ptr(zi, _lib.C.c_int32))
    h.call("bd_sim_set_states", _lib.ptr(z8, _lib.C.c_int8))
    h.call("bd_sim_run", launches, K, None)
    st, steps, rets = sim.outcomes()
    c = np.zeros(3 * C)
    q = np.zeros(4 * C)
    traj, sst, srt = (np.zeros(C, dtype=np.int32) for _ in range(3))
    sstat = np.zeros(C, dtype=np.int8)
    live = _lib.C.c_int32()
    h.call("bd_sim_snapshot", _lib.ptr(c), _lib.ptr(q), _lib.ptr(traj, _lib.C.c_int32),
           _lib.ptr(sst, _lib.C.c_int32), _lib.ptr(srt, _lib.C.c_int32), _lib.ptr(sstat, _lib.C.c_int8),
           _lib.C.byref(live), _lib.ptr(ctr, _lib.C.c_uint64))
    eng.close()
    gst = st.astype(np.int32).copy()
    gsteps = steps.astype(np.int64).copy()
    grets = rets.astype(np.int64).copy()
    gpos = np.full((n, 3), np.nan)
    gq = np.full((n, 4), np.nan)
    for k in range(live.value):
        if sstat[k] == 0:  # still running after launches * K steps
            t = traj[k]
            gst[t] = 3
            gsteps[t] = sst[k]
            grets[t] = srt[k]
            gpos[t] = c.reshape(3, C)[:, k]
            gq[t] = q.reshape(4, C)[:, k]
    eo = oracle_engine(s, born_chunk_skip=False)
    fn = (lambda *a, **k: eo(*a, torque_mode="centroid", **k)) if torque == "centroid" else eo
    o = ost.run(step_system(s, fn), step_params(s, n, s.seed, M, hi_mode=hi_mode), noise="philox",
                termination="complete", init=(c0, q0))
    run = gst == 3
    per = np.where(run, np.max(np.abs(np.nan_to_num(gpos) - o.pos), axis=1), 0.0)
    dpos = float(np.max(per)) if run.any() else 0.0
    dq = float(np.max(np.abs(gq[run] - o.q[run]))) if run.any() else 0.0
    return {"gpu": (gst, gsteps, grets), "oracle": (o.status, o.n_steps, o.n_returns), "running": int(run.sum()),
            "max_pose_diff_A": dpos, "max_quat_diff": dq, "steps": int(o.total_steps),
            "overlap_rejections": int(o.n_overlap_rejected), "pose_diff_per_trajectory": per,
            "start": (c0, q0)}


def oracle_sensitivity(name, start, M, torque=None, s=None, hi_mode="reference_gpu", rel=1e-13):
    """Per-trajectory pose change of the oracle run from ``start`` when every force is scaled by
    (1 + rel): how strongly the dynamics amplify a rounding-sized force difference in M steps."""
    s = s or system(name)
    torque = torque or ("centroid" if len(s.lig_q) > 100 else "zero")
    c0, q0 = start
    n = len(c0)
    eo = oracle_engine(s, born_chunk_skip=False)
    out = []
    for eps in (0.0, rel):
        def fn(*a, _e=eps, **k):
            F, T, E = eo(*a, torque_mode="centroid", **k) if torque == "centroid" else eo(*a, **k)
            return F * (1.0 + _e), T, E

        out.append(ost.run(step_system(s, fn), step_params(s, n, s.seed, M, hi_mode=hi_mode), noise="philox",
                           termination="complete", init=(c0, q0)))
    return np.max(np.abs(out[0].pos - out[1].pos), axis=1)


def analytic_p_rxn(s, return_prob):
    """Exact reaction probability of radial diffusion from b with absorption at the reaction
    distance a and, at r_escape = q, a return to b with probability ``return_prob`` (the
    Smoluchowski solution the reference's two-sphere example checks against,
    examples/two_charged_spheres/analytical.py:50-70):

        P_s = int_b^q e^{U(r)} / (r^2 D) dr / int_a^q e^{U(r)} / (r^2 D) dr,
        P_rxn = P_s / (1 - (1 - P_s) return_prob),

    with U the ligand charge times the receptor sphere's Debye-Hueckel potential (the field the
    129^3 grid samples) and D the constant relative diffusion coefficient.
    """
    from scipy.integrate import quad

    q_rec = float(np.sum(s.rec_q))
    q_lig = float(np.sum(s.lig_q))
    a_sph = float(np.max(s.rec_r))
    kappa = 1.0 / s.debye
    eps = s.sdie * 0.000142

    def U(r):
        return q_lig * q_rec * math.exp(kappa * (a_sph - r)) / (4 * math.pi * eps * r * (1 + kappa * a_sph))

    D = s.mobility().relative_translational_diffusion()
    a, b, q = s.pairs[0][2], s.r_start, s.r_escape
    f = lambda r: math.exp(U(r)) / (r * r * D)
    Sbq = quad(f, b, q, limit=500)[0]
    Saq = quad(f, a, q, limit=500)[0]
    Ps = Sbq / Saq
    return Ps / (1.0 - (1.0 - Ps) * return_prob)


def main():
    rows = []
    for name in NAMES:
        for prec in ("fp64", "mixed"):
            rows.append(force_report(name, prec))
            print(json.dumps(rows[-1]), flush=True)
    print(json.dumps({"force_error": rows}))


if __name__ == "__main__":
    main()
