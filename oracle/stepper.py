"""FP64 NumPy restatement of the reference's batched BD step loop (test infrastructure).

Follows ``GPUBatchSimulator.run`` (pystarc/simulation/gpu_batch_simulator.py:462-1594)
in its flattened-pairs and state-machine modes, one vectorised operation per reference operation and
in the same order, so that with ``noise="pcg64"`` it consumes NumPy's PCG64
stream exactly as the reference does and reproduces its tallies bit for bit:

  start poses                       :509-513, :1597-1609
  discrete reaction test            :818-878, :1690-1751
  escape / return at r_esc          :879-911
  forces                            :929-943  (the force engine is a callable)
  old pair distances                :950-960
  adaptive dt                       :961-1067 (state-machine refinement :1005-1060)
  HI D(r)                           :741-751, :1074-1084
  translation, rotation             :1085-1101, :1631-1660
  overlap rejection                 :1102-1128
  Brownian bridge                   :637-671, :1142-1252 (state machine :1170-1234)
  state-machine tables              :216-319, :523-545
  counters, termination             :1253-1254, :1341-1356, :1485-1489

With ``noise="philox"`` every draw is keyed by (trajectory, its own step index)
through ``oracle.philox.KeyedDraws`` -- the CUDA engine's layout -- and each
trajectory is stepped independently of the others, so its fate and step count
do not depend on the batch.  That mode is the deterministic checker of the GPU
stepper.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .physics import return_prob_and_kb
from .philox import KeyedDraws

EPS0 = 0.000142


@dataclass
class StepSystem:
    lig_body: np.ndarray  # (A,3) ligand atoms about the ligand centroid
    lig_q: np.ndarray  # (A,)
    rec_pos: np.ndarray  # (Nr,3) receptor atoms (receptor at the origin)
    engine: object  # callable(lig_positions, lig_q, R, c) -> (F, T, E)
    rxn_rec_pos: np.ndarray  # (P,3)
    rxn_lig_idx: np.ndarray  # (P,)
    rxn_cutoff: np.ndarray  # (P,)
    n_needed: int
    D_t: float  # relative translational diffusion
    D_r: float  # relative rotational diffusion
    r_h_rec: float
    r_h_lig: float
    q_rec_total: float
    q_lig_total: float
    debye: float  # engine._debye
    # state-machine reactions (None: flattened pairs): per reaction pair its source and
    # destination state index, and per state whether no reaction leaves it (sm_tables)
    sm_before: np.ndarray | None = None
    sm_after: np.ndarray | None = None
    sm_terminal: np.ndarray | None = None
    # kBT/eta of the RPY coupling, sqrt(D_t1 6 pi a1 D_t2 6 pi a2) (rotne_prager.py:121-122); hi_mode "zuk"
    hi_kT_eta: float | None = None


@dataclass
class StepParams:
    n_traj: int
    seed: int
    r_b: float
    r_esc: float
    max_steps: int
    max_dt: float = 0.0
    min_core_dt: float = 0.0
    use_hi: bool = False
    overlap: bool = True
    kT_scale: float = 1.0
    return_prob: float | None = None
    k_b: float | None = None
    min_core_rxn_dt: float = 0.0  # params.minimum_core_reaction_dt (:636)
    # with use_hi: "reference_gpu" (the reference stepper's D(r), :741-751) or "zuk"
    # (MobilityTensor.relative_translational_diffusion, rotne_prager.py:177-200)
    hi_mode: str = "reference_gpu"
    save_interval: int = 10  # path / energy rows every save_interval steps (:579-581)


@dataclass
class StepResult:
    status: np.ndarray
    n_steps: np.ndarray
    n_reacted: int
    n_escaped: int
    n_max_steps: int
    total_steps: int
    loop_steps: int
    return_prob: float
    k_b: float
    n_returns: np.ndarray = field(default=None)
    n_overlap_rejected: int = 0
    stats: "StepStats" = None
    state: np.ndarray = field(default=None)  # state-machine state of every trajectory at the end
    sm_fires_discrete: np.ndarray = field(default=None)  # per reaction
    sm_fires_bridge: np.ndarray = field(default=None)
    pos: np.ndarray = field(default=None)  # (N, 3) centroids at the end (the pose where each trajectory stopped)
    q: np.ndarray = field(default=None)  # (N, 4) quaternions at the end


def sm_tables(state_before, state_after, first_state=None):
    """State indices of the state-machine reactions (gpu_batch_simulator.py:262-299).

    The first state (``first_state``, else the first reaction's source) gets index
    0; every other label gets the next index the first time it is met, in the order
    source, destination of each reaction; an unlabelled state is -1.  A state is
    terminal when no reaction has it as its source.  Returns (before, after, terminal).
    """
    index = {}

    def idx(label):
        if label is None:
            return -1
        if label not in index:
            index[label] = len(index)
        return index[label]

    fs = first_state if first_state is not None else (state_before[0] if state_before else None)
    if fs is not None:
        idx(fs)
    before, after = [], []
    for b, a in zip(state_before, state_after):
        before.append(idx(b))
        after.append(idx(a))
    sources = set(before)
    terminal = np.array([k not in sources for k in range(len(index))], dtype=bool)
    return np.array(before, dtype=np.int64), np.array(after, dtype=np.int64), terminal


def n_needed_of(n_needed_raw, n_pairs):
    """-1 (or too many) means all pairs (gpu_batch_simulator.py:200-205)."""
    return n_pairs if (n_needed_raw < 0 or n_needed_raw > n_pairs) else n_needed_raw


def rotmats(q):
    """(N,4) (w,x,y,z) -> (N,3,3), gpu_batch_simulator.py:1611-1629."""
    w, x, y, z = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    N = q.shape[0]
    return np.stack([
        1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y),
        2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x),
        2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y),
    ], axis=1).reshape(N, 3, 3)


def apply_rotation(q, omega):
    """q <- normalize(q (x) dq(omega)), gpu_batch_simulator.py:1631-1660."""
    angle = np.linalg.norm(omega, axis=1, keepdims=True)
    safe = angle > 1e-10
    axis = np.where(safe, omega / np.where(safe, angle, 1.0), 0.0)
    half = angle * 0.5
    dq = np.stack([np.cos(half[:, 0]), axis[:, 0] * np.sin(half[:, 0]), axis[:, 1] * np.sin(half[:, 0]),
                   axis[:, 2] * np.sin(half[:, 0])], axis=1)
    w1, x1, y1, z1 = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    w2, x2, y2, z2 = dq[:, 0], dq[:, 1], dq[:, 2], dq[:, 3]
    qnew = np.stack([
        w1 * w2 - x1 * x2 - y1 * y2 - z1 * z2,
        w1 * x2 + x1 * w2 + y1 * z2 - z1 * y2,
        w1 * y2 - x1 * z2 + y1 * w2 + z1 * x2,
        w1 * z2 + x1 * y2 - y1 * x2 + z1 * w2,
    ], axis=1)
    qnew /= np.linalg.norm(qnew, axis=1, keepdims=True)
    return qnew


def shoemake(u):
    """Uniform random quaternion from three uniforms (gpu_batch_simulator.py:1597-1609)."""
    return np.stack([
        np.sqrt(1 - u[:, 0]) * np.sin(2 * np.pi * u[:, 1]),
        np.sqrt(1 - u[:, 0]) * np.cos(2 * np.pi * u[:, 1]),
        np.sqrt(u[:, 0]) * np.sin(2 * np.pi * u[:, 2]),
        np.sqrt(u[:, 0]) * np.cos(2 * np.pi * u[:, 2]),
    ], axis=1)


def bridge_D_eff(sys: StepSystem):
    """Per-pair D_eff = D_t + D_rot,rec L_rec^2 + D_rot,lig L_lig^2 (gpu_batch_simulator.py:643-660)."""
    if len(sys.rxn_cutoff) == 0:
        return None
    D_t = sys.D_t
    r_h_rec, r_h_lig = sys.r_h_rec, sys.r_h_lig
    a_sum = r_h_rec + r_h_lig if (r_h_rec + r_h_lig) > 0 else 1.0
    D_trans_rec = D_t * r_h_lig / a_sum
    D_trans_lig = D_t * r_h_rec / a_sum
    D_rot_rec = D_trans_rec * 3.0 / (4.0 * r_h_rec ** 2) if r_h_rec > 0 else 0.0
    D_rot_lig = D_trans_lig * 3.0 / (4.0 * r_h_lig ** 2) if r_h_lig > 0 else 0.0
    L_rec = np.linalg.norm(sys.rxn_rec_pos, axis=1)
    L_lig = np.linalg.norm(sys.lig_body[sys.rxn_lig_idx], axis=1)
    return D_t + D_rot_rec * L_rec ** 2 + D_rot_lig * L_lig ** 2


def hi_constants(r_h_rec, r_h_lig):
    """mu = 0.243 hard-coded (gpu_batch_simulator.py:741-751)."""
    Df = 1.0 / 0.243
    pi6, pi8 = 6.0 * math.pi, 8.0 * math.pi
    a0, a1 = float(r_h_rec), float(r_h_lig)
    a2 = 0.5 * (a0 ** 2 + a1 ** 2)
    ainv = (Df / (pi6 * a0) + Df / (pi6 * a1)) / Df
    return Df, pi8, a2, ainv


def adaptive_dt(r_sr, sys: StepSystem, prm: StepParams, rxn_coord=None):
    """Per-trajectory dt (gpu_batch_simulator.py:961-1067).  ``rxn_coord`` (state-machine mode):
    per trajectory, the distance above the nearest reaction surface reachable from its state."""
    D_t = sys.D_t
    r_b, r_esc = prm.r_b, prm.r_esc
    adt_debye = float(sys.debye)
    adt_eps = 78.0 * EPS0
    V0 = float(sys.q_rec_total) * float(sys.q_lig_total) / (4.0 * math.pi * adt_eps)
    in_outer = r_sr > (1.1 * r_b)
    frac = 0.1
    dt_pair = (frac * frac / 2.0) * r_sr * r_sr / D_t
    if abs(V0) > 1e-9:
        expf = np.exp(-r_sr / adt_debye)
        Fr0 = V0 * expf * (1.0 / r_sr ** 2 + 1.0 / (r_sr * adt_debye))
        Fr1 = -V0 * expf / adt_debye ** 2 - 2.0 * Fr0 / r_sr
        DFr1 = np.abs(D_t * Fr1)
        with np.errstate(divide="ignore"):
            dt_force = np.where((DFr1 > 1e-15) & (r_sr < 3.0 * adt_debye), 0.01 / DFr1, dt_pair)
    else:
        dt_force = dt_pair
    dist_b = np.maximum(r_sr - r_b, np.full_like(r_sr, 1e-3))
    dist_esc = np.maximum(r_esc - r_sr, np.full_like(r_sr, 1e-3))
    dt_edge = np.minimum(dist_b, dist_esc) ** 2 / (18.0 * D_t)
    dt_outer = np.minimum(np.minimum(dt_force, dt_edge), dt_pair)
    dt_inner = np.minimum(dt_force, dt_pair)
    dt_arr = np.where(in_outer, dt_outer, dt_inner)
    if rxn_coord is not None:
        # reaction-surface refinement: 12 sigma must stay below the reaction coordinate (:1034-1060)
        sigma_now = np.sqrt(2.0 * D_t * dt_arr)
        needs = 12.0 * sigma_now > rxn_coord
        crit = rxn_coord * rxn_coord / (288.0 * D_t)
        floored = np.maximum(crit, prm.min_core_rxn_dt) if prm.min_core_rxn_dt > 0 else crit
        dt_arr = np.where(needs, np.minimum(dt_arr, floored), dt_arr)
    if prm.max_dt > 0:
        dt_arr = np.minimum(dt_arr, np.full_like(dt_arr, prm.max_dt))
    if prm.min_core_dt > 0:
        dt_arr = np.maximum(dt_arr, np.full_like(dt_arr, prm.min_core_dt))
    return dt_arr


def zuk_diffusion(r, a, b, kT_eta, D0):
    """D0 - (2/3) tr M12(r) with the three-regime RPY tensor of rotne_prager.py:67-124 (whose
    trace is kBT/eta (3 tt_I + tt_uu)), clamped at 1e-12 (:177-200); vectorised over r."""
    r = np.asarray(r, dtype=np.float64)
    PI = math.pi
    r2 = r * r
    r3 = r2 * r
    s2 = a * a + b * b
    with np.errstate(divide="ignore", invalid="ignore"):
        far_I = (1.0 + s2 / (3.0 * r2)) / (8.0 * PI * r)
        far_uu = (1.0 - s2 / r2) / (8.0 * PI * r)
        am2 = (a - b) ** 2
        den = 6.0 * 32.0 * PI * a * b * r3
        mid_I = (16.0 * r3 * (a + b) - (am2 + 3.0 * r2) ** 2) / den
        mid_uu = 3.0 * (am2 - r2) ** 2 / den
    in_I = 1.0 / (6.0 * PI * max(a, b))
    tI = np.where(r > a + b, far_I, np.where(r > abs(a - b), mid_I, in_I))
    tuu = np.where(r > a + b, far_uu, np.where(r > abs(a - b), mid_uu, 0.0))
    tr = np.where(r < 1e-10, 0.0, kT_eta * (3.0 * tI + tuu))
    return np.maximum(D0 - (2.0 / 3.0) * tr, 1e-12)


def hi_diffusion(r_sr, sys: StepSystem, prm: StepParams):
    if prm.use_hi and prm.hi_mode == "zuk":
        return zuk_diffusion(r_sr, float(sys.r_h_rec), float(sys.r_h_lig), float(sys.hi_kT_eta), sys.D_t)
    if prm.use_hi:
        Df, pi8, a2, ainv = hi_constants(sys.r_h_rec, sys.r_h_lig)
        rm1 = 1.0 / np.maximum(r_sr, np.full_like(r_sr, 0.01))
        rm3 = rm1 ** 3
        Di = -2.0 * Df * (2.0 * rm1 - (4.0 / 3.0) * a2 * rm3) / pi8
        D = Df * ainv + Di
        return np.maximum(D, np.full_like(D, 1e-6))
    return np.full(r_sr.shape[0], sys.D_t, dtype=np.float64)


class StepStats:
    """Per-step statistics of the reference stepper (gpu_batch_simulator.py:577-620, :1255-1317).

    Steps are indexed by each trajectory's own step count, which equals the
    reference's loop counter when nothing refills.  Encounter records are kept
    per trajectory (the reference appends them in event order).
    """

    def __init__(self, pos, q, N, r_b, r_esc, n_pairs):
        self.start_pos = pos.copy()
        self.start_q = q.copy()
        self.min_dist = np.full(N, 1e30)
        self.step_at_min = np.zeros(N, dtype=np.int64)
        self.total_time = np.zeros(N)
        self.nm_pos = pos.copy()
        self.nm_q = q.copy()
        self.bridge = np.zeros(N, dtype=np.int64)
        self.enc_pos = np.zeros((N, 3))
        self.enc_q = np.zeros((N, 4))
        self.enc_step = np.zeros(N, dtype=np.int64)
        self.prev_r = np.linalg.norm(pos, axis=1)
        self.rad_bins = np.linspace(0, float(r_esc * 1.2), 201)
        self.rad_counts = np.zeros(200, dtype=np.int64)
        self.ang_counts = np.zeros((36, 72), dtype=np.int64)
        self.ms_radii = np.linspace(float(r_b), float(r_esc), 11)
        self.ms_out = np.zeros(11, dtype=np.int64)
        self.ms_in = np.zeros(11, dtype=np.int64)
        self.contact = np.zeros(max(n_pairs, 1), dtype=np.int64)
        self.contact_total = 0
        self.trans_bins = np.linspace(0, float(r_esc * 1.2), 51)
        self.trans = np.zeros((50, 50), dtype=np.int64)
        self.path_steps = []  # (n, 8) per recorded step: traj, step, x, y, z, q0, q1, q2
        self.energy_steps = []  # (n, 6) per recorded step: traj, step, fx, fy, fz, dt

    def trace(self, sr_idx, pos, q, steps, forces, dt_arr, save_interval):
        """Path and energy rows of the trajectories that stepped at a step index that is a multiple of
        save_interval (gpu_batch_simulator.py:1319-1340): pose after the step, force and dt of it."""
        on = steps[sr_idx] % save_interval == 0
        if not np.any(on):
            return
        i = sr_idx[on]
        st = steps[i].astype(np.float64)
        self.path_steps.append(np.column_stack([i.astype(np.float64), st, pos[i], q[i][:, :3]]))
        self.energy_steps.append(np.column_stack([i.astype(np.float64), st, forces[on], dt_arr[on]]))

    def encounter(self, idx, pos, q, steps, bridge):
        self.enc_pos[idx] = pos[idx]
        self.enc_q[idx] = q[idx]
        self.enc_step[idx] = steps[idx]
        if bridge:
            self.bridge[idx] = 1

    def step(self, sr_idx, pos, q, steps, dt_arr, pair_d_at_force, cutoffs):
        cur = np.linalg.norm(pos[sr_idx], axis=1)
        better = cur < self.min_dist[sr_idx]
        ti = sr_idx[better]
        self.min_dist[ti] = cur[better]
        self.step_at_min[ti] = steps[ti]
        self.nm_pos[ti] = pos[ti]
        self.nm_q[ti] = q[ti]
        self.total_time[sr_idx] += dt_arr
        np.add.at(self.rad_counts, np.clip(np.searchsorted(self.rad_bins, cur) - 1, 0, 199), 1)
        cen = pos[sr_idx]
        r_safe = np.maximum(cur, 1e-30)
        theta = np.arccos(np.clip(cen[:, 2] / r_safe, -1, 1))
        phi = np.arctan2(cen[:, 1], cen[:, 0]) + np.pi
        t_i = np.clip((theta / np.pi * 36).astype(int), 0, 35)
        p_i = np.clip((phi / (2 * np.pi) * 72).astype(int), 0, 71)
        np.add.at(self.ang_counts, (t_i, p_i), 1)
        prev = self.prev_r[sr_idx]
        for mi, mr in enumerate(self.ms_radii):
            self.ms_out[mi] += int(((prev < mr) & (cur >= mr)).sum())
            self.ms_in[mi] += int(((prev >= mr) & (cur < mr)).sum())
        ob = np.clip(np.searchsorted(self.trans_bins, prev) - 1, 0, 49)
        nb = np.clip(np.searchsorted(self.trans_bins, cur) - 1, 0, 49)
        np.add.at(self.trans, (ob, nb), 1)
        if pair_d_at_force is not None and len(cutoffs) and len(sr_idx):
            self.contact[: len(cutoffs)] += (pair_d_at_force < cutoffs[None, :]).sum(axis=0)
            self.contact_total += len(sr_idx)
        self.prev_r[sr_idx] = cur


def _overlap_inside(new_pos, rec_pos, threshold=1.5):
    N = new_pos.shape[0]
    chunk = max(1, int(500 * 1024 * 1024 / (rec_pos.shape[0] * 3 * 8)))
    chunk = min(chunk, N)
    inside = np.zeros(N, dtype=bool)
    for c0 in range(0, N, chunk):
        c1 = min(c0 + chunk, N)
        d = np.linalg.norm(new_pos[c0:c1, None, :] - rec_pos[None, :, :], axis=2)
        inside[c0:c1] = d.min(axis=1) < threshold
    return inside


def _forces(sys, R_sr, cen_sr, force_batch=None):
    N_sr = R_sr.shape[0]
    A = sys.lig_body.shape[0]
    fb = force_batch or max(1000, int(4 * 1024 ** 3 / max(1, A * 150)))
    fb = min(fb, N_sr)
    F = np.zeros((N_sr, 3))
    T = np.zeros((N_sr, 3))
    for b0 in range(0, N_sr, fb):
        b1 = min(b0 + fb, N_sr)
        R_b = R_sr[b0:b1]
        c_b = cen_sr[b0:b1]
        pos_lig = np.einsum("nij,kj->nki", R_b, sys.lig_body) + c_b[:, None, :]
        f, t, _ = sys.engine(pos_lig, sys.lig_q, R_matrices=R_b, centroids=c_b)
        F[b0:b1] = f
        T[b0:b1] = t
    return F, T


def run(sys: StepSystem, prm: StepParams, noise: str = "pcg64", termination: str = "reference",
        force_batch=None, id_offset: int = 0, init=None) -> StepResult:
    """Run ``prm.n_traj`` trajectories; see the module docstring for the two noise modes.

    ``termination="reference"`` stops the loop when 99.5 % are done or on a stall
    (gpu_batch_simulator.py:1347-1356); ``"complete"`` runs until every
    trajectory has reacted, escaped or used ``max_steps`` steps.  With keyed
    noise, local trajectory i draws as global trajectory ``id_offset + i``.
    ``init`` = (centroids (N, 3), quaternions (N, 4)) starts the trajectories
    from given poses instead of the b-sphere (used to time the loop on an aged
    pool; not part of the reference).
    """
    N = prm.n_traj
    keyed = noise == "philox"
    if keyed:
        draws = KeyedDraws(prm.seed, id_offset)
    else:
        rng = np.random.default_rng(prm.seed)
    if prm.return_prob is None or prm.k_b is None:
        rp, kb = return_prob_and_kb(prm.r_b, prm.r_esc, sys.q_rec_total, sys.q_lig_total, sys.debye, sys.D_t,
                                    prm.use_hi, sys.r_h_rec, sys.r_h_lig, prm.kT_scale)
    else:
        rp, kb = prm.return_prob, prm.k_b
    r_b, r_esc = prm.r_b, prm.r_esc
    all_ids = np.arange(N, dtype=np.int64)
    if keyed:
        v = draws.start_normals(all_ids)
    else:
        v = rng.standard_normal((N, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    pos = v * r_b
    q = shoemake(draws.start_uniforms(all_ids) if keyed else rng.random((N, 3)).astype(np.float64))
    if init is not None:
        pos = np.array(init[0], dtype=np.float64).reshape(N, 3)
        q = np.array(init[1], dtype=np.float64).reshape(N, 4)
    status = np.zeros(N, dtype=np.int32)
    n_steps = np.zeros(N, dtype=np.int64)
    n_returns = np.zeros(N, dtype=np.int64)
    total_steps = 0
    n_overlap = 0
    stall_done = 0
    P = len(sys.rxn_cutoff)
    have_pairs = P > 0
    gho_body = sys.lig_body[sys.rxn_lig_idx] if have_pairs else None
    rec_gho = sys.rxn_rec_pos
    cutoffs = np.asarray(sys.rxn_cutoff, dtype=np.float64)
    n_needed = sys.n_needed
    D_eff = bridge_D_eff(sys)
    sm = sys.sm_before is not None and have_pairs
    state = np.zeros(N, dtype=np.int64)
    fires_d = np.zeros(P, dtype=np.int64)
    fires_b = np.zeros(P, dtype=np.int64)
    if sm:
        before = np.asarray(sys.sm_before, dtype=np.int64)
        after = np.asarray(sys.sm_after, dtype=np.int64)
        terminal = np.asarray(sys.sm_terminal, dtype=bool)
        # bridge draws of state-machine mode come from their own stream (:473-479)
        rng_bb = None if keyed else np.random.default_rng(int(prm.seed) + 1)
    loop_steps = 0
    max_loop = prm.max_steps if termination == "reference" else 1 << 62
    stats = StepStats(pos, q, N, r_b, r_esc, P)
    step = 0
    while step < max_loop:
        running = status == 0
        if keyed:
            running &= n_steps < prm.max_steps
        n_run = int(running.sum())
        if n_run == 0:
            break
        loop_steps += 1
        run_idx = np.where(running)[0]
        pos_run = pos[run_idx]
        q_run = q[run_idx]
        R = rotmats(q_run)
        still_running_mask = status[run_idx] == 0
        if sm:
            # lowest-numbered reaction from the current state within its cutoff (:818-852, :1690-1735)
            gho_pos = np.einsum("nij,kj->nki", R, gho_body) + pos_run[:, None, :]
            d = np.linalg.norm(gho_pos - rec_gho[None, :, :], axis=2)
            fire = (d < cutoffs[None, :]) & (state[run_idx][:, None] == before[None, :])
            reacted = fire.any(axis=1)
            fidx = np.argmax(fire, axis=1)
            fm = reacted & still_running_mask
            newly = run_idx[:0]
            if np.any(fm):
                fg = run_idx[fm]
                fr = fidx[fm]
                ns = after[fr]
                state[fg] = ns
                np.add.at(fires_d, fr, 1)
                newly = fg[terminal[ns]]
        else:
            if have_pairs:
                gho_pos = np.einsum("nij,kj->nki", R, gho_body) + pos_run[:, None, :]
                d = np.linalg.norm(gho_pos - rec_gho[None, :, :], axis=2)
                reacted = (d < cutoffs[None, :]).sum(axis=1) >= n_needed
            else:
                reacted = np.zeros(len(run_idx), dtype=bool)
            newly = run_idx[reacted & still_running_mask]
        status[newly] = 1
        stats.encounter(newly, pos, q, n_steps, bridge=False)
        r_mag = np.linalg.norm(pos_run, axis=1)
        at_escape = (r_mag >= r_esc) & still_running_mask & ~reacted
        if np.any(at_escape):
            esc_idx = run_idx[at_escape]
            if keyed:
                u_outer = draws.u_escape(n_steps[esc_idx], esc_idx)
            else:
                u_outer = rng.random(int(at_escape.sum()))
            returns = u_outer < rp
            if np.any(returns):
                ret_idx = esc_idx[returns]
                new_ret = ret_idx[status[ret_idx] == 0]
                if len(new_ret) > 0:
                    dirs = pos[new_ret] / np.linalg.norm(pos[new_ret], axis=1, keepdims=True)
                    pos[new_ret] = dirs * r_b
                    if keyed:
                        u = draws.return_uniforms(n_steps[new_ret], new_ret)
                    else:
                        u = rng.random((int(len(new_ret)), 3)).astype(np.float64)
                    q[new_ret] = shoemake(u)
                    n_returns[new_ret] += 1
            if np.any(~returns):
                true_esc = esc_idx[~returns]
                new_esc = true_esc[status[true_esc] == 0]
                status[new_esc] = 2
        still_running = status[run_idx] == 0
        pos_run = pos[run_idx]
        q_run = q[run_idx]
        R = rotmats(q_run)
        r_mag = np.linalg.norm(pos_run, axis=1)
        sr_mask = still_running
        sr_idx = run_idx[sr_mask]
        if len(sr_idx) == 0:
            step += 1
            continue
        R_sr = R[sr_mask]
        cen_sr = pos_run[sr_mask]
        N_sr = len(sr_idx)
        forces, torques = _forces(sys, R_sr, cen_sr, force_batch)
        old_d = None
        if have_pairs:
            lig_old = np.einsum("nij,kj->nki", R_sr, gho_body) + cen_sr[:, None, :]
            old_d = np.linalg.norm(lig_old - rec_gho[None, :, :], axis=2)
        r_sr = r_mag[sr_mask]
        rxn_coord = None
        if sm:
            reach = state[sr_idx][:, None] == before[None, :]
            coord = np.maximum(old_d - cutoffs[None, :], np.zeros_like(old_d))
            rxn_coord = np.min(np.where(reach, coord, 1.0e30), axis=1)
        dt_arr = adaptive_dt(r_sr, sys, prm, rxn_coord)
        D_arr = hi_diffusion(r_sr, sys, prm)
        if keyed:
            xi_t, xi_r = draws.step_normals(n_steps[sr_idx], sr_idx)
        else:
            xi_t = rng.standard_normal((N_sr, 3))
        sigma_t = np.sqrt(2.0 * D_arr * dt_arr)[:, None]
        drift = D_arr[:, None] * dt_arr[:, None] * forces
        old_pos = pos[sr_idx].copy() if prm.overlap else None
        old_q = q[sr_idx].copy() if prm.overlap else None
        pos[sr_idx] += drift + sigma_t * xi_t
        if not keyed:
            xi_r = rng.standard_normal((N_sr, 3))
        sigma_r = np.sqrt(2.0 * sys.D_r * dt_arr)[:, None]
        omega = sys.D_r * dt_arr[:, None] * torques + sigma_r * xi_r
        q[sr_idx] = apply_rotation(q[sr_idx], omega)
        if prm.overlap and sys.rec_pos is not None and len(sys.rec_pos) > 0:
            inside = _overlap_inside(pos[sr_idx], sys.rec_pos)
            if np.any(inside):
                ii = np.where(inside)[0]
                pos[sr_idx[ii]] = old_pos[ii]
                q[sr_idx[ii]] = old_q[ii]
                n_overlap += int(ii.shape[0])
        if old_d is not None:
            R_new = rotmats(q[sr_idx])
            lig_new = np.einsum("nij,kj->nki", R_new, gho_body) + pos[sr_idx][:, None, :]
            new_d = np.linalg.norm(lig_new - rec_gho[None, :, :], axis=2)
            x0 = old_d - cutoffs[None, :]
            x1 = new_d - cutoffs[None, :]
            both = (x0 > 0) & (x1 > 0)
            # The reference evaluates the bridge only when some trajectory of the
            # batch has a pair above the surface at both ends (:1161); per
            # trajectory the outcome is the same either way (a pair below the
            # surface is caught by the next discrete test at the same pose).
            if keyed or np.any(both):
                if D_eff is not None:
                    Ddt = D_eff[None, :] * dt_arr[:, None]
                else:
                    Ddt = sys.D_t * dt_arr[:, None]
                Ddt = np.maximum(Ddt, np.full_like(Ddt, 1e-30))
                p_cross = np.exp(-x0 * x1 / Ddt)
                p_cross = np.where(both, p_cross, np.zeros_like(p_cross))
                if keyed:
                    u_bb = draws.bridge_uniforms(n_steps[sr_idx], sr_idx, P)
                elif sm:
                    u_bb = rng_bb.random(p_cross.shape)
                else:
                    u_bb = rng.random(p_cross.shape)
                fired = (u_bb < p_cross) | (new_d < cutoffs[None, :])
                if sm:
                    fm = fired & (state[sr_idx][:, None] == before[None, :])
                    anyf = fm.any(axis=1)
                    if np.any(anyf):
                        fidx = np.argmax(fm, axis=1)
                        proceed = anyf & (status[sr_idx] == 0)
                        if np.any(proceed):
                            g = sr_idx[proceed]
                            fr = fidx[proceed]
                            ns = after[fr]
                            state[g] = ns
                            np.add.at(fires_b, fr, 1)
                            gt = g[terminal[ns]]
                            status[gt] = 1
                            stats.encounter(gt, pos, q, n_steps, bridge=True)
                else:
                    bb = fired.sum(axis=1) >= n_needed
                    if np.any(bb):
                        g = sr_idx[bb]
                        g = g[status[g] == 0]
                        status[g] = 1
                        stats.encounter(g, pos, q, n_steps, bridge=True)
        stats.step(sr_idx, pos, q, n_steps, dt_arr, old_d, cutoffs)
        stats.trace(sr_idx, pos, q, n_steps, forces, dt_arr, prm.save_interval)
        n_steps[sr_idx] += 1
        total_steps += int(sr_mask.sum())
        done = int((status != 0).sum())
        if termination == "reference":
            if done >= int(N * 0.995):
                break
            if step > 0 and step % 10000 == 0:
                if done > int(N * 0.95) and done - stall_done < max(2, int(N * 0.001)):
                    break
                stall_done = done
        step += 1
    if keyed:
        status[(status == 0) & (n_steps >= prm.max_steps)] = 3
    n_max = int((status == 0).sum()) + int((status == 3).sum())
    status[status == 0] = 3
    return StepResult(status=status, n_steps=n_steps, n_reacted=int((status == 1).sum()),
                      n_escaped=int((status == 2).sum()), n_max_steps=n_max, total_steps=total_steps,
                      loop_steps=loop_steps, return_prob=rp, k_b=kb, n_returns=n_returns,
                      n_overlap_rejected=n_overlap, stats=stats, state=state, sm_fires_discrete=fires_d,
                      sm_fires_bridge=fires_b, pos=pos, q=q)
