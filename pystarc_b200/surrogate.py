"""Learned surrogate for the reverse-Born plus far-field force and torque.

No reference counterpart: this is the engine's learned part.  An ensemble of
MLPs (13 features -> 256 x 4 SiLU -> 6 outputs by default) is trained on poses
from exact-kernel BD trajectories and on the exact kernels' reverse-Born plus
far-field force and torque at those poses.  Training and inference run in the
CUDA library (``bd_mlp_*``: BF16 tensor-core forward, backward and Adam with
FP32 accumulation); PyTorch only holds the device tensors.

Features of a pose (centroid c in the receptor frame, quaternion q):
``c / r_scale`` (3), ``|c| / r_scale`` (1), ``q`` with ``w >= 0`` (4; q and -q are
the same rotation), and Gaussian radial basis values of ``|c|`` (5 centres on
25-80 A).  Targets are force and torque divided by per-component scales taken
from the training set.  The surrogate is trusted only for
``contact + margin <= |c| <= r_max`` and while the ensemble agrees (member spread
of the force within ``threshold`` of its size); elsewhere the exact kernels
run.  Which force terms it replaces is ``SurrogateSpec.terms``: the far-field and
reverse Born by default, or with the grid terms too (the total force, which is
smooth where a ligand atom leaves the electrostatic grid and the far-field takes
over, while each term alone jumps there).
"""

from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass, field

import numpy as np

from . import _lib

N_FEATURES = 13
N_OUT = 6


@dataclass
class SurrogateSpec:
    """Feature map, output scales and trust region of a trained surrogate."""

    r_scale: float = 80.0
    rbf_centres: tuple = (25.0, 38.75, 52.5, 66.25, 80.0)
    rbf_width: float = 13.75
    out_scale: tuple = (1.0,) * N_OUT
    r_min: float = 0.0  # contact + margin
    r_max: float = 80.0  # upper end of the training poses
    threshold: float = 0.02  # ensemble force spread / force size above which the exact path runs
    force_floor: float = 0.0  # in envelope units: force sizes below force_floor * envelope count as that
    env_r0: float = 0.0  # radial envelope: log force size at N_ENV radii from env_r0 to env_r1
    env_r1: float = 0.0
    env_log: tuple = (0.0,) * 32
    terms: int = _lib.TERM_FARFIELD | _lib.TERM_REV_BORN  # force terms the surrogate replaces

    def features(self, c, q):
        """(n, 13) float32 features of centroids c (n, 3) and quaternions q (n, 4, w first)."""
        c = np.asarray(c, dtype=np.float64).reshape(-1, 3)
        q = np.asarray(q, dtype=np.float64).reshape(-1, 4)
        r = np.linalg.norm(c, axis=1)
        qs = np.where(q[:, :1] < 0, -q, q)
        mu = np.asarray(self.rbf_centres)
        rbf = np.exp(-0.5 * ((r[:, None] - mu[None, :]) / self.rbf_width) ** 2)
        f = np.concatenate([c / self.r_scale, (r / self.r_scale)[:, None], qs, rbf], axis=1)
        return f.astype(np.float32)

    def envelope(self, r):
        """Radial envelope of the outputs (the device's sur_envelope)."""
        r = np.asarray(r, dtype=np.float64)
        if not self.env_r1 > self.env_r0:
            return np.ones_like(r)
        k = len(self.env_log)
        u = np.clip((r - self.env_r0) / (self.env_r1 - self.env_r0) * (k - 1), 0.0, k - 1.0)
        i = np.minimum(u.astype(np.int64), k - 2)
        t = u - i
        lg = np.asarray(self.env_log)
        return np.exp((1.0 - t) * lg[i] + t * lg[i + 1])

    def fit_envelope(self, r, force, bins=32):
        """Envelope from training targets: log RMS force size in evenly spaced radial bins."""
        r = np.asarray(r, dtype=np.float64)
        f2 = np.sum(np.asarray(force, dtype=np.float64) ** 2, axis=1)
        lo, hi = float(r.min()), float(r.max())
        edges = np.linspace(lo, hi, bins + 1)
        idx = np.clip(np.searchsorted(edges, r, side="right") - 1, 0, bins - 1)
        cnt = np.bincount(idx, minlength=bins)
        rms = np.sqrt(np.bincount(idx, weights=f2, minlength=bins) / np.maximum(cnt, 1))
        ok = (cnt > 0) & (rms > 0)
        centres = 0.5 * (edges[:-1] + edges[1:])
        grid = np.linspace(lo, hi, bins)
        if ok.sum() == 0:
            self.env_r0 = self.env_r1 = 0.0
            return
        self.env_log = tuple(float(v) for v in np.interp(grid, centres[ok], np.log(rms[ok])))
        self.env_r0, self.env_r1 = lo, hi

    def c_params(self):
        """The ``BdSurrogateParams`` of this spec."""
        p = _lib.BdSurrogateParams()
        p.r_scale = self.r_scale
        for k in range(5):
            p.rbf_centre[k] = self.rbf_centres[k]
        p.rbf_width = self.rbf_width
        for k in range(N_OUT):
            p.out_scale[k] = self.out_scale[k]
        p.r_min, p.r_max, p.threshold, p.force_floor = self.r_min, self.r_max, self.threshold, self.force_floor
        p.env_r0, p.env_r1 = self.env_r0, self.env_r1
        for k in range(32):
            p.env_log[k] = self.env_log[k]
        p.terms = int(self.terms)
        return p

    def trusted(self, c):
        r = np.linalg.norm(np.asarray(c, dtype=np.float64).reshape(-1, 3), axis=1)
        return (r >= self.r_min) & (r <= self.r_max)


class MLPEnsemble:
    """``bd_mlp_*`` ensemble on one device; inputs and outputs are CUDA float32 tensors."""

    def __init__(self, n_members=5, in_dim=N_FEATURES, hidden=256, n_hidden=4, out_dim=N_OUT, seed=0, device=0):
        self.lib = _lib.load()
        d = _lib.BdMlpDesc(n_members, in_dim, hidden, n_hidden, out_dim, 0, int(seed) & 0xFFFFFFFFFFFFFFFF)
        h = _lib.P()
        rc = self.lib.bd_mlp_create(int(device), C.byref(d), C.byref(h))
        if rc != _lib.BD_OK:
            raise _lib.BdError(rc, "bd_mlp_create failed (check the shape limits and the device)")
        self.h = h
        self.device = int(device)
        self.n_members, self.in_dim, self.hidden, self.n_hidden, self.out_dim = (n_members, in_dim, hidden,
                                                                                  n_hidden, out_dim)
        n = C.c_int64()
        self._call("bd_mlp_n_params", C.byref(n))
        self.n_params = int(n.value)

    def _call(self, name, *args):
        return _lib.check_mlp(getattr(self.lib, name)(self.h, *args), self.h)

    @property
    def dims(self):
        d = [self.in_dim] + [self.hidden] * self.n_hidden + [self.out_dim]
        return list(zip(d[:-1], d[1:]))

    def _stream(self):
        import torch

        return _lib.P(torch.cuda.current_stream(self.device).cuda_stream)

    def _dev(self, x):
        import torch

        return torch.as_tensor(x, dtype=torch.float32, device=f"cuda:{self.device}").contiguous()

    def get_params(self, member):
        out = np.empty(self.n_params, dtype=np.float32)
        self._call("bd_mlp_get_params", int(member), _lib.ptr(out, C.c_float))
        return out

    def set_params(self, member, params):
        a = np.ascontiguousarray(params, dtype=np.float32)
        if a.size != self.n_params:
            raise ValueError(f"expected {self.n_params} parameters, got {a.size}")
        self._call("bd_mlp_set_params", int(member), _lib.ptr(a, C.c_float))

    def forward(self, member, X):
        import torch

        X = self._dev(X)
        Y = torch.empty((X.shape[0], self.out_dim), dtype=torch.float32, device=X.device)
        self._call("bd_mlp_forward", int(member), X.shape[0], _lib.P(X.data_ptr()), _lib.P(Y.data_ptr()),
                   self._stream())
        return Y

    def grad(self, member, X, T):
        """(loss, gradient) of the mean squared error on a batch (rows a multiple of 32)."""
        import torch

        X, T = self._dev(X), self._dev(T)
        g = torch.empty(self.n_params, dtype=torch.float32, device=X.device)
        loss = torch.empty(1, dtype=torch.float32, device=X.device)
        self._call("bd_mlp_grad", int(member), X.shape[0], _lib.P(X.data_ptr()), _lib.P(T.data_ptr()),
                   _lib.P(g.data_ptr()), _lib.P(loss.data_ptr()), self._stream())
        return float(loss.item()), g

    def train_step(self, member, X, T, lr, loss=None):
        """One Adam step; ``loss`` (a 1-element CUDA tensor) receives the batch loss if given."""
        self._call("bd_mlp_train_step", int(member), X.shape[0], _lib.P(X.data_ptr()), _lib.P(T.data_ptr()),
                   C.c_float(lr), _lib.P(loss.data_ptr() if loss is not None else 0), self._stream())

    def set_inference(self, mode):
        """1: tcgen05 inference kernel (default), 0: the mma.sync GEMM chain."""
        self._call("bd_mlp_set_inference", int(mode))

    def set_gemm(self, mode):
        """GEMMs of training and of the GEMM chain: 1 tcgen05 (default), 0 mma.sync."""
        self._call("bd_mlp_set_gemm", int(mode))

    def train(self, member, X, T, batch, steps, lr, seed=0, trace=True):
        """``steps`` Adam steps on random batches of device-resident (X, T); returns the loss trace."""
        import torch

        X, T = self._dev(X), self._dev(T)
        tr = torch.zeros(max(steps, 1), dtype=torch.float32, device=X.device) if trace else None
        self._call("bd_mlp_train", int(member), X.shape[0], _lib.P(X.data_ptr()), _lib.P(T.data_ptr()), int(batch),
                   int(steps), C.c_float(lr), int(seed) & 0xFFFFFFFFFFFFFFFF,
                   _lib.P(tr.data_ptr() if tr is not None else 0), self._stream())
        return tr

    def ensemble(self, X):
        import torch

        X = self._dev(X)
        mean = torch.empty((X.shape[0], self.out_dim), dtype=torch.float32, device=X.device)
        spread = torch.empty_like(mean)
        self._call("bd_mlp_ensemble", X.shape[0], _lib.P(X.data_ptr()), _lib.P(mean.data_ptr()),
                   _lib.P(spread.data_ptr()), self._stream())
        return mean, spread

    def close(self):
        if self.h:
            self.lib.bd_mlp_destroy(self.h)
            self.h = _lib.P()

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown
            pass


# ---------------------------------------------------------------------------------------- training
def sample_poses(sim, n_poses, r_lo=25.0, r_hi=80.0, launches_between=2, steps_per_launch=16, max_rounds=100000,
                 max_seconds=None):
    """Poses (c, q) of live trajectories of an exact-kernel BD run, kept where r_lo <= |c| <= r_hi.

    ``sim`` is a configured ``B200BatchSimulator`` (any precision); its pool is
    advanced ``launches_between`` launches between snapshots.  Raises RuntimeError when
    ``max_rounds`` snapshots or ``max_seconds`` seconds pass with fewer than ``n_poses`` kept.
    """
    t_end = None if max_seconds is None else time.perf_counter() + max_seconds
    h = sim.engine.handle
    sim._setup()
    h.call("bd_sim_reset", None)
    cap = _lib.C.c_int32()
    h.call("bd_sim_capacity", _lib.C.byref(cap))
    C_ = int(cap.value)
    cs, qs, got = [], [], 0
    for _ in range(max_rounds):
        h.call("bd_sim_run", launches_between, steps_per_launch, None)
        c = np.empty((3, C_))
        q = np.empty((4, C_))
        traj = np.empty(C_, dtype=np.int32)
        steps = np.empty(C_, dtype=np.int32)
        rets = np.empty(C_, dtype=np.int32)
        st = np.empty(C_, dtype=np.int8)
        live = _lib.C.c_int32()
        ctr = np.empty(_lib.N_CTR + 2, dtype=np.uint64)
        h.call("bd_sim_snapshot", _lib.ptr(c), _lib.ptr(q), _lib.ptr(traj, C.c_int32), _lib.ptr(steps, C.c_int32),
               _lib.ptr(rets, C.c_int32), _lib.ptr(st, C.c_int8), _lib.C.byref(live), _lib.ptr(ctr, C.c_uint64))
        n = int(live.value)
        if n == 0:
            h.call("bd_sim_reset", None)
            continue
        cc = c[:, :n].T.copy()
        qq = q[:, :n].T.copy()
        r = np.linalg.norm(cc, axis=1)
        keep = (r >= r_lo) & (r <= r_hi) & (st[:n] == 0)
        cs.append(cc[keep])
        qs.append(qq[keep])
        got += int(keep.sum())
        if got >= n_poses:
            break
        if t_end is not None and time.perf_counter() > t_end:
            break
    if got < n_poses:
        raise RuntimeError(f"sample_poses: {got} of {n_poses} poses in [{r_lo}, {r_hi}] A kept")
    c = np.concatenate(cs)[:n_poses]
    q = np.concatenate(qs)[:n_poses]
    return c, q


def exact_targets(engine, c, q, chunk=200_000, precision="fp64", terms=_lib.TERM_FARFIELD | _lib.TERM_REV_BORN):
    """Exact force and torque (n, 6) of the ``terms`` (``_lib.TERM_*`` bits; by default reverse Born
    plus far-field) of the engine's ligand at poses (``precision="mixed"``: FP32 force arithmetic,
    ~1e-6 relative, far below the network's error)."""
    out = []
    for i in range(0, len(c), chunk):
        F, T, _ = engine.eval_poses(c[i:i + chunk], q[i:i + chunk], precision=precision, terms=terms)
        out.append(np.concatenate([F, T], axis=1))
    return np.concatenate(out) if out else np.zeros((0, 6))


@dataclass
class TrainReport:
    steps: int
    batch: int
    seconds: float
    final_loss: list = field(default_factory=list)
    heldout_rel_err: dict = field(default_factory=dict)


def fit(ens, spec, c, q, targets, steps=20000, batch=8192, lr=1e-3, seed=0, log=None):
    """Train every member on (features(c, q), targets / out_scale); returns a TrainReport.

    Members see the same data in different orders (seed + member).  The output
    scales are set on ``spec`` from the targets' RMS per component.
    """
    import torch

    rr = np.linalg.norm(np.asarray(c, dtype=np.float64), axis=1)
    spec.fit_envelope(rr, np.asarray(targets)[:, :3])
    env = spec.envelope(rr)[:, None]
    t = np.asarray(targets, dtype=np.float64) / env
    rms = np.sqrt(np.mean(t ** 2, axis=0))
    spec.out_scale = tuple(float(max(v, 1e-12)) for v in rms)
    spec.force_floor = float(0.05 * np.sqrt(np.mean(np.sum(t[:, :3] ** 2, axis=1))))
    dev = f"cuda:{ens.device}"
    X = torch.as_tensor(spec.features(c, q), device=dev)
    Y = torch.as_tensor((t / np.asarray(spec.out_scale)).astype(np.float32), device=dev)
    n = X.shape[0]
    batch = min(batch, n - n % 32)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    finals = []
    for m in range(ens.n_members):
        tr = ens.train(m, X, Y, batch, steps, lr, seed=int(seed) * 1000 + m)
        t = tr.cpu().numpy()
        tail = t[-max(1, steps // 20):]
        finals.append(float(tail.mean()))
        if log:
            for s in range(0, steps, max(1, steps // 10)):
                log(f"member {m} step {s} loss {t[s]:.4e}")
            log(f"member {m} final loss {finals[-1]:.4e}")
    torch.cuda.synchronize(dev)
    return TrainReport(steps=steps, batch=batch, seconds=time.perf_counter() - t0, final_loss=finals)


def heldout_error(ens, spec, c, q, targets):
    """Relative force error of the ensemble mean on held-out poses, against the exact targets."""
    mean, spread = ens.ensemble(spec.features(c, q))
    env = spec.envelope(np.linalg.norm(np.asarray(c, dtype=np.float64), axis=1))[:, None]
    pred = mean.cpu().numpy().astype(np.float64) * np.asarray(spec.out_scale) * env
    t = np.asarray(targets, dtype=np.float64)
    fn = np.linalg.norm(t[:, :3], axis=1)
    denom = np.maximum(fn, spec.force_floor * env[:, 0])
    err = np.linalg.norm(pred[:, :3] - t[:, :3], axis=1) / denom
    zero = np.linalg.norm(t[:, :3], axis=1) / denom  # the method without the surrogate terms
    sp = spread.cpu().numpy().astype(np.float64) * np.asarray(spec.out_scale) * env
    dis = np.linalg.norm(sp[:, :3], axis=1) / denom
    return {"median": float(np.median(err)), "p99": float(np.percentile(err, 99)), "max": float(err.max()),
            "without_surrogate_median": float(np.median(zero)), "fallback_fraction": float(np.mean(dis > spec.threshold)),
            "n": int(len(err))}


def contact_distance(rec_pos, lig_pos):
    """Receptor and ligand extents from their centres: the centre distance at contact."""
    rec = np.asarray(rec_pos, dtype=np.float64)
    lig = np.asarray(lig_pos, dtype=np.float64)
    return float(np.linalg.norm(rec, axis=1).max() + np.linalg.norm(lig - lig.mean(axis=0), axis=1).max())


def rbf_default(r_lo=25.0, r_hi=80.0, k=5):
    c = np.linspace(r_lo, r_hi, k)
    return tuple(float(v) for v in c), float((r_hi - r_lo) / (k - 1))


__all__ = ["SurrogateSpec", "MLPEnsemble", "sample_poses", "exact_targets", "fit", "heldout_error",
           "contact_distance", "rbf_default", "TrainReport", "N_FEATURES", "N_OUT"]
