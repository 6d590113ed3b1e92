"""``B200ForceEngine``: drop-in for the reference's ``GPUBatchForceEngine``.

Constructor arguments and ``__call__`` follow pystarc/forces/gpu_batch_engine.py:139-154
and :531-605; the attributes the reference stepper reads (``_debye``,
``_has_yukawa``, ``_V_factor``, ``_rec_charge``, ``_elec_grids_gpu``,
``_born_grids_gpu``, ``alpha``) exist with the same meaning.  The arithmetic
runs in ``libpystarc_b200.so`` on the GPU; there is no CPU path.

``use_lj`` with ``rec_radii`` / ``lig_radii`` adds the WCA contact forces
(gpu_batch_engine.py:474-529) to every force evaluation, the stepper's included.

Beyond the reference: ``precision`` ("fp64" or "mixed": FP32 force arithmetic
with FP64 geometry and sums) and ``torque_mode`` ("zero", the reference GPU
path's placeholder, or "centroid": torque about the ligand centroid argument).
"""

from __future__ import annotations

import math

import numpy as np

from . import _lib
from .hostphys import EPS0

PRECISIONS = {"fp64": _lib.PREC_FP64, "mixed": _lib.PREC_MIXED}
TORQUES = {"zero": _lib.TORQUE_ZERO, "centroid": _lib.TORQUE_CENTROID}


def _grid_args(g):
    data = np.ascontiguousarray(np.asarray(g.data), dtype=np.float32)
    delta = np.asarray(g.delta, dtype=float)
    sp = np.ascontiguousarray([delta[i, i] for i in range(3)], dtype=np.float64)
    origin = np.ascontiguousarray(g.origin, dtype=np.float64)
    return data, sp, origin


def _sp(g):
    return float(np.asarray(g.delta, dtype=float)[0, 0])


class EngineHandle:
    """Owns one ``BdHandle`` (device memory lives until ``close``)."""

    def __init__(self, device=0):
        lib = _lib.load()
        h = _lib.P()
        _lib.check(lib.bd_create(int(device), _lib.C.byref(h)), None)
        self.lib = lib
        self.h = h
        self.device = int(device)

    def call(self, name, *args):
        return _lib.check(getattr(self.lib, name)(self.h, *args), self.h)

    def close(self):
        if self.h:
            self.lib.bd_destroy(self.h)
            self.h = _lib.P()

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown
            pass


class B200ForceEngine:
    def __init__(self, elec_grids, born_grids, alpha: float = 0.07957747, receptor_charge: float = 0.0,
                 debye_length: float = 7.858, sdie: float = 78.0, lig_born_grids=None, rec_positions=None,
                 rec_charges=None, multipole_expansion=None, rec_radii=None, lig_radii=None, use_lj=False, *,
                 precision: str = "fp64", torque_mode: str = "zero", device: int = 0, layout=None):
        if precision not in PRECISIONS or torque_mode not in TORQUES:
            raise ValueError(f"precision in {list(PRECISIONS)}, torque_mode in {list(TORQUES)}")
        self.alpha = float(alpha)
        self._rec_charge = float(receptor_charge)
        self._debye = float(debye_length)
        self._sdie = float(sdie)
        eps_s = self._sdie * EPS0
        self._V_factor = self._rec_charge / (4.0 * math.pi * eps_s) if eps_s > 0 else 0.0
        self._has_yukawa = abs(self._rec_charge) > 1e-9 and self._debye > 0
        self._multipole = multipole_expansion
        self.precision = precision
        self.torque_mode = torque_mode
        self.handle = EngineHandle(device)
        if layout is not None:  # bit flags of the device data layout (identical results in every layout)
            self.handle.call("bd_set_layout", int(layout))
        elec = sorted(list(elec_grids or []), key=_sp)
        born = sorted(list(born_grids or []), key=_sp)
        if self._has_yukawa and len(elec) > 1:
            elec = elec[:1]
        born = born[:1]
        self._elec_grids_gpu = [self._grid_info(g) for g in elec]
        self._born_grids_gpu = [self._grid_info(g) for g in born]
        for g in elec:
            self._add(_lib.GRID_ELEC, g)
        for g in born:
            self._add(_lib.GRID_BORN, g)
        self._lig_born_grids_gpu = []
        self.rec_positions = None
        self.rec_charges = None
        if rec_positions is not None and rec_charges is not None:
            self.rec_positions = np.ascontiguousarray(rec_positions, dtype=np.float64).reshape(-1, 3)
            self.rec_charges = np.ascontiguousarray(rec_charges, dtype=np.float64).reshape(-1)
            self.handle.call("bd_set_receptor", len(self.rec_charges), _lib.ptr(self.rec_positions),
                             _lib.ptr(self.rec_charges))
            if lig_born_grids:
                lb = sorted(list(lig_born_grids), key=_sp)[:1]
                self._lig_born_grids_gpu = [self._grid_info(g) for g in lb]
                for g in lb:
                    self._add(_lib.GRID_LIG_BORN, g)
        # WCA contact forces from the atom radii (gpu_batch_engine.py:233-246): on when use_lj and both
        # radii are given; every receptor atom, charged or not, takes part
        self._use_lj = bool(use_lj)
        self._rec_radii_gpu = None
        self._lig_radii_gpu = None
        if use_lj and rec_radii is not None and lig_radii is not None:
            if self.rec_positions is None:
                raise ValueError("use_lj needs rec_positions and rec_charges")
            self._rec_radii_gpu = np.ascontiguousarray(rec_radii, dtype=np.float64).reshape(-1)
            self._lig_radii_gpu = np.ascontiguousarray(lig_radii, dtype=np.float64).reshape(-1)
            if self._rec_radii_gpu.shape[0] != self.rec_positions.shape[0]:
                raise ValueError("rec_radii does not match rec_positions")
            self._lj_epsilon = 0.17
            self._lj_activation = float(self._rec_radii_gpu.max() + self._lig_radii_gpu.max()) * 2.5
            self.handle.call("bd_set_contact", len(self._rec_radii_gpu), _lib.ptr(self._rec_radii_gpu),
                             len(self._lig_radii_gpu), _lib.ptr(self._lig_radii_gpu), self._lj_epsilon,
                             self._lj_activation)
        fp = _lib.BdForceParams()
        fp.receptor_charge = self._rec_charge
        fp.debye_length = self._debye
        fp.sdie = self._sdie
        fp.alpha = self.alpha
        if multipole_expansion is not None:
            fp.use_multipole = 1
            for i in range(3):
                fp.dipole[i] = float(multipole_expansion.dipole[i])
            Q = np.asarray(multipole_expansion.quadrupole, dtype=float).reshape(9)
            for i in range(9):
                fp.quadrupole[i] = float(Q[i])
            fp.four_pi_eps = float(multipole_expansion.four_pi_eps)
        self.handle.call("bd_set_force_params", _lib.C.byref(fp))
        self._lig_key = None
        self._call_count = 0

    @staticmethod
    def _grid_info(g):
        data = np.asarray(g.data)
        delta = np.asarray(g.delta, dtype=float)
        sp = np.array([delta[i, i] for i in range(3)])
        dims = np.array(data.shape)
        origin = np.asarray(g.origin, dtype=float)
        return {"nx": int(dims[0]), "ny": int(dims[1]), "nz": int(dims[2]), "origin": origin, "sp": sp,
                "lo": origin + 3.0 * sp, "hi": origin + (dims - 1 - 3.0) * sp}

    def _add(self, kind, g):
        data, sp, origin = _grid_args(g)
        nx, ny, nz = data.shape
        self.handle.call("bd_add_grid", kind, _lib.ptr(data, _lib.C.c_float), nx, ny, nz, _lib.ptr(origin),
                         _lib.ptr(sp))

    def set_ligand(self, body_xyz, charges):
        """Ligand atoms about its centroid (the stepper sets this; __call__ needs only the charges)."""
        body = np.ascontiguousarray(body_xyz, dtype=np.float64).reshape(-1, 3)
        q = np.ascontiguousarray(charges, dtype=np.float64).reshape(-1)
        key = (body.tobytes(), q.tobytes())
        if key != self._lig_key:
            self.handle.call("bd_set_ligand", len(q), _lib.ptr(body), _lib.ptr(q))
            self._lig_key = key

    # ------------------------------------------------------------------
    def __call__(self, lig_positions, lig_charges, R_matrices=None, centroids=None):
        """Net (forces (N,3), torques (N,3), energies (N,)) for N trajectories.

        Accepts NumPy arrays (copied to and from the device) or CUDA torch tensors
        (used in place; results are torch tensors on the same device).
        """
        import torch

        as_torch = isinstance(lig_positions, torch.Tensor)
        dev = torch.device("cuda", self.handle.device)
        pos = torch.as_tensor(lig_positions, dtype=torch.float64, device=dev).contiguous()
        N, A, _ = pos.shape
        q = np.asarray(lig_charges.detach().cpu() if isinstance(lig_charges, torch.Tensor) else lig_charges,
                       dtype=np.float64).reshape(-1)
        if q.shape[0] != A:
            raise ValueError("lig_charges does not match lig_positions")
        if self._lig_key is None or np.frombuffer(self._lig_key[1], dtype=np.float64).shape[0] != A or \
                not np.array_equal(np.frombuffer(self._lig_key[1], dtype=np.float64), q):
            self.set_ligand(np.zeros((A, 3)), q)
        if R_matrices is None or centroids is None:
            R = torch.eye(3, dtype=torch.float64, device=dev).expand(N, 3, 3).contiguous()
            c = pos.mean(dim=1).contiguous()
            if self._lig_born_grids_gpu:
                raise ValueError("Born direction 2 needs R_matrices and centroids")
        else:
            R = torch.as_tensor(R_matrices, dtype=torch.float64, device=dev).reshape(N, 9).contiguous()
            c = torch.as_tensor(centroids, dtype=torch.float64, device=dev).reshape(N, 3).contiguous()
        F = torch.empty((N, 3), dtype=torch.float64, device=dev)
        T = torch.empty((N, 3), dtype=torch.float64, device=dev)
        E = torch.empty((N,), dtype=torch.float64, device=dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        self.handle.call("bd_eval_forces_atoms", N, _lib.P(pos.data_ptr()), _lib.P(R.data_ptr()),
                         _lib.P(c.data_ptr()), _lib.P(F.data_ptr()), _lib.P(T.data_ptr()), _lib.P(E.data_ptr()),
                         PRECISIONS[self.precision], TORQUES[self.torque_mode], _lib.P(stream))
        self._call_count += 1
        if as_torch:
            return F, T, E
        return F.cpu().numpy(), T.cpu().numpy(), E.cpu().numpy()

    def eval_overlap(self, centroids):
        """The stepper's overlap test (gpu_batch_simulator.py:770-781, 1102-1128): a bool per centroid,
        True when some receptor atom lies within 1.5 A of it."""
        import torch

        dev = torch.device("cuda", self.handle.device)
        c = torch.as_tensor(centroids, dtype=torch.float64, device=dev).reshape(-1, 3).contiguous()
        out = torch.empty(c.shape[0], dtype=torch.int8, device=dev)
        self.handle.call("bd_eval_overlap", c.shape[0], _lib.P(c.data_ptr()), _lib.P(out.data_ptr()),
                         _lib.P(torch.cuda.current_stream(dev).cuda_stream))
        return out.cpu().numpy().astype(bool)

    def eval_poses(self, centroids, rotations, precision=None, torque_mode=None, terms=None):
        """Forces for poses (centroid + quaternion (w,x,y,z) or 3x3 matrix) with the ligand from ``set_ligand``.

        ``terms`` (``_lib.TERM_*`` bits) restricts the sum to some force terms; the
        surrogate's training targets are the terms it replaces (``SurrogateSpec.terms``).
        """
        import torch

        if terms is not None:
            self.handle.call("bd_set_terms", int(terms))
            try:
                return self.eval_poses(centroids, rotations, precision, torque_mode)
            finally:
                self.handle.call("bd_set_terms", _lib.TERM_ALL)

        dev = torch.device("cuda", self.handle.device)
        as_torch = isinstance(centroids, torch.Tensor)
        c = torch.as_tensor(centroids, dtype=torch.float64, device=dev).reshape(-1, 3).contiguous()
        N = c.shape[0]
        r = torch.as_tensor(rotations, dtype=torch.float64, device=dev)
        is_mat = r.numel() == 9 * N
        r = r.reshape(N, 9 if is_mat else 4).contiguous()
        F = torch.empty((N, 3), dtype=torch.float64, device=dev)
        T = torch.empty((N, 3), dtype=torch.float64, device=dev)
        E = torch.empty((N,), dtype=torch.float64, device=dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        self.handle.call("bd_eval_forces", N, _lib.P(c.data_ptr()), _lib.P(r.data_ptr()), int(is_mat),
                         _lib.P(F.data_ptr()), _lib.P(T.data_ptr()), _lib.P(E.data_ptr()),
                         PRECISIONS[precision or self.precision], TORQUES[torque_mode or self.torque_mode],
                         _lib.P(stream))
        if as_torch:
            return F, T, E
        return F.cpu().numpy(), T.cpu().numpy(), E.cpu().numpy()

    def close(self):
        self.handle.close()
