"""FP64 CPU restatement of the reference's batched force engine (test infrastructure).

This is the checker for the CUDA force kernels: only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg use it.  Each
function follows one piece of pystarc/forces/gpu_batch_engine.py:

* ``k1_batch_force``   -- ``batch_force_kernel`` (gpu_batch_engine.py:65-123)
* ``prepare_grids``    -- ``_upload_grids`` margins, finest-first order and the
                          grid-dropping rules of ``__init__`` (:179-211, :248-287)
* ``eval_batch``       -- ``_eval_batch`` (:289-391)
* ``yukawa_forces``    -- ``_yukawa_forces_gpu`` (:393-472)
* ``born_reverse``     -- ``_eval_born_reverse`` (:607-657)
* ``wca_forces``       -- ``_wca_forces_gpu`` and its activation radius (:233-246, :474-529)
* ``OracleForceEngine.__call__`` -- ``GPUBatchForceEngine.__call__`` (:531-605)

Beyond the reference, ``OracleForceEngine`` can also return the torque about the
ligand centroid (the rotation centre of the stepper,
gpu_batch_simulator.py:172-174) and the per-atom force magnitudes used by the
force-error metric.  The reference GPU path returns zero torque (:597-599).
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

EPS0 = 0.000142  # e^2/(kBT*A), pystarc/forces/multipole_farfield.py:87
GRID_MARGIN = 3.0  # spacings, gpu_batch_engine.py:271


# --------------------------------------------------------------------------
# K1: batch_force_kernel
# --------------------------------------------------------------------------
def _interp(data, origin, inv_sp, x, y, z):
    """Trilinear interpolation with the kernel's bounds rule (gpu_batch_engine.py:95-110)."""
    nx, ny, nz = data.shape
    ix = (x - origin[0]) * inv_sp[0]
    iy = (y - origin[1]) * inv_sp[1]
    iz = (z - origin[2]) * inv_sp[2]
    i0 = np.floor(ix)
    j0 = np.floor(iy)
    k0 = np.floor(iz)
    valid = (i0 >= 0) & (i0 < nx - 1) & (j0 >= 0) & (j0 < ny - 1) & (k0 >= 0) & (k0 < nz - 1)
    i0 = np.where(valid, i0, 0).astype(np.int64)
    j0 = np.where(valid, j0, 0).astype(np.int64)
    k0 = np.where(valid, k0, 0).astype(np.int64)
    fx = ix - i0
    fy = iy - j0
    fz = iz - k0
    d = data
    val = (
        d[i0, j0, k0] * (1 - fx) * (1 - fy) * (1 - fz)
        + d[i0 + 1, j0, k0] * fx * (1 - fy) * (1 - fz)
        + d[i0, j0 + 1, k0] * (1 - fx) * fy * (1 - fz)
        + d[i0, j0, k0 + 1] * (1 - fx) * (1 - fy) * fz
        + d[i0 + 1, j0 + 1, k0] * fx * fy * (1 - fz)
        + d[i0 + 1, j0, k0 + 1] * fx * (1 - fy) * fz
        + d[i0, j0 + 1, k0 + 1] * (1 - fx) * fy * fz
        + d[i0 + 1, j0 + 1, k0 + 1] * fx * fy * fz
    )
    return np.where(valid, val, 0.0)


def k1_batch_force(positions, charges, data, origin, sp, alpha, is_born):
    """Per-(trajectory, atom) force and energy of one grid.

    positions (..., 3) and charges (...) broadcast together; atoms with
    |q| < 1e-9 give exactly zero (gpu_batch_engine.py:90).  The gradient is the
    central difference of trilinear interpolants at +-sp/2 (:111-114);
    F = coeff * grad, E = e_coeff * phi with coeff = -q (elec) or -alpha q^2
    (Born) (:116-121).
    """
    data = np.asarray(data, dtype=np.float64)
    origin = np.asarray(origin, dtype=np.float64)
    sp = np.asarray(sp, dtype=np.float64)
    inv_sp = 1.0 / sp
    q = np.asarray(charges, dtype=np.float64)
    px, py, pz = positions[..., 0], positions[..., 1], positions[..., 2]
    h0, h1, h2 = sp[0] * 0.5, sp[1] * 0.5, sp[2] * 0.5
    gx = (_interp(data, origin, inv_sp, px + h0, py, pz) - _interp(data, origin, inv_sp, px - h0, py, pz)) / (2 * h0)
    gy = (_interp(data, origin, inv_sp, px, py + h1, pz) - _interp(data, origin, inv_sp, px, py - h1, pz)) / (2 * h1)
    gz = (_interp(data, origin, inv_sp, px, py, pz + h2) - _interp(data, origin, inv_sp, px, py, pz - h2)) / (2 * h2)
    phi = _interp(data, origin, inv_sp, px, py, pz)
    if is_born:
        coeff = -alpha * q * q
        e_coeff = alpha * q * q
    else:
        coeff = -q
        e_coeff = q
    skip = np.abs(q) < 1e-9
    forces = np.stack([coeff * gx, coeff * gy, coeff * gz], axis=-1)
    forces = np.where(skip[..., None], 0.0, forces)
    energies = np.where(skip, 0.0, e_coeff * phi)
    return forces, energies


def k1_batch_force_flat(positions, charges, grid_data, origin, inv_sp, sp, alpha, is_born,
                        nx, ny, nz, n_traj, n_atoms, atom_forces, atom_energies):
    """Same as ``k1_batch_force`` with the kernel's flat argument list (:67-79).

    Writes into ``atom_forces`` (n_traj*n_atoms*3) and ``atom_energies``
    (n_traj*n_atoms) in place, like the CUDA kernel does.
    """
    n_traj, n_atoms = int(n_traj), int(n_atoms)
    data = np.asarray(grid_data).reshape(int(nx), int(ny), int(nz))
    pos = np.asarray(positions).reshape(n_traj, n_atoms, 3)
    q = np.asarray(charges).reshape(n_traj, n_atoms)
    f, e = k1_batch_force(pos, q, data, np.asarray(origin), np.asarray(sp), float(alpha), bool(is_born))
    atom_forces[...] = f.reshape(-1)
    atom_energies[...] = e.reshape(-1)


# --------------------------------------------------------------------------
# Grids
# --------------------------------------------------------------------------
@dataclass
class OracleGrid:
    data: np.ndarray  # (nx, ny, nz) float64, z fastest
    origin: np.ndarray
    sp: np.ndarray

    @property
    def lo(self):
        return self.origin + GRID_MARGIN * self.sp

    @property
    def hi(self):
        return self.origin + (np.array(self.data.shape) - 1 - GRID_MARGIN) * self.sp

    @classmethod
    def from_dx(cls, g):
        """From any object with ``.data`` (nx,ny,nz), ``.origin`` and ``.delta`` (3x3)."""
        delta = np.asarray(g.delta, dtype=np.float64)
        return cls(np.asarray(g.data, dtype=np.float64), np.asarray(g.origin, dtype=np.float64),
                   np.array([delta[i, i] for i in range(3)]))


def sort_finest_first(grids):
    """``sorted(grids, key=delta[0,0])`` (gpu_batch_engine.py:259)."""
    return sorted(grids, key=lambda g: float(g.sp[0]))


def in_box(positions, grid):
    """Strict in-grid test on all three axes (gpu_batch_engine.py:317-319)."""
    return np.all(positions > grid.lo, axis=-1) & np.all(positions < grid.hi, axis=-1)


# --------------------------------------------------------------------------
# Far field
# --------------------------------------------------------------------------
@dataclass
class FarField:
    """Receptor far-field parameters (gpu_batch_engine.py:162-175)."""

    receptor_charge: float
    debye: float
    sdie: float
    dipole: np.ndarray | None = None  # (3,)  MultipoleExpansion.dipole
    quadrupole: np.ndarray | None = None  # (3,3) MultipoleExpansion.quadrupole
    four_pi_eps: float | None = None  # MultipoleExpansion.four_pi_eps

    @property
    def V_factor(self):
        eps_s = self.sdie * EPS0
        return self.receptor_charge / (4.0 * math.pi * eps_s) if eps_s > 0 else 0.0

    @property
    def has_yukawa(self):
        return abs(self.receptor_charge) > 1e-9 and self.debye > 0


def multipole_moments(positions, charges):
    """Dipole and traceless quadrupole 1/2 sum q (3 r r - r^2 I) (multipole_farfield.py:90-107)."""
    positions = np.asarray(positions, dtype=np.float64)
    charges = np.asarray(charges, dtype=np.float64)
    dipole = np.sum(charges[:, None] * positions, axis=0)
    r2 = np.sum(positions ** 2, axis=1)
    quad = np.zeros((3, 3))
    for a in range(3):
        for b in range(3):
            quad[a, b] = np.sum(charges * (3.0 * positions[:, a] * positions[:, b] - (r2 if a == b else 0.0)))
    return dipole, 0.5 * quad


def yukawa_forces(positions, charges, ff: FarField, mask=None):
    """Per-atom far-field force/energy, radial derivative only (gpu_batch_engine.py:393-472).

    Returns per-atom arrays (forces (...,3), energies (...)); the reference sums
    them over atoms afterwards.
    """
    debye = ff.debye
    r_mag = np.linalg.norm(positions, axis=-1)
    safe_r = np.maximum(r_mag, 1.0)
    exp_term = np.exp(-safe_r / debye)
    r_hat = positions / safe_r[..., None]
    V_fac = ff.V_factor
    phi = V_fac * exp_term / safe_r
    dphi_dr = V_fac * exp_term * (-1.0 / safe_r ** 2 - 1.0 / (safe_r * debye))
    if ff.dipole is not None:
        p = np.asarray(ff.dipole, dtype=np.float64)
        Q = np.asarray(ff.quadrupole, dtype=np.float64)
        fpe = ff.four_pi_eps
        lam = debye
        p_dot_r = np.sum(r_hat * p, axis=-1)
        if float(np.linalg.norm(p)) > 1e-9:
            phi = phi + p_dot_r / (fpe * safe_r ** 2) * (1.0 + safe_r / lam) * exp_term
            dphi_dr = dphi_dr + p_dot_r / fpe * exp_term * (
                -2.0 / safe_r ** 3 - 2.0 / (safe_r ** 2 * lam) - 1.0 / (safe_r * lam ** 2))
        if float(np.linalg.norm(Q)) > 1e-9:
            rQr = np.sum(r_hat * np.einsum("ij,...j->...i", Q, r_hat), axis=-1)
            phi = phi + rQr / (fpe * safe_r ** 3) * (1.0 + safe_r / lam + safe_r ** 2 / (3.0 * lam ** 2)) * exp_term
            dphi_dr = dphi_dr + rQr / fpe * exp_term * (
                -3.0 / safe_r ** 4 - 3.0 / (safe_r ** 3 * lam) - 1.0 / (safe_r ** 2 * lam ** 2)
                - 1.0 / (3.0 * safe_r * lam ** 3))
    grad_phi = dphi_dr[..., None] * r_hat
    q = np.asarray(charges, dtype=np.float64)
    atom_forces = -q[..., None] * grad_phi
    atom_energies = q * phi
    if mask is not None:
        atom_forces = atom_forces * mask[..., None].astype(np.float64)
        atom_energies = atom_energies * mask.astype(np.float64)
    return atom_forces, atom_energies


# --------------------------------------------------------------------------
# _eval_batch
# --------------------------------------------------------------------------
def eval_batch_atoms(positions, charges, grids, alpha, is_born, ff: FarField | None):
    """Per-atom forces/energies of ``_eval_batch`` (gpu_batch_engine.py:289-391).

    Finest grid first; an atom strictly inside a grid's margin box that no finer
    grid claimed is evaluated on it (masked atoms get zero charge, :320-327).
    For electrostatics with a Yukawa far-field, unassigned atoms use the
    far-field (:358-366).  With no grids at all, elec uses the far-field for
    every atom (:304-309).
    """
    return eval_batch(positions, charges, grids, alpha, is_born, ff)[:2]


def eval_batch(positions, charges, grids, alpha, is_born, ff: FarField | None):
    """``eval_batch_atoms`` plus the per-trajectory totals summed in the reference's order
    (each grid's atoms, then the far-field atoms; gpu_batch_engine.py:302-366)."""
    N, A, _ = positions.shape
    atom_f = np.zeros((N, A, 3))
    atom_e = np.zeros((N, A))
    tot_f = np.zeros((N, 3))
    tot_e = np.zeros((N,))
    use_ff = (not is_born) and ff is not None and ff.has_yukawa
    if not grids:
        if use_ff:
            f, e = yukawa_forces(positions, np.broadcast_to(charges, (N, A)), ff)
            atom_f += f
            atom_e += e
            tot_f += f.sum(axis=1)
            tot_e += e.sum(axis=1)
        return atom_f, atom_e, tot_f, tot_e
    assigned = np.zeros((N, A), dtype=bool)
    q_full = np.broadcast_to(np.asarray(charges, dtype=np.float64), (N, A))
    for g in grids:
        to_process = in_box(positions, g) & ~assigned
        assigned |= to_process
        if not np.any(to_process):
            continue
        pos_masked = np.where(to_process[..., None], positions, 0.0)
        chg_masked = np.where(to_process, q_full, 0.0)
        f, e = k1_batch_force(pos_masked, chg_masked, g.data, g.origin, g.sp, alpha, is_born)
        atom_f += f
        atom_e += e
        tot_f += f.sum(axis=1)
        tot_e += e.sum(axis=1)
    if use_ff:
        not_assigned = ~assigned
        if np.any(not_assigned):
            f, e = yukawa_forces(positions, q_full, ff, mask=not_assigned)
            atom_f += f
            atom_e += e
            tot_f += f.sum(axis=1)
            tot_e += e.sum(axis=1)
    return atom_f, atom_e, tot_f, tot_e


def born_reverse_atoms(R, centroids, rec_pos, rec_q, lig_born_grid, alpha, chunk_skip=True):
    """Per-receptor-atom reverse-Born forces in the lab frame (gpu_batch_engine.py:607-657).

    Receptor atoms are moved into the ligand frame, R^T (x_rec - c), evaluated on
    the ligand Born grid, rotated back with R.  Returns the force ON THE
    RECEPTOR atoms (N, Nr, 3); the force on the ligand is minus their sum.

    ``chunk_skip`` applies the reference's whole-batch cull (:635-639): when
    min|c| - max|x_rec| exceeds the grid's x half-width, the batch gets zero.
    The reference applies it per memory chunk; here the batch is one chunk.
    """
    return born_reverse(R, centroids, rec_pos, rec_q, lig_born_grid, alpha, chunk_skip)[0]


def born_reverse(R, centroids, rec_pos, rec_q, lig_born_grid, alpha, chunk_skip=True):
    """(per-receptor-atom lab forces, force on the ligand summed as the reference sums it:
    minus R times the ligand-frame total, gpu_batch_engine.py:646-656)."""
    N = R.shape[0]
    out = np.zeros((N, rec_pos.shape[0], 3))
    g = lig_born_grid
    lig_grid_radius = float(max(abs(g.lo[0]), abs(g.hi[0])))
    if chunk_skip:
        r_cen = np.linalg.norm(centroids, axis=1)
        rec_max_r = float(np.linalg.norm(rec_pos, axis=1).max())
        if float(r_cen.min()) - rec_max_r > lig_grid_radius:
            return out, np.zeros((N, 3))
    rec_pos_rel = rec_pos[None, :, :] - centroids[:, None, :]
    R_T = np.swapaxes(R, 1, 2)
    rec_in_lig = np.einsum("nij,nkj->nki", R_T, rec_pos_rel)
    f_lig, _, f_lig_tot, _ = eval_batch(rec_in_lig, rec_q, [g], alpha, True, None)
    out[...] = np.einsum("nij,nkj->nki", R, f_lig)
    return out, -np.einsum("nij,nj->ni", R, f_lig_tot)


WCA_EPSILON = 0.17  # kBT, gpu_batch_engine.py:239
WCA_CUTOFF = 1.122462  # in units of sigma, gpu_batch_engine.py:512


def wca_activation(rec_radii, lig_radii):
    """Centroid distance below which the contact term is evaluated (gpu_batch_engine.py:241-242)."""
    return (float(np.max(rec_radii)) + float(np.max(lig_radii))) * 2.5


def wca_forces(lig_positions, centroids, rec_pos, rec_radii, lig_radii, eps=WCA_EPSILON, activation=None):
    """WCA contact forces on the ligand atoms (gpu_batch_engine.py:474-529).

    Every (ligand, receptor) atom pair with sigma = r_lig + r_rec and
    r = sqrt(max(r^2, 1e-6)) < 1.122462 sigma contributes
    eps (12 (sigma/r)^12 - 6 (sigma/r)^6) / r^2 * (x_lig - x_rec) / r, with the
    unclamped r^2 as divisor.  Trajectories whose centroid is at or beyond the
    activation radius get zero.  Returns per-ligand-atom forces (N, A, 3) and
    their totals (N, 3).
    """
    lig_positions = np.asarray(lig_positions, dtype=np.float64)
    N, A, _ = lig_positions.shape
    rec_pos = np.asarray(rec_pos, dtype=np.float64)
    rr = np.asarray(rec_radii, dtype=np.float64)
    rl = np.asarray(lig_radii, dtype=np.float64)
    act = wca_activation(rr, rl) if activation is None else float(activation)
    f_atoms = np.zeros((N, A, 3))
    active = np.linalg.norm(np.asarray(centroids, dtype=np.float64), axis=1) < act
    sig = rl[:, None] + rr[None, :]
    for n in np.flatnonzero(active):
        diff = lig_positions[n][:, None, :] - rec_pos[None, :, :]
        r2 = (diff * diff).sum(axis=2)
        r = np.sqrt(np.maximum(r2, 1e-6))
        in_range = r < WCA_CUTOFF * sig
        sr = sig / r
        sr2 = sr * sr
        sr6 = sr2 * sr2 * sr2
        sr12 = sr6 * sr6
        with np.errstate(divide="ignore", invalid="ignore"):
            f_mag = np.where(in_range, eps * (12.0 * sr12 - 6.0 * sr6) / r2, 0.0)
        f_atoms[n] = (f_mag[:, :, None] * diff / r[:, :, None]).sum(axis=1)
    return f_atoms, f_atoms.sum(axis=1)


# --------------------------------------------------------------------------
# Engine
# --------------------------------------------------------------------------
class OracleForceEngine:
    """FP64 restatement of ``GPUBatchForceEngine`` (gpu_batch_engine.py:126-657).

    Grids are ``OracleGrid``; ``elec_grids``/``born_grids``/``lig_born_grids``
    follow the reference's selection rules.  ``__call__`` has the reference
    signature and returns (forces, torques, energies); ``torque_mode`` is
    ``"zero"`` (the reference GPU path) or ``"centroid"`` (torque about the
    centroid argument, from every per-atom force including the reaction of the
    reverse-Born forces, which act at the receptor atoms).
    """

    def __init__(self, elec_grids, born_grids, alpha=0.07957747, farfield: FarField | None = None,
                 lig_born_grids=None, rec_positions=None, rec_charges=None, born_chunk_skip=True,
                 rec_radii=None, lig_radii=None, use_lj=False):
        self.alpha = float(alpha)
        self.ff = farfield
        self.elec = sort_finest_first(list(elec_grids or []))
        self.born = sort_finest_first(list(born_grids or []))
        if self.ff is not None and self.ff.has_yukawa and len(self.elec) > 1:
            self.elec = [self.elec[0]]
        if len(self.born) > 1:
            self.born = [self.born[0]]
        self.lig_born = []
        self.rec_pos = None
        self.rec_q = None
        if lig_born_grids and rec_positions is not None and rec_charges is not None:
            self.lig_born = sort_finest_first(list(lig_born_grids))[:1]
            self.rec_pos = np.asarray(rec_positions, dtype=np.float64)
            self.rec_q = np.asarray(rec_charges, dtype=np.float64)
        self.born_chunk_skip = born_chunk_skip
        self.wca = None  # (receptor positions, receptor radii, ligand radii): gpu_batch_engine.py:233-246
        if use_lj and rec_radii is not None and lig_radii is not None:
            self.wca = (np.asarray(rec_positions, dtype=np.float64), np.asarray(rec_radii, dtype=np.float64),
                        np.asarray(lig_radii, dtype=np.float64))

    def atoms(self, lig_positions, lig_charges, R_matrices=None, centroids=None):
        """Per-atom terms and totals: (direct ligand forces (N,A,3), energies (N,A), receptor
        reverse-Born forces (N,Nr,3) or None, net force (N,3), energy (N,)).  The totals are
        summed in the reference's order: elec, Born direction 1, Born direction 2, WCA contact (:556-602)."""
        N, A, _ = lig_positions.shape
        f = np.zeros((N, A, 3))
        e = np.zeros((N, A))
        forces = np.zeros((N, 3))
        energies = np.zeros((N,))
        ff = self.ff
        if self.elec:
            f1, e1, tf, te = eval_batch(lig_positions, lig_charges, self.elec, 0.0, False, ff)
            f += f1
            e += e1
            forces += tf
            energies += te
        elif ff is not None and ff.has_yukawa:
            f1, e1 = yukawa_forces(lig_positions, np.broadcast_to(lig_charges, (N, A)), ff)
            f += f1
            e += e1
            forces += f1.sum(axis=1)
            energies += e1.sum(axis=1)
        if self.born:
            f2, e2, tf, te = eval_batch(lig_positions, lig_charges, self.born, self.alpha, True, None)
            f += f2
            e += e2
            forces += tf
            energies += te
        f_rec = None
        if (self.lig_born and self.rec_pos is not None and R_matrices is not None
                and centroids is not None and self.alpha > 1e-12):
            f_rec, f2_tot = born_reverse(np.asarray(R_matrices), np.asarray(centroids), self.rec_pos, self.rec_q,
                                         self.lig_born[0], self.alpha, self.born_chunk_skip)
            forces += f2_tot
        if self.wca is not None:
            fw, tw = wca_forces(lig_positions, centroids, *self.wca)
            f += fw
            forces += tw
        return f, e, f_rec, forces, energies

    def __call__(self, lig_positions, lig_charges, R_matrices=None, centroids=None, torque_mode="zero",
                 return_scale=False):
        lig_positions = np.asarray(lig_positions, dtype=np.float64)
        f_atoms, e_atoms, f_rec, forces, energies = self.atoms(lig_positions, lig_charges, R_matrices, centroids)
        scale = np.linalg.norm(f_atoms, axis=2).sum(axis=1)
        if f_rec is not None:
            scale = scale + np.linalg.norm(f_rec, axis=2).sum(axis=1)
        torques = np.zeros_like(forces)
        if torque_mode == "centroid":
            c = np.asarray(centroids, dtype=np.float64)
            torques = np.cross(lig_positions - c[:, None, :], f_atoms).sum(axis=1)
            if f_rec is not None:
                torques = torques - np.cross(self.rec_pos[None, :, :] - c[:, None, :], f_rec).sum(axis=1)
        elif torque_mode != "zero":
            raise ValueError(f"unknown torque_mode {torque_mode!r}")
        if return_scale:
            return forces, torques, energies, scale
        return forces, torques, energies


def force_error(F, F_ref, scale_ref):
    """Per-trajectory force error ||F - F_ref|| / max(||F_ref||, 1e-3 * sum_i ||F_ref,i||).

    The denominator keeps the metric finite for near-neutral ligands whose net
    force cancels between atoms.
    """
    num = np.linalg.norm(np.asarray(F) - np.asarray(F_ref), axis=-1)
    den = np.maximum(np.linalg.norm(F_ref, axis=-1), 1e-3 * np.asarray(scale_ref))
    den = np.where(den > 0, den, 1.0)
    return num / den
