"""Seeded synthetic receptor/ligand systems with the shapes of the benchmark configs.

No benchmark structure ships with this project (the reference's examples need
APBS and AmberTools), so each config is restated as seeded synthetic input:
atoms placed uniformly in a ball with a minimum separation, Gaussian charges
shifted to a stated net charge, and FP32 potential grids filled by direct
Debye-Hueckel sums (Born grids by the unscreened Coulomb sum with dielectric
4, mirroring an APBS Born run with pdie 4, sdie 1, no ions).  Molecules are
centred on their centroid and carry a zero-charge ghost (GHO) atom at the
centroid, as the reference pipeline appends one to each PQR.

``config1`` .. ``config3`` follow the five benchmark configurations; the
``scale`` arguments shrink atom counts and grids for CPU-sized tests while
keeping the same construction.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .dx import DXGrid
from . import structures as st

EPS0 = 0.000142
ALPHA_BORN = 0.07957747


def debye_length(ionic_strength_M: float) -> float:
    """Debye length of a monovalent salt in water at 298 K: 3.04 A / sqrt(I)."""
    return 3.04 / math.sqrt(ionic_strength_M)


def ball_atoms(n: int, radius: float, min_sep: float, rng: np.random.Generator) -> np.ndarray:
    """n points uniform in a ball, rejection-sampled to a minimum pairwise separation."""
    out = np.zeros((0, 3))
    tries = 0
    while out.shape[0] < n:
        tries += 1
        if tries > 200:
            raise RuntimeError("could not place atoms; ball too dense")
        m = 4 * (n - out.shape[0]) + 16
        cand = rng.uniform(-radius, radius, size=(m, 3))
        cand = cand[np.einsum("ij,ij->i", cand, cand) <= radius * radius]
        for p in cand:
            if out.shape[0] >= n:
                break
            if out.shape[0] == 0 or np.min(np.sum((out - p) ** 2, axis=1)) >= min_sep * min_sep:
                out = np.vstack([out, p])
    return out


def net_charges(n: int, sigma: float, net: float, rng: np.random.Generator) -> np.ndarray:
    q = rng.normal(0.0, sigma, size=n)
    return q + (net - q.sum()) / n


def grid_axes(dims, spacing, centre=(0.0, 0.0, 0.0)):
    dims = np.asarray(dims, dtype=int)
    sp = np.full(3, float(spacing)) if np.ndim(spacing) == 0 else np.asarray(spacing, dtype=float)
    origin = np.asarray(centre, dtype=float) - 0.5 * (dims - 1) * sp
    return origin, sp


def _grid_points(dims, origin, sp):
    ax = [origin[i] + sp[i] * np.arange(dims[i]) for i in range(3)]
    return ax


def fill_sum_grid(positions, charges, radii, dims, spacing, debye, eps, centre=(0, 0, 0), device=None):
    """phi(x) = sum_j q_j exp(-d/lambda) / (4 pi eps d), d = max(|x - r_j|, radius_j).

    ``debye`` = 0 or inf gives the unscreened sum.  Returns a float32 DXGrid.
    With ``device`` (a torch device string) the sum runs in torch FP64 there.
    """
    dims = tuple(int(d) for d in dims)
    origin, sp = grid_axes(dims, spacing, centre)
    pos = np.asarray(positions, dtype=np.float64)
    q = np.asarray(charges, dtype=np.float64)
    rad = np.maximum(np.asarray(radii, dtype=np.float64), 1e-3)
    keep = np.abs(q) > 0
    pos, q, rad = pos[keep], q[keep], rad[keep]
    inv_lam = 0.0 if (not debye or not np.isfinite(debye)) else 1.0 / debye
    pref = 1.0 / (4.0 * math.pi * eps)
    ax = _grid_points(dims, origin, sp)
    if device is not None:
        import torch

        dev = torch.device(device)
        tpos = torch.tensor(pos, device=dev)
        tq = torch.tensor(q, device=dev)
        trad = torch.tensor(rad, device=dev)
        gx, gy, gz = (torch.tensor(a, device=dev) for a in ax)
        out = torch.empty(dims, dtype=torch.float32, device=dev)
        yz = torch.stack(torch.meshgrid(gy, gz, indexing="ij"), dim=-1).reshape(-1, 2)
        for i in range(dims[0]):
            pts = torch.cat([gx[i].expand(yz.shape[0], 1), yz], dim=1)
            for c0 in range(0, pts.shape[0], 8192):
                p = pts[c0:c0 + 8192]
                d = torch.cdist(p, tpos)
                d = torch.maximum(d, trad[None, :])
                v = (tq[None, :] * torch.exp(-d * inv_lam) / d).sum(dim=1) * pref
                out[i].view(-1)[c0:c0 + p.shape[0]] = v.to(torch.float32)
        data = out.cpu().numpy()
    else:
        data = np.empty(dims, dtype=np.float32)
        yy, zz = np.meshgrid(ax[1], ax[2], indexing="ij")
        yz = np.stack([yy.ravel(), zz.ravel()], axis=1)
        for i in range(dims[0]):
            acc = np.zeros(yz.shape[0])
            for c0 in range(0, len(q), 256):
                pp = pos[c0:c0 + 256]
                d = np.sqrt((ax[0][i] - pp[None, :, 0]) ** 2 + (yz[:, 0:1] - pp[None, :, 1]) ** 2
                            + (yz[:, 1:2] - pp[None, :, 2]) ** 2)
                d = np.maximum(d, rad[None, c0:c0 + 256])
                acc += (q[None, c0:c0 + 256] * np.exp(-d * inv_lam) / d).sum(axis=1)
            data[i] = (acc * pref).reshape(dims[1], dims[2]).astype(np.float32)
    return DXGrid(origin, np.diag(sp), data)


def sphere_dh_grid(Q, a, dims, spacing, debye, eps):
    """Debye-Hueckel potential of a charged sphere: Q e^{k(a-r)} / (4 pi eps r (1 + k a)), phi(a) inside."""
    origin, sp = grid_axes(dims, spacing)
    ax = _grid_points(dims, origin, sp)
    X, Y, Z = np.meshgrid(*ax, indexing="ij")
    r = np.maximum(np.sqrt(X * X + Y * Y + Z * Z), a)
    k = 1.0 / debye
    phi = Q * np.exp(k * (a - r)) / (4.0 * math.pi * eps * r * (1.0 + k * a))
    return DXGrid(origin, np.diag(sp), phi.astype(np.float32))


@dataclass
class BDSystem:
    """Everything one benchmark configuration needs, in reference units (A, ps, kBT, e)."""

    name: str
    rec_pos: np.ndarray
    rec_q: np.ndarray
    rec_r: np.ndarray
    lig_pos: np.ndarray
    lig_q: np.ndarray
    lig_r: np.ndarray
    elec_grids: list
    born_grids: list
    lig_born_grids: list
    pairs: list  # (rec_idx, lig_idx, cutoff)
    n_needed: int
    r_start: float
    r_escape: float
    r_hydro_rec: float
    r_hydro_lig: float
    debye: float
    sdie: float = 78.5
    eta: float = 0.89e-3
    temperature: float = 298.15
    alpha: float = ALPHA_BORN
    max_dt: float = 0.0
    hi: bool = False
    overlap: bool = True
    multipole: bool = True
    n_traj: int = 1000
    seed: int = 20261203
    max_steps: int = 1_000_000
    meta: dict = field(default_factory=dict)

    # reference-style objects -------------------------------------------------
    def molecules(self):
        return (st.Molecule.from_arrays("receptor", self.rec_pos, self.rec_q, self.rec_r),
                st.Molecule.from_arrays("ligand", self.lig_pos, self.lig_q, self.lig_r))

    def mobility(self):
        return st.MobilityTensor.from_radii(self.r_hydro_rec, self.r_hydro_lig, eta=self.eta, T=self.temperature)

    def pathway_set(self):
        pairs = [st.ContactPair(int(a), int(b), float(c)) for a, b, c in self.pairs]
        crit = st.ReactionCriteria(name="stage_0", pairs=pairs, n_needed=self.n_needed)
        return st.PathwaySet([st.ReactionInterface(name="stage_0", criteria=crit)])

    def params(self, n_traj=None, seed=None, max_steps=None):
        p = st.NAMParameters(n_trajectories=int(n_traj or self.n_traj), max_steps=int(max_steps or self.max_steps),
                             r_start=self.r_start, r_escape=self.r_escape, seed=int(seed or self.seed),
                             hydrodynamic_interactions=self.hi)
        p.max_dt = self.max_dt
        p.checkpoint_interval = 0
        p.convergence_interval = 10
        p._kT_scale = self.temperature / 298.15
        p._overlap_check = self.overlap
        return p

    def multipole_moments(self):
        q = np.asarray(self.rec_q, dtype=float)
        pos = np.asarray(self.rec_pos, dtype=float)
        dip = np.sum(q[:, None] * pos, axis=0)
        r2 = np.sum(pos ** 2, axis=1)
        quad = 0.5 * (3.0 * np.einsum("i,ia,ib->ab", q, pos, pos) - np.sum(q * r2) * np.eye(3))
        return dip, quad, 4.0 * math.pi * (self.sdie * EPS0)

    def engine_kwargs(self):
        return dict(elec_grids=self.elec_grids, born_grids=self.born_grids, alpha=self.alpha,
                    receptor_charge=float(np.sum(self.rec_q)), debye_length=self.debye, sdie=self.sdie,
                    lig_born_grids=self.lig_born_grids or None, rec_positions=self.rec_pos, rec_charges=self.rec_q)


def _with_gho(pos, q, r):
    pos = np.asarray(pos, dtype=float)
    pos = pos - pos.mean(axis=0)
    return (np.vstack([pos, np.zeros((1, 3))]), np.concatenate([q, [0.0]]), np.concatenate([r, [0.0]]))


def config1(n_traj=100_000, grid_dims=129, spacing=1.0, seed=20261203):
    """Two charged spheres: +5 e (a = 20 A) at the origin, -5 e ligand (a = 5 A); no Born, no HI."""
    lam = debye_length(0.15)
    sdie = 78.5
    eps = sdie * EPS0
    rec_pos, rec_q, rec_r = _with_gho(np.zeros((1, 3)), np.array([5.0]), np.array([20.0]))
    lig_pos, lig_q, lig_r = _with_gho(np.zeros((1, 3)), np.array([-5.0]), np.array([5.0]))
    g = sphere_dh_grid(5.0, 20.0, (grid_dims,) * 3, spacing, lam, eps)
    return BDSystem("config1_two_spheres", rec_pos, rec_q, rec_r, lig_pos, lig_q, lig_r,
                    elec_grids=[g], born_grids=[], lig_born_grids=[], pairs=[(0, 0, 26.0)], n_needed=1,
                    r_start=50.0, r_escape=100.0, r_hydro_rec=20.0, r_hydro_lig=5.0, debye=lam, sdie=sdie,
                    alpha=0.0, hi=False, overlap=False, n_traj=n_traj, seed=seed)


def _protein(n, radius, net, sigma, seed):
    rng = np.random.default_rng(seed)
    pos = ball_atoms(n, radius, 1.2, rng)
    q = net_charges(n, sigma, net, rng)
    r = rng.uniform(1.2, 2.0, size=n)
    return _with_gho(pos, q, r)


def _pole_atoms(pos, n, direction):
    d = np.asarray(direction, dtype=float)
    tgt = d * np.max(np.linalg.norm(pos, axis=1))
    return list(np.argsort(np.linalg.norm(pos[:-1] - tgt, axis=1))[:n])


def config2(n_traj=1_000_000, scale=1.0, device=None, seed=20261203):
    """Protein (3200 atoms, 22 A ball, +8 e) + small ligand (18 atoms, 4 A ball, +1 e).

    ``scale`` < 1 shrinks the receptor (atoms ~ scale^3, radius ~ scale) and
    the grids for CPU tests.  Nested elec grids (fine + coarse, the coarse one
    dropped by the engine as the reference does), Born grids on the same
    lattices, and a ligand Born grid for the reverse direction.
    """
    lam = debye_length(0.15)
    sdie = 78.5
    n_rec = max(16, int(round(3200 * scale ** 3)))
    R_rec = 22.0 * scale
    rec_pos, rec_q, rec_r = _protein(n_rec, R_rec, 8.0 * min(1.0, scale ** 2), 0.35, 2001)
    lig_pos, lig_q, lig_r = _protein(18, 4.0, 1.0, 0.35, 2002)
    fine = max(33, int(round(192 * scale)) | 1)
    coarse = max(17, int(round(128 * scale)) | 1)
    eps_e, eps_b = sdie * EPS0, 4.0 * EPS0
    elec = [fill_sum_grid(rec_pos, rec_q, rec_r, (fine,) * 3, 0.5, lam, eps_e, device=device),
            fill_sum_grid(rec_pos, rec_q, rec_r, (coarse,) * 3, 2.0, lam, eps_e, device=device)]
    born = [fill_sum_grid(rec_pos, rec_q, rec_r, (fine,) * 3, 0.5, 0, eps_b, device=device),
            fill_sum_grid(rec_pos, rec_q, rec_r, (coarse,) * 3, 2.0, 0, eps_b, device=device)]
    lig_born = [fill_sum_grid(lig_pos, lig_q, lig_r, (65,) * 3, 0.5, 0, eps_b, device=device)]
    rec_idx = _pole_atoms(rec_pos, 3, (1, 0, 0))
    pairs = [(int(rec_idx[i]), i, 4.5) for i in range(3)]
    r_h_rec = float(np.max(np.linalg.norm(rec_pos, axis=1)) + 1.4)
    r_h_lig = float(np.max(np.linalg.norm(lig_pos, axis=1)) + 1.4)
    b = 60.0 * max(scale, 0.5)
    return BDSystem(f"config2_protein_ligand_s{scale:g}", rec_pos, rec_q, rec_r, lig_pos, lig_q, lig_r,
                    elec, born, lig_born, pairs, 2, r_start=b, r_escape=2 * b, r_hydro_rec=r_h_rec,
                    r_hydro_lig=r_h_lig, debye=lam, sdie=sdie, max_dt=20.0, hi=False, overlap=True,
                    n_traj=n_traj, seed=seed)


def config3(n_traj=10_000_000, scale=1.0, device=None, seed=20261203):
    """Protein-protein pair: 1700-atom receptor (17 A, +2 e) and 1400-atom ligand (16 A, -6 e).

    Bidirectional Born, hydrodynamic interactions, overlap rejection, all grids
    161^3 at 0.6 A (scaled down for tests).  Reaction: 4 pairs between the
    receptor atoms nearest its +x pole and the ligand atoms nearest its -x pole.
    """
    lam = debye_length(0.15)
    sdie = 78.5
    n_rec = max(16, int(round(1700 * scale ** 3)))
    n_lig = max(16, int(round(1400 * scale ** 3)))
    rec_pos, rec_q, rec_r = _protein(n_rec, 17.0 * scale, 2.0, 0.4, 3001)
    lig_pos, lig_q, lig_r = _protein(n_lig, 16.0 * scale, -6.0, 0.4, 3002)
    n = max(33, int(round(160 * scale)) | 1)
    eps_e, eps_b = sdie * EPS0, 4.0 * EPS0
    elec = [fill_sum_grid(rec_pos, rec_q, rec_r, (n,) * 3, 0.6, lam, eps_e, device=device)]
    born = [fill_sum_grid(rec_pos, rec_q, rec_r, (n,) * 3, 0.6, 0, eps_b, device=device)]
    lig_born = [fill_sum_grid(lig_pos, lig_q, lig_r, (n,) * 3, 0.6, 0, eps_b, device=device)]
    rec_idx = _pole_atoms(rec_pos, 4, (1, 0, 0))
    lig_idx = _pole_atoms(lig_pos, 4, (-1, 0, 0))
    pairs = [(int(a), int(b), 5.0) for a, b in zip(rec_idx, lig_idx)]
    b = 80.0 * max(scale, 0.5)
    return BDSystem(f"config3_protein_protein_s{scale:g}", rec_pos, rec_q, rec_r, lig_pos, lig_q, lig_r,
                    elec, born, lig_born, pairs, 3, r_start=b, r_escape=2 * b, r_hydro_rec=17.5 * scale,
                    r_hydro_lig=16.5 * scale, debye=lam, sdie=sdie, max_dt=100.0, hi=True, overlap=True,
                    n_traj=n_traj, seed=seed)


C5_DIMS = (97, 129, 161, 193, 225)


def config5(index, device=None, seed_base=5000, traj_scale=1.0):
    """System ``index`` of the heterogeneous batch (16 systems, seed 5000 + index).

    Receptor atoms log-uniform 500-8000, ligand atoms log-uniform 10-2000, at
    the atom density of config 2 (3200 atoms in a 22 A ball); charges N(0, 0.35)
    shifted to a net receptor charge of +2..+8 e and a ligand charge of -1..-4 e;
    radii U(1.2, 2.0).  Receptor elec and Born grids share one lattice with dims
    drawn from {97, 129, 161, 193, 225} at 0.5-1.0 A; the ligand Born grid spans
    the ligand plus 10 A at 0.5 A (at most 129^3).  Trajectories log-uniform
    1e4-1e6 (times ``traj_scale``), b-surface U(50, 90) A (at least contact +
    10 A), r_escape = 2b, max_dt 20 ps, no HI, overlap on.  Reaction: 3 pairs at
    the poles, cutoff 4.5 A, 2 needed.
    """
    rng = np.random.default_rng(seed_base + index)
    lam = debye_length(0.15)
    sdie = 78.5
    rho = 3200 / (4.0 / 3.0 * math.pi * 22.0 ** 3)
    n_rec = int(round(math.exp(rng.uniform(math.log(500), math.log(8000)))))
    n_lig = int(round(math.exp(rng.uniform(math.log(10), math.log(2000)))))
    R_rec = (3 * n_rec / (4 * math.pi * rho)) ** (1 / 3)
    R_lig = max(2.0, (3 * n_lig / (4 * math.pi * rho)) ** (1 / 3))
    q_rec = float(rng.integers(2, 9))
    q_lig = -float(rng.integers(1, 5))
    rec_pos, rec_q, rec_r = _protein(n_rec, R_rec, q_rec, 0.35, seed_base * 10 + 2 * index)
    lig_pos, lig_q, lig_r = _protein(n_lig, R_lig, q_lig, 0.35, seed_base * 10 + 2 * index + 1)
    dims = int(rng.choice(C5_DIMS))
    sp = float(rng.uniform(0.5, 1.0))
    eps_e, eps_b = sdie * EPS0, 4.0 * EPS0
    elec = [fill_sum_grid(rec_pos, rec_q, rec_r, (dims,) * 3, sp, lam, eps_e, device=device)]
    born = [fill_sum_grid(rec_pos, rec_q, rec_r, (dims,) * 3, sp, 0, eps_b, device=device)]
    ld = min(129, int(2 * (R_lig + 10.0) / 0.5) | 1)
    lig_born = [fill_sum_grid(lig_pos, lig_q, lig_r, (ld,) * 3, 0.5, 0, eps_b, device=device)]
    rec_idx = _pole_atoms(rec_pos, 3, (1, 0, 0))
    lig_idx = _pole_atoms(lig_pos, 3, (-1, 0, 0))
    pairs = [(int(a), int(b), 4.5) for a, b in zip(rec_idx, lig_idx)]
    b = max(float(rng.uniform(50.0, 90.0)), R_rec + R_lig + 10.0)
    n_traj = max(1, int(round(math.exp(rng.uniform(math.log(1e4), math.log(1e6))) * traj_scale)))
    return BDSystem(f"config5_{index:02d}", rec_pos, rec_q, rec_r, lig_pos, lig_q, lig_r, elec, born, lig_born,
                    pairs, 2, r_start=b, r_escape=2 * b, r_hydro_rec=R_rec + 1.4, r_hydro_lig=R_lig + 1.4,
                    debye=lam, sdie=sdie, max_dt=20.0, hi=False, overlap=True, n_traj=n_traj,
                    seed=20261203 + index,
                    meta={"n_rec": n_rec, "n_lig": n_lig, "grid": dims, "spacing": round(sp, 3), "b": round(b, 1)})
