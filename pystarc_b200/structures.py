"""Host-side mirror of the reference data types the batched stepper consumes.

The engine accepts either these classes or the reference's own (pystarc is
duck-typed): only the attributes and methods listed here are read.

* ``Atom`` / ``Molecule``          -- pystarc/structures/molecules.py:13-117
* ``ContactPair`` / ``ReactionCriteria`` -- pystarc/structures/molecules.py:185-240
* ``ReactionInterface`` / ``PathwaySet`` -- pystarc/pathways/reaction_interface.py:14-95
* ``NAMParameters``                -- pystarc/simulation/nam_simulator.py:80-106
* ``MobilityTensor``               -- pystarc/hydrodynamics/rotne_prager.py:127-215
* ``stokes_*``, ``rpy_offdiagonal`` -- rotne_prager.py:43-124 (Zuk et al. 2014)
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

KB_SI = 1.380649e-23
T_DEFAULT = 298.15
ETA_WATER = 1.002e-3
ANG_TO_M = 1.0e-10
PS_TO_S = 1.0e-12


@dataclass
class Atom:
    index: int = 0
    name: str = ""
    residue_name: str = ""
    residue_index: int = 0
    chain: str = "A"
    x: float = 0.0
    y: float = 0.0
    z: float = 0.0
    charge: float = 0.0
    radius: float = 1.5

    @property
    def position(self) -> np.ndarray:
        return np.array([self.x, self.y, self.z], dtype=float)


@dataclass
class Molecule:
    name: str = ""
    atoms: List[Atom] = field(default_factory=list)

    @classmethod
    def from_arrays(cls, name, positions, charges, radii=None):
        positions = np.asarray(positions, dtype=float)
        charges = np.asarray(charges, dtype=float)
        radii = np.full(len(charges), 1.5) if radii is None else np.asarray(radii, dtype=float)
        atoms = [Atom(index=i + 1, name="A", x=float(p[0]), y=float(p[1]), z=float(p[2]), charge=float(q),
                      radius=float(r)) for i, (p, q, r) in enumerate(zip(positions, charges, radii))]
        return cls(name, atoms)

    def centroid(self) -> np.ndarray:
        if not self.atoms:
            return np.zeros(3)
        return self.positions_array().mean(axis=0)

    def total_charge(self) -> float:
        return sum(a.charge for a in self.atoms)

    def positions_array(self) -> np.ndarray:
        return np.array([[a.x, a.y, a.z] for a in self.atoms], dtype=float).reshape(-1, 3)

    def charges_array(self) -> np.ndarray:
        return np.array([a.charge for a in self.atoms], dtype=float)

    def radii_array(self) -> np.ndarray:
        return np.array([a.radius for a in self.atoms], dtype=float)

    def __len__(self):
        return len(self.atoms)


@dataclass
class ContactPair:
    mol1_atom_index: int = 0
    mol2_atom_index: int = 0
    distance_cutoff: float = 5.0


@dataclass
class ReactionCriteria:
    name: str = "reaction"
    pairs: List[ContactPair] = field(default_factory=list)
    n_needed: int = -1
    state_before: Optional[str] = None
    state_after: Optional[str] = None


@dataclass
class ReactionInterface:
    name: str
    criteria: ReactionCriteria
    probability: float = 1.0
    state_before: Optional[str] = None
    state_after: Optional[str] = None


class PathwaySet:
    def __init__(self, reactions=None, first_state=None):
        self.reactions = list(reactions or [])
        self.first_state = first_state

    def __len__(self):
        return len(self.reactions)


@dataclass
class NAMParameters:
    n_trajectories: int = 1_000
    dt: float = 0.2
    dt_rxn: float = 0.05
    minimum_core_dt: float = 0.0
    minimum_core_reaction_dt: float = 0.0
    max_steps: int = 1_000_000
    r_start: float = 100.0
    r_escape: float = 0.0
    seed: Optional[int] = None
    n_threads: int = 1
    use_hard_sphere: bool = True
    hydrodynamic_interactions: bool = False
    verbose: bool = False

    def __post_init__(self):
        if self.r_escape == 0.0:
            self.r_escape = self.r_start * 1.1


def stokes_translational_diffusion(radius_ang, eta=ETA_WATER, T=T_DEFAULT):
    """D_t = kBT / (6 pi eta r) in A^2/ps."""
    r_m = radius_ang * ANG_TO_M
    return KB_SI * T / (6.0 * math.pi * eta * r_m) / (ANG_TO_M ** 2) * PS_TO_S


def stokes_rotational_diffusion(radius_ang, eta=ETA_WATER, T=T_DEFAULT):
    """D_r = kBT / (8 pi eta r^3) in rad^2/ps."""
    r_m = radius_ang * ANG_TO_M
    return KB_SI * T / (8.0 * math.pi * eta * r_m ** 3) * PS_TO_S


def rpy_offdiagonal(r_vec, a, b, D_a, D_b):
    """Zuk three-regime off-diagonal translational mobility (far / partial overlap / enclosed)."""
    r = float(np.linalg.norm(r_vec))
    if r < 1e-10:
        return np.zeros((3, 3))
    rhat = np.asarray(r_vec, dtype=float) / r
    a2, b2, r2 = a * a, b * b, r * r
    r3 = r2 * r
    if r > a + b:
        den = 8.0 * math.pi * r
        tt_I = (1.0 + (a2 + b2) / (3.0 * r2)) / den
        tt_uu = (1.0 - (a2 + b2) / r2) / den
    elif r > abs(a - b):
        den = 192.0 * math.pi * a * b * r3
        tt_I = (16.0 * r3 * (a + b) - ((a - b) ** 2 + 3.0 * r2) ** 2) / den
        tt_uu = 3.0 * ((a - b) ** 2 - r2) ** 2 / den
    else:
        tt_I = 1.0 / (6.0 * math.pi * max(a, b))
        tt_uu = 0.0
    kT_over_eta = math.sqrt(D_a * 6.0 * math.pi * a * D_b * 6.0 * math.pi * b)
    return kT_over_eta * (tt_I * np.eye(3) + tt_uu * np.outer(rhat, rhat))


class MobilityTensor:
    def __init__(self, D_trans1, D_rot1, D_trans2, D_rot2, radius1=0.0, radius2=0.0, use_rpy=True):
        self.D_trans1, self.D_rot1 = D_trans1, D_rot1
        self.D_trans2, self.D_rot2 = D_trans2, D_rot2
        self.radius1, self.radius2 = radius1, radius2
        self.use_rpy = use_rpy

    @classmethod
    def from_radii(cls, radius1, radius2, eta=ETA_WATER, T=T_DEFAULT, use_rpy=True):
        return cls(stokes_translational_diffusion(radius1, eta, T), stokes_rotational_diffusion(radius1, eta, T),
                   stokes_translational_diffusion(radius2, eta, T), stokes_rotational_diffusion(radius2, eta, T),
                   radius1, radius2, use_rpy)

    def relative_translational_diffusion(self, r_vec=None) -> float:
        D0 = self.D_trans1 + self.D_trans2
        if not self.use_rpy or r_vec is None or self.radius1 <= 0.0 or self.radius2 <= 0.0:
            return D0
        M12 = rpy_offdiagonal(r_vec, self.radius1, self.radius2, self.D_trans1, self.D_trans2)
        return max(D0 - (2.0 / 3.0) * float(np.trace(M12)), 1e-12)

    def relative_rotational_diffusion(self) -> float:
        return self.D_rot1 + self.D_rot2
