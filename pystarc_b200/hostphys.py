"""Host-side, once-per-run physics of the stepper (FP64 scalars).

* ``romberg``            -- pystarc/lib/numerical.py:74-97
* ``return_prob_and_kb`` -- GPUBatchSimulator._compute_return_prob
                            (pystarc/simulation/gpu_batch_simulator.py:320-404): Yukawa U with
                            the dielectric hard-coded to 78 * 0.000142, optional HI D_parallel
* ``bradius_cover``      -- the cover-zone boundary b + x0 (:406-460); the stepper does not
                            use it, the simulator keeps it as ``_bradius_cover`` as the reference does
* ``bridge_d_eff``       -- per-pair D_eff of the Brownian bridge (:637-660)
* ``multipole``          -- MultipoleExpansion moments (pystarc/forces/multipole_farfield.py:86-110)
* ``wilson_ci`` / ``rate_constant`` -- GPUBatchResult (:61-113)
"""

from __future__ import annotations

import math
from statistics import NormalDist

import numpy as np

EPS0 = 0.000142
CONV = 6.022e23 * 1e-30 / 1e-12 / 1e-3


def romberg(f, a, b, tol=1e-8, max_order=12):
    R = [[0.0] * (max_order + 1) for _ in range(max_order + 1)]
    h = b - a
    R[0][0] = 0.5 * h * (f(a) + f(b))
    for i in range(1, max_order + 1):
        h /= 2.0
        s = sum(f(a + (2 * k - 1) * h) for k in range(1, 2 ** i // 2 + 1))
        R[i][0] = 0.5 * R[i - 1][0] + h * s
        for j in range(1, i + 1):
            R[i][j] = R[i][j - 1] + (R[i][j - 1] - R[i - 1][j - 1]) / (4 ** j - 1)
        if i >= 2 and abs(R[i][i] - R[i - 1][i - 1]) < tol:
            return R[i][i]
    return R[max_order][max_order]


def return_prob_and_kb(r_start, r_escape, q_rec, q_lig, debye, D_t, use_hi=False, a_rec=0.0, a_lig=0.0,
                       kT_scale=1.0):
    """(probability to return from r_escape to the b-sphere, k_b in A^3/ps)."""
    b, q_out = float(r_start), float(r_escape)
    eps = 78.0 * EPS0
    if abs(q_rec * q_lig) < 1e-9:
        return b / q_out, 4.0 * math.pi * D_t * b
    if use_hi:
        a2 = 0.5 * (a_rec ** 2 + a_lig ** 2)
        ainv = 1.0 / a_rec + 1.0 / a_lig
        dpre = D_t / ainv

    def integrand(s):
        if s == 0.0:
            return 1.0 / D_t
        r = 1.0 / s
        v = q_rec * q_lig / (4.0 * math.pi * eps * r) * math.exp(-r / debye) / kT_scale
        if use_hi:
            return math.exp(v) / (dpre * (ainv - 3.0 / r + 2.0 * a2 / r ** 3))
        return math.exp(v) / D_t

    try:
        k_b = 4.0 * math.pi / romberg(integrand, 0.0, 1.0 / b)
        k_q = 4.0 * math.pi / romberg(integrand, 0.0, 1.0 / q_out)
        rp = k_b / k_q if k_q > 0 else 0.5
        return float(max(0.0, min(1.0, rp))), k_b
    except (OverflowError, ZeroDivisionError, ValueError):
        return b / q_out, 4.0 * math.pi * D_t * b


def bradius_cover(b, q_rec, q_lig, debye, eps=78.0 * EPS0):
    """b + x0: the radius beyond the b-sphere where the Yukawa force stops being linear enough.

    Two bisections, as the reference takes them:
      1. the linear-region width L: the first r > b where the force's relative curvature
         (2 l^2 + 2 r l + r^2) |r - b| / (r l (l + r)) reaches 0.05 (l = Debye length), found by
         doubling from 2b and halving to 1e-6 b, capped at 0.1 b;
      2. x0 in (0, L) where the probability of a step leaving the linear region,
         erfc((L - x0^2 F(b) - x0) / (2 x0)) / (erf((x0 F(b) + 1) / 2) + 1), falls to 0.01
         (F = the Yukawa force, in kT/A), to 1e-6 L or 100 halvings.
    """
    from scipy.special import erf, erfc  # the reference's error functions

    v_factor = q_rec * q_lig / (4.0 * math.pi * eps)
    lam = debye

    def excess_curvature(r):
        return (2 * lam ** 2 + 2 * r * lam + r ** 2) * abs(r - b) / (r * lam * (lam + r)) - 0.05

    hi = 2.0 * b
    while excess_curvature(hi) < 0.0:
        hi *= 2.0
    lo = b
    while hi - lo > 1e-6 * b:
        mid = 0.5 * (lo + hi)
        if excess_curvature(mid) * excess_curvature(hi) < 0.0:
            lo = mid
        else:
            hi = mid
    width = min(0.5 * (lo + hi) - b, 0.1 * b)
    rm1 = 1.0 / b
    f_b = v_factor * math.exp(-b / lam) * rm1 * (rm1 + 1.0 / lam)

    def p_leave(x0):
        if x0 <= 1e-10:
            return 1.0
        try:
            return erfc((width - x0 ** 2 * f_b - x0) / (2.0 * x0)) / (erf((x0 * f_b + 1.0) / 2.0) + 1.0 + 1e-30)
        except (OverflowError, ValueError, ZeroDivisionError):
            return 0.0

    lo, hi = 0.0, width
    for _ in range(100):
        if hi - lo < 1e-6 * max(width, 1e-10):
            break
        mid = 0.5 * (lo + hi)
        if p_leave(mid) > 0.01:
            hi = mid
        else:
            lo = mid
    return float(b + 0.5 * (lo + hi))


def bridge_d_eff(D_t, r_h_rec, r_h_lig, rec_pair_xyz, lig_pair_body):
    """D_t + D_rot,rec L_rec^2 + D_rot,lig L_lig^2 per reaction pair; L = distance to the molecule's centre."""
    a_sum = r_h_rec + r_h_lig if (r_h_rec + r_h_lig) > 0 else 1.0
    D_tr_rec = D_t * r_h_lig / a_sum
    D_tr_lig = D_t * r_h_rec / a_sum
    D_rot_rec = D_tr_rec * 3.0 / (4.0 * r_h_rec ** 2) if r_h_rec > 0 else 0.0
    D_rot_lig = D_tr_lig * 3.0 / (4.0 * r_h_lig ** 2) if r_h_lig > 0 else 0.0
    L_rec = np.linalg.norm(np.asarray(rec_pair_xyz, dtype=float).reshape(-1, 3), axis=1)
    L_lig = np.linalg.norm(np.asarray(lig_pair_body, dtype=float).reshape(-1, 3), axis=1)
    return D_t + D_rot_rec * L_rec ** 2 + D_rot_lig * L_lig ** 2


def multipole(positions, charges, sdie):
    """(Q, dipole, traceless quadrupole 1/2 sum q (3 r r - r^2 I), 4 pi eps)."""
    pos = np.asarray(positions, dtype=float)
    q = np.asarray(charges, dtype=float)
    dip = np.sum(q[:, None] * pos, axis=0)
    r2 = np.sum(pos ** 2, axis=1)
    quad = np.zeros((3, 3))
    for a in range(3):
        for b in range(3):
            quad[a, b] = np.sum(q * (3.0 * pos[:, a] * pos[:, b] - (r2 if a == b else 0.0)))
    return float(q.sum()), dip, 0.5 * quad, 4.0 * math.pi * (sdie * EPS0)


def wilson_ci(n_reacted, n_escaped, confidence=0.95):
    n = n_reacted + n_escaped
    if n == 0:
        return (0.0, 1.0)
    z = NormalDist().inv_cdf(0.5 + confidence / 2.0)
    p = n_reacted / n
    z2n = z ** 2 / n
    denom = 1.0 + z2n
    centre = (p + z2n / 2.0) / denom
    margin = z * math.sqrt(max(p * (1 - p) / n + z2n / (4.0 * n), 0)) / denom
    return (max(0.0, centre - margin), min(1.0, centre + margin))


def rate_constant(P, D_rel, k_b, r_start, r_escape):
    if P <= 0.0:
        return 0.0
    if k_b > 0.0:
        return CONV * k_b * P
    k_D = 4.0 * math.pi * D_rel * r_start
    beta = r_start / r_escape
    return CONV * k_D * P / (1.0 - P * (1.0 - beta))
