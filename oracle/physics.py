"""Host-side physics of the batched stepper, restated in FP64 (test infrastructure).

* ``romberg``            -- pystarc/lib/numerical.py:74-97
* ``return_prob_and_kb`` -- GPUBatchSimulator._compute_return_prob
                            (pystarc/simulation/gpu_batch_simulator.py:320-404)
* ``stokes_*``           -- pystarc/hydrodynamics/rotne_prager.py:43-64
* ``rpy_offdiagonal``    -- Zuk three-regime tensor, rotne_prager.py:67-124
* ``wilson_ci`` / ``rate_constant`` -- GPUBatchResult (gpu_batch_simulator.py:61-113)
"""

from __future__ import annotations

import math

import numpy as np

KB_SI = 1.380649e-23
T_DEFAULT = 298.15
ETA_WATER = 1.002e-3
ANG_TO_M = 1.0e-10
PS_TO_S = 1.0e-12
EPS0 = 0.000142
CONV = 6.022e23 * 1e-30 / 1e-12 / 1e-3


def romberg(f, a, b, tol=1e-8, max_order=12):
    R = [[0.0] * (max_order + 1) for _ in range(max_order + 1)]
    h = b - a
    R[0][0] = 0.5 * h * (f(a) + f(b))
    for i in range(1, max_order + 1):
        h /= 2.0
        n_new = 2 ** i
        s = sum(f(a + (2 * k - 1) * h) for k in range(1, n_new // 2 + 1))
        R[i][0] = 0.5 * R[i - 1][0] + h * s
        for j in range(1, i + 1):
            R[i][j] = R[i][j - 1] + (R[i][j - 1] - R[i - 1][j - 1]) / (4 ** j - 1)
        if i >= 2 and abs(R[i][i] - R[i - 1][i - 1]) < tol:
            return R[i][i]
    return R[max_order][max_order]


def stokes_translational(radius, eta=ETA_WATER, T=T_DEFAULT):
    r_m = radius * ANG_TO_M
    return KB_SI * T / (6.0 * math.pi * eta * r_m) / (ANG_TO_M ** 2) * PS_TO_S


def stokes_rotational(radius, eta=ETA_WATER, T=T_DEFAULT):
    r_m = radius * ANG_TO_M
    return KB_SI * T / (8.0 * math.pi * eta * r_m ** 3) * PS_TO_S


def rpy_offdiagonal(r_vec, a, b, D_a, D_b):
    r = float(np.linalg.norm(r_vec))
    if r < 1e-10:
        return np.zeros((3, 3))
    rhat = np.asarray(r_vec, dtype=np.float64) / r
    outer = np.outer(rhat, rhat)
    PI = math.pi
    a2, b2, r2 = a * a, b * b, r * r
    r3 = r2 * r
    if r > a + b:
        den = 8.0 * PI * r
        tt_I = (1.0 + (a2 + b2) / (3.0 * r2)) / den
        tt_uu = (1.0 - (a2 + b2) / r2) / den
    elif r > abs(a - b):
        den = 6.0 * 32.0 * PI * a * b * r3
        am2 = (a - b) ** 2
        tt_I = (16.0 * r3 * (a + b) - (am2 + 3.0 * r2) ** 2) / den
        tt_uu = 3.0 * (am2 - r2) ** 2 / den
    else:
        tt_I = 1.0 / (6.0 * PI * max(a, b))
        tt_uu = 0.0
    kT_over_eta = math.sqrt(D_a * 6.0 * PI * a * D_b * 6.0 * PI * b)
    return kT_over_eta * (tt_I * np.eye(3) + tt_uu * outer)


def return_prob_and_kb(r_start, r_escape, q_rec, q_lig, debye, D_t, use_hi=False, radius1=0.0, radius2=0.0,
                       kT_scale=1.0):
    """(return probability, k_b) as in _compute_return_prob (gpu_batch_simulator.py:320-404).

    U is the point-charge Yukawa potential with the dielectric hard-coded to
    78 * 0.000142 (:338-340).  Returns the reference's fallbacks on failure.
    """
    b = r_start
    q_out = r_escape
    eps = 78.0 * EPS0
    if abs(q_rec * q_lig) < 1e-9:
        return b / q_out, 4.0 * math.pi * D_t * b

    def U(r):
        return q_rec * q_lig / (4.0 * math.pi * eps * r) * math.exp(-r / debye)

    if use_hi:
        a0, a1 = float(radius1), float(radius2)
        a2 = 0.5 * (a0 ** 2 + a1 ** 2)
        ainv = 1.0 / a0 + 1.0 / a1
        dpre = D_t / ainv

    def intgd(s):
        if s == 0.0:
            return 1.0 / D_t
        r = 1.0 / s
        v = U(r) / kT_scale
        if use_hi:
            return math.exp(v) / (dpre * (ainv - 3.0 / r + 2.0 * a2 / (r ** 3)))
        return math.exp(v) / D_t

    try:
        k_b = 4.0 * math.pi / romberg(intgd, 0.0, 1.0 / b, tol=1e-8)
        k_q = 4.0 * math.pi / romberg(intgd, 0.0, 1.0 / q_out, tol=1e-8)
        rp = k_b / k_q if k_q > 0 else 0.5
        return float(max(0.0, min(1.0, rp))), k_b
    except Exception:
        return b / q_out, 4.0 * math.pi * D_t * b


def wilson_ci(n_reacted, n_escaped, confidence=0.95, z=None):
    """Wilson interval of GPUBatchResult.reaction_probability_ci (:70-80), z = Phi^-1(0.5 + c/2)."""
    from statistics import NormalDist

    n = n_reacted + n_escaped
    if n == 0:
        return (0.0, 1.0)
    if z is None:
        z = NormalDist().inv_cdf(0.5 + confidence / 2.0)
    p = n_reacted / n
    z2n = z ** 2 / n
    denom = 1.0 + z2n
    centre = (p + z2n / 2.0) / denom
    margin = z * math.sqrt(max(p * (1 - p) / n + z2n / (4.0 * n), 0)) / denom
    return (max(0.0, centre - margin), min(1.0, centre + margin))


def rate_constant(P, D_rel, k_b, r_start, r_escape):
    """k_on from P (GPUBatchResult.rate_constant, :82-96)."""
    if P <= 0.0:
        return 0.0
    if k_b > 0.0:
        return CONV * k_b * P
    k_D = 4.0 * math.pi * D_rel * r_start
    beta = r_start / r_escape
    return CONV * k_D * P / (1.0 - P * (1.0 - beta))
