"""NumPy Philox4x32-10 and the engine's keyed draw layout (test infrastructure).

Philox4x32-10 is the counter-based generator of Salmon, Moraes, Dror and Shaw,
"Parallel random numbers: as easy as 1, 2, 3" (SC'11): ten rounds of two
32x32->64-bit multiplies with the published multipliers and Weyl key
increments.  The CUDA engine implements the same function; this restatement is
the checker for it and drives the oracle stepper's "philox" noise mode.

Draw layout, keyed by (seed, trajectory id, the trajectory's own step index):

  counter = (step, sub, traj_lo, traj_hi), key = (seed_lo, seed_hi)

  step-time subs: 0 -> u_escape (words 0,1)
                  1,2,3 -> six normals: translation xyz, rotation xyz
                  4,5 -> three uniforms of the return quaternion
                  6 + p//2 -> bridge uniform of pair p (words 0,1 or 2,3)
  start (step = 0xFFFFFFFF): 0,1 -> three normals of the start direction
                             2,3 -> three uniforms of the start quaternion
"""

from __future__ import annotations

import numpy as np

M0 = np.uint64(0xD2511F53)
M1 = np.uint64(0xCD9E8D57)
W0 = np.uint32(0x9E3779B9)
W1 = np.uint32(0xBB67AE85)
MASK32 = np.uint64(0xFFFFFFFF)
INIT_STEP = 0xFFFFFFFF

SUB_ESCAPE = 0
SUB_NORMALS = 1
SUB_RETURN_Q = 4
SUB_BRIDGE = 6
SUB_INIT_DIR = 0
SUB_INIT_Q = 2


def philox4x32_10(c0, c1, c2, c3, k0, k1):
    """Vectorised Philox4x32-10; all inputs broadcast, returns four uint32 arrays."""
    c0, c1, c2, c3 = (np.asarray(x, dtype=np.uint64) & MASK32 for x in (c0, c1, c2, c3))
    k0 = np.asarray(k0, dtype=np.uint64) & MASK32
    k1 = np.asarray(k1, dtype=np.uint64) & MASK32
    for r in range(10):
        if r > 0:
            k0 = (k0 + np.uint64(W0)) & MASK32
            k1 = (k1 + np.uint64(W1)) & MASK32
        p0 = M0 * c0
        p1 = M1 * c2
        hi0, lo0 = p0 >> np.uint64(32), p0 & MASK32
        hi1, lo1 = p1 >> np.uint64(32), p1 & MASK32
        c0, c1, c2, c3 = (hi1 ^ c1 ^ k0), lo1, (hi0 ^ c3 ^ k1), lo0
    return tuple(x.astype(np.uint32) for x in (c0, c1, c2, c3))


def uniform53(a, b):
    """Double in [0,1) from two 32-bit words: 27 high bits of a, 26 of b."""
    a = np.asarray(a, dtype=np.uint64) >> np.uint64(5)
    b = np.asarray(b, dtype=np.uint64) >> np.uint64(6)
    return (a.astype(np.float64) * 67108864.0 + b.astype(np.float64)) * (1.0 / 9007199254740992.0)


def box_muller(u1, u2):
    """Two standard normals from two uniforms in [0,1)."""
    rad = np.sqrt(-2.0 * np.log(1.0 - u1))
    ang = 2.0 * np.pi * u2
    return rad * np.cos(ang), rad * np.sin(ang)


class KeyedDraws:
    """Per-(trajectory, step) draws with the layout in the module docstring."""

    def __init__(self, seed: int, id_offset: int = 0):
        seed = int(seed) & 0xFFFFFFFFFFFFFFFF
        self.k0 = np.uint64(seed & 0xFFFFFFFF)
        self.k1 = np.uint64(seed >> 32)
        self.offset = np.uint64(id_offset)

    def words(self, step, sub, traj):
        traj = np.asarray(traj, dtype=np.uint64) + self.offset
        return philox4x32_10(step, sub, traj & MASK32, traj >> np.uint64(32), self.k0, self.k1)

    def uniform_pair(self, step, sub, traj):
        w = self.words(step, sub, traj)
        return uniform53(w[0], w[1]), uniform53(w[2], w[3])

    def u_escape(self, step, traj):
        return self.uniform_pair(step, SUB_ESCAPE, traj)[0]

    def step_normals(self, step, traj):
        """(N,3) translation and (N,3) rotation normals."""
        n = []
        for s in range(3):
            u1, u2 = self.uniform_pair(step, SUB_NORMALS + s, traj)
            a, b = box_muller(u1, u2)
            n += [a, b]
        xi_t = np.stack(n[0:3], axis=-1)
        xi_r = np.stack(n[3:6], axis=-1)
        return xi_t, xi_r

    def return_uniforms(self, step, traj):
        u0, u1 = self.uniform_pair(step, SUB_RETURN_Q, traj)
        u2, _ = self.uniform_pair(step, SUB_RETURN_Q + 1, traj)
        return np.stack([u0, u1, u2], axis=-1)

    def bridge_uniforms(self, step, traj, n_pairs):
        cols = []
        for p in range(n_pairs):
            a, b = self.uniform_pair(step, SUB_BRIDGE + p // 2, traj)
            cols.append(a if p % 2 == 0 else b)
        return np.stack(cols, axis=-1) if cols else np.zeros((np.size(traj), 0))

    def start_normals(self, traj):
        u1, u2 = self.uniform_pair(INIT_STEP, SUB_INIT_DIR, traj)
        a, b = box_muller(u1, u2)
        u3, u4 = self.uniform_pair(INIT_STEP, SUB_INIT_DIR + 1, traj)
        c, _ = box_muller(u3, u4)
        return np.stack([a, b, c], axis=-1)

    def start_uniforms(self, traj):
        u0, u1 = self.uniform_pair(INIT_STEP, SUB_INIT_Q, traj)
        u2, _ = self.uniform_pair(INIT_STEP, SUB_INIT_Q + 1, traj)
        return np.stack([u0, u1, u2], axis=-1)
