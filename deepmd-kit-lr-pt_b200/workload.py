"""Seeded synthetic water frames for the se_e2_a benchmarks.

No public dataset is used. A frame is n x n x n water molecules: each O on a
cubic grid of spacing 3.104 A with a uniform +-0.3 A jitter per axis, two H at
0.9572 A from it with an H-O-H angle of 104.52 deg, the molecule rigidly
rotated by a uniformly random rotation. Types are O=0, H=1 in [O, H, H] order
per molecule. n = 4 gives the 64-molecule / 192-atom box of 12.4172 A; n = 16
gives 4096 molecules / 12,288 atoms in 49.6688 A (the 4x4x4 replica of the
small box, with fresh jitter and rotations in every replica).
"""

from __future__ import annotations

import numpy as np

SPACING = 3.104
BOX_PER_SIDE = 12.4172 / 4  # 3.1043 A per molecule along each axis
OH = 0.9572
HOH = np.deg2rad(104.52)


def random_rotations(rng: np.random.Generator, n: int) -> np.ndarray:
    """n uniformly distributed rotation matrices (unit-quaternion sampling)."""
    u1, u2, u3 = rng.random(n), rng.random(n), rng.random(n)
    q = np.stack([np.sqrt(1 - u1) * np.sin(2 * np.pi * u2),
                  np.sqrt(1 - u1) * np.cos(2 * np.pi * u2),
                  np.sqrt(u1) * np.sin(2 * np.pi * u3),
                  np.sqrt(u1) * np.cos(2 * np.pi * u3)], axis=1)
    x, y, z, w = q.T
    return np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1),
    ], axis=1)


def water_frame(n_side: int = 4, seed: int = 0):
    """Returns (coord [3*n^3, 3] float64, atype [3*n^3] int32, box [9])."""
    rng = np.random.default_rng(seed)
    L = BOX_PER_SIDE * n_side
    g = np.arange(n_side) * SPACING
    o = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    o = o + rng.uniform(-0.3, 0.3, size=o.shape)
    nm = o.shape[0]
    half = HOH / 2
    h_local = np.array([[OH * np.sin(half), OH * np.cos(half), 0.0],
                        [-OH * np.sin(half), OH * np.cos(half), 0.0]])
    R = random_rotations(rng, nm)
    h = np.einsum("mij,kj->mki", R, h_local) + o[:, None, :]
    coord = np.concatenate([o[:, None, :], h], axis=1).reshape(-1, 3)
    coord = np.mod(coord, L)
    atype = np.tile(np.array([0, 1, 1], np.int32), nm)
    box = np.diag([L, L, L]).reshape(9)
    return coord, atype, box
