"""Seeded synthetic inputs of the se_e2_a benchmarks: the model definition
with seeded random weights, and water / Cu frames.

This module uses numpy only, so that a CPU-only caller (the reference arm of
the benchmark, the golden-fixture scripts) can make the same inputs without
loading the GPU library.

No public dataset is used. A frame is n x n x n water molecules: each O on a
cubic grid of spacing 3.104 A with a uniform +-0.3 A jitter per axis, two H at
0.9572 A from it with an H-O-H angle of 104.52 deg, the molecule rigidly
rotated by a uniformly random rotation. Types are O=0, H=1 in [O, H, H] order
per molecule. n = 4 gives the 64-molecule / 192-atom box of 12.4172 A; n = 16
gives 4096 molecules / 12,288 atoms in 49.6688 A (the 4x4x4 replica of the
small box, with fresh jitter and rotations in every replica).
"""

from __future__ import annotations

from dataclasses import dataclass, field

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


# ------------------------------------------------ batched uneven frames ---
WATER_VOLUME_PER_MOLECULE = 18.015 / 0.60221408  # A^3 per molecule at 1.0 g/cm^3
CU_A = 3.615                                      # FCC lattice constant (A)
FCC_BASIS = np.array([[0.0, 0.0, 0.0], [0.0, 0.5, 0.5], [0.5, 0.0, 0.5], [0.5, 0.5, 0.0]])


def water_frame_density(n_atoms: int, rng: np.random.Generator):
    """Water of about n_atoms atoms (round(n/3) molecules) in a cubic box at
    1.0 g/cm^3: O on the sites of an n_side^3 grid over the box (a random
    subset when the molecule count is not a cube), +-0.3 A jitter, H placed as
    in water_frame. Types O=0, H=1."""
    nm = max(1, int(round(n_atoms / 3)))
    L = (nm * WATER_VOLUME_PER_MOLECULE) ** (1.0 / 3.0)
    n_side = int(np.ceil(nm ** (1.0 / 3.0) - 1e-9))
    g = (np.arange(n_side) + 0.5) * (L / n_side)
    sites = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    o = sites[np.sort(rng.choice(sites.shape[0], nm, replace=False))]
    o = o + rng.uniform(-0.3, 0.3, size=o.shape)
    half = HOH / 2
    h_local = np.array([[OH * np.sin(half), OH * np.cos(half), 0.0],
                        [-OH * np.sin(half), OH * np.cos(half), 0.0]])
    R = random_rotations(rng, nm)
    h = np.einsum("mij,kj->mki", R, h_local) + o[:, None, :]
    coord = np.mod(np.concatenate([o[:, None, :], h], axis=1).reshape(-1, 3), L)
    atype = np.tile(np.array([0, 1, 1], np.int32), nm)
    return coord, atype, np.diag([L, L, L]).reshape(9)


def cu_frame(n_atoms: int, rng: np.random.Generator, sigma: float = 0.05):
    """FCC copper (a = 3.615 A) of exactly n_atoms atoms: the smallest cubic
    supercell of k^3 unit cells (k >= 2, so every box edge exceeds the 6 A
    cutoff) that holds them, Gaussian jitter sigma, then random atoms deleted
    down to n_atoms (vacancies; the periodic box is kept). Type Cu=2."""
    k = max(2, int(np.ceil((n_atoms / 4.0) ** (1.0 / 3.0) - 1e-9)))
    g = np.arange(k)
    cells = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 1, 3)
    pos = ((cells + FCC_BASIS[None]) * CU_A).reshape(-1, 3)
    pos = pos + rng.normal(0.0, sigma, size=pos.shape)
    keep = np.sort(rng.choice(pos.shape[0], n_atoms, replace=False))
    L = k * CU_A
    return np.mod(pos[keep], L), np.full(n_atoms, 2, np.int32), np.diag([L, L, L]).reshape(9)


def batched_frames(n_frames: int = 512, seed: int = 0, n_min: int = 24, n_max: int = 3000):
    """Frames of log-uniform atom counts in [n_min, n_max]: even frames water
    at 1.0 g/cm^3, odd frames FCC Cu with vacancies. Returns a list of
    (coord [n, 3], atype [n], box [9])."""
    rng = np.random.default_rng(seed)
    counts = np.exp(rng.uniform(np.log(n_min), np.log(n_max), size=n_frames)).astype(int)
    return [water_frame_density(int(n), rng) if f % 2 == 0 else cu_frame(int(n), rng)
            for f, n in enumerate(counts)]


# ------------------------------------------------------------ the model ---
@dataclass
class SeAConfig:
    rcut: float = 6.0
    rcut_smth: float = 0.5
    sel: tuple = (46, 92)
    neuron: tuple = (25, 50, 100)
    axis_neuron: int = 16
    fitting: tuple = (240, 240, 240)

    @property
    def ntypes(self) -> int:
        return len(self.sel)

    @property
    def nnei(self) -> int:
        return int(sum(self.sel))

    @property
    def sec(self) -> np.ndarray:
        return np.concatenate([[0], np.cumsum(self.sel)]).astype(np.int32)


@dataclass
class SeAParams:
    cfg: SeAConfig
    emb: list                 # per neighbor type: [(W, b), ...]
    fit: list                 # per center type: [(W, b, idt|None), ...] + out (W, b)
    bias_atom_e: np.ndarray
    davg: np.ndarray = None   # [ntypes, nnei * 4]
    dstd: np.ndarray = None
    tables: list = field(default_factory=list)  # [(table f64, info f64)] per neighbor type


def init_params(cfg: SeAConfig, seed: int = 0) -> SeAParams:
    """Seeded random weights: W ~ N(0, 1/fan_in), b ~ N(0, 1); timestep
    vectors ~ N(0.1, 0.001) as the reference initialises them
    (deepmd/dpmodel/utils/network.py:135-146)."""
    rng = np.random.default_rng(seed)

    def layer(n_in, n_out, idt=False):
        W = rng.normal(0.0, np.sqrt(1.0 / n_in), size=(n_in, n_out))
        b = rng.normal(0.0, 1.0, size=n_out)
        d = rng.normal(0.1, 0.001, size=n_out) if idt else None
        return W, b, d

    emb = []
    for _ in range(cfg.ntypes):
        widths = [1, *cfg.neuron]
        emb.append([layer(widths[k], widths[k + 1])[:2] for k in range(len(cfg.neuron))])
    fit = []
    din = cfg.neuron[-1] * cfg.axis_neuron
    for _ in range(cfg.ntypes):
        widths = [din, *cfg.fitting]
        layers = []
        for k in range(len(cfg.fitting)):
            W, b, d = layer(widths[k], widths[k + 1], idt=True)
            layers.append((W, b, d if widths[k] == widths[k + 1] else None))
        Wo, bo, _ = layer(cfg.fitting[-1], 1)
        fit.append({"layers": layers, "out": (Wo, bo)})
    return SeAParams(cfg=cfg, emb=emb, fit=fit, bias_atom_e=np.zeros(cfg.ntypes))
