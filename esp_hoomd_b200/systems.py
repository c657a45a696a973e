"""Seeded synthetic systems for the ESP workloads.

HOOMD-blue (which would normally supply particle data) is not available,
so these generators build the inputs the workloads are defined on:
rock-salt lattices (charges +-1 alternating on a jittered simple-cubic
lattice) and rigid three-site water boxes. All are orthorhombic periodic
boxes with positions wrapped into [0, L).
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Tuple

import numpy as np


@dataclasses.dataclass
class System:
    pos: np.ndarray  # [N,3] float64
    q: np.ndarray  # [N] float64
    vel: np.ndarray  # [N,3] float64
    mass: np.ndarray  # [N] float64
    box: Tuple[float, float, float]
    name: str = ""

    @property
    def N(self) -> int:
        return int(self.pos.shape[0])


def rocksalt(n: int, spacing: float = 1.0, jitter: float = 0.1, seed: int = 0, T: float = 1.0,
             shape: Tuple[int, int, int] = None) -> System:
    """n^3 (or shape[0] x shape[1] x shape[2]) simple-cubic lattice,
    q = (-1)^(ix+iy+iz), uniform jitter U(-jitter, jitter) per axis, Maxwell
    velocities at temperature T with the centre-of-mass momentum removed,
    mass 1. Box edges = lattice counts x spacing."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = shape if shape is not None else (n, n, n)
    ix, iy, iz = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    idx = np.stack([ix.ravel(), iy.ravel(), iz.ravel()], -1)
    pos = (idx + 0.5) * spacing + rng.uniform(-jitter, jitter, idx.shape)
    L = np.array([nx, ny, nz], dtype=np.float64) * spacing
    pos = np.mod(pos, L)
    q = np.where(np.sum(idx, -1) % 2 == 0, 1.0, -1.0)
    vel = rng.normal(0.0, math.sqrt(T), idx.shape)
    vel -= vel.mean(0)
    return System(pos=pos, q=q, vel=vel, mass=np.ones(pos.shape[0]), box=tuple(float(v) for v in L),
                  name="rocksalt%dx%dx%d" % (nx, ny, nz))


def water(n_mol: int, density: float = 33.4, seed: int = 0, q_o: float = -0.8476, r_oh: float = 0.1,
          angle_deg: float = 109.47) -> System:
    """Rigid three-site water molecules (O, H, H) at a number density of
    molecules per nm^3, centres on a jittered cubic lattice (m^3 sites,
    m = ceil(n_mol^(1/3)); when n_mol is not a cube a seeded random subset
    of the sites is occupied), uniformly random orientations (unit
    quaternions). Velocities zero; masses 16/1/1."""
    rng = np.random.default_rng(seed)
    m = int(round(n_mol ** (1.0 / 3.0)))
    if m ** 3 < n_mol:
        m += 1
    L = (n_mol / density) ** (1.0 / 3.0)
    a = L / m
    ix, iy, iz = np.meshgrid(np.arange(m), np.arange(m), np.arange(m), indexing="ij")
    centres = (np.stack([ix.ravel(), iy.ravel(), iz.ravel()], -1) + 0.5) * a
    if m ** 3 != n_mol:
        centres = centres[np.sort(rng.choice(m ** 3, size=n_mol, replace=False))]
    centres += rng.uniform(-0.05 * a, 0.05 * a, centres.shape)
    half = math.radians(angle_deg) / 2.0
    body = np.array([[0.0, 0.0, 0.0],
                     [r_oh * math.sin(half), 0.0, r_oh * math.cos(half)],
                     [-r_oh * math.sin(half), 0.0, r_oh * math.cos(half)]])
    body -= body.mean(0)
    qv = rng.normal(size=(n_mol, 4))
    qv /= np.linalg.norm(qv, axis=1, keepdims=True)
    w, x, y, z = qv.T
    R = np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1)], 1)
    pos = centres[:, None, :] + np.einsum("mij,sj->msi", R, body)
    pos = np.mod(pos.reshape(-1, 3), L)
    q = np.tile([q_o, -q_o / 2, -q_o / 2], n_mol)
    mass = np.tile([16.0, 1.0, 1.0], n_mol)
    return System(pos=pos, q=q, vel=np.zeros_like(pos), mass=mass, box=(L, L, L), name="water%d" % n_mol)


def batched_rocksalt(n_sys: int = 256, seed: int = 1004, n_lo: int = 8, n_hi: int = 40) -> List[System]:
    """The mixed batch: system i is an n^3 rock-salt lattice with n even,
    drawn seeded-uniform from n_lo..n_hi, built with seed seed*100000+i."""
    rng = np.random.default_rng(seed)
    evens = np.arange(n_lo, n_hi + 1, 2)
    ns = rng.choice(evens, size=n_sys)
    return [rocksalt(int(n), seed=seed * 100000 + i) for i, n in enumerate(ns)]
