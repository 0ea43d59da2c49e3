"""Seeded synthetic structures for the five SOAP workloads.

No dataset is shipped with the reference other than one 3000-atom water
cluster (``examples/water.xyz``); every workload here is generated from a
fixed seed with the sizes, densities and species mixes the benchmark
specification gives:

* ``water_cluster(nx, ny, nz)`` -- (H2O)_n on a jittered cubic lattice
  (spacing 3.1 A, uniform +-0.3 A jitter on O, two H at 0.96 A with a
  104.5 degree H-O-H angle, uniformly random molecular orientation).
  4x4x4 -> 192 atoms, 10x10x10 -> 3000 atoms, and a 70x70x69 grid truncated
  to its first 333,334 sites in lexicographic order -> 1,000,002 atoms.
* ``random_cells(n, ...)`` -- periodic cubic cells with A ~ U{8..400} atoms
  at 0.1 atoms/A^3, Poisson-disk positions (dart throwing, 0.9 A minimum
  periodic distance), species uniform over {H, C, N, O}.
* ``water_box(n_mol, side)`` -- periodic bulk water, random orientations,
  O-O minimum periodic distance 2.6 A (667 molecules in a 27.1 A cube).

Atoms of a molecule are stored O, H, H.
"""
from __future__ import annotations

import math
from typing import Dict, List

import numpy as np

OH = 0.96
HOH = math.radians(104.5)


def _random_rotations(rng, n):
    q = rng.standard_normal((n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    R = np.empty((n, 3, 3))
    R[:, 0, 0] = 1 - 2 * (y * y + z * z)
    R[:, 0, 1] = 2 * (x * y - z * w)
    R[:, 0, 2] = 2 * (x * z + y * w)
    R[:, 1, 0] = 2 * (x * y + z * w)
    R[:, 1, 1] = 1 - 2 * (x * x + z * z)
    R[:, 1, 2] = 2 * (y * z - x * w)
    R[:, 2, 0] = 2 * (x * z - y * w)
    R[:, 2, 1] = 2 * (y * z + x * w)
    R[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return R


def _add_hydrogens(rng, O):
    n = O.shape[0]
    h = np.array([[OH * math.sin(HOH / 2), 0.0, OH * math.cos(HOH / 2)],
                  [-OH * math.sin(HOH / 2), 0.0, OH * math.cos(HOH / 2)]])
    R = _random_rotations(rng, n)
    H = O[:, None, :] + np.einsum("nij,kj->nki", R, h)
    pos = np.concatenate([O[:, None, :], H], axis=1).reshape(-1, 3)
    Z = np.tile(np.array([8, 1, 1], np.int64), n)
    return pos, Z


def water_cluster(nx: int, ny: int, nz: int, n_mol: int | None = None, seed: int = 0,
                  spacing: float = 3.1, jitter: float = 0.3) -> Dict[str, np.ndarray]:
    """Non-periodic (H2O)_n cluster on a jittered nx*ny*nz lattice."""
    rng = np.random.default_rng(seed)
    g = np.stack(np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij"), -1).reshape(-1, 3)
    if n_mol is not None:
        g = g[:n_mol]
    O = g * spacing + rng.uniform(-jitter, jitter, g.shape)
    pos, Z = _add_hydrogens(rng, O)
    return {"positions": pos, "atomic_numbers": Z}


def _dart_throw(rng, n, side, dmin, max_tries=2_000_000, batch=64):
    pts = np.empty((0, 3))
    tries = 0
    while pts.shape[0] < n:
        cand = rng.uniform(0.0, side, (batch, 3))
        tries += batch
        if tries > max_tries:
            raise RuntimeError("dart throwing did not converge")
        for p in cand:
            if pts.shape[0] >= n:
                break
            if pts.shape[0]:
                d = pts - p
                d -= side * np.round(d / side)
                if np.min((d * d).sum(1)) < dmin * dmin:
                    continue
            pts = np.vstack([pts, p])
    return pts


def random_cells(n_cells: int = 512, seed: int = 0, a_min: int = 8, a_max: int = 400,
                 density: float = 0.1, dmin: float = 0.9,
                 species=(1, 6, 7, 8)) -> List[Dict[str, np.ndarray]]:
    """Periodic cubic cells of uneven size (the batched workload)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_cells):
        A = int(rng.integers(a_min, a_max + 1))
        side = (A / density) ** (1.0 / 3.0)
        pos = _dart_throw(rng, A, side, dmin)
        Z = rng.choice(np.asarray(species, np.int64), size=A)
        out.append({"positions": pos, "atomic_numbers": Z, "cell": np.eye(3) * side,
                    "pbc": np.array([True, True, True])})
    return out


def water_box(n_mol: int = 667, side: float = 27.1, seed: int = 0, dmin: float = 2.6) -> Dict[str, np.ndarray]:
    """Periodic bulk water: O by dart throwing (O-O >= dmin), random orientations."""
    rng = np.random.default_rng(seed)
    O = _dart_throw(rng, n_mol, side, dmin, max_tries=50_000_000, batch=256)
    pos, Z = _add_hydrogens(rng, O)
    return {"positions": pos, "atomic_numbers": Z, "cell": np.eye(3) * side,
            "pbc": np.array([True, True, True])}


# Parameters of each workload, in the reference constructor's vocabulary.
CONFIGS = {
    "cluster192": dict(species=[1, 8], r_cut=5.0, n_max=4, l_max=3, sigma=0.5, average="off"),
    "cluster3000": dict(species=[1, 8], r_cut=10.0, n_max=7, l_max=3, sigma=0.5, average="off"),
    "cells512": dict(species=[1, 6, 7, 8], r_cut=6.0, n_max=8, l_max=6, sigma=0.4, average="inner",
                     periodic=True),
    "waterbox2001": dict(species=[1, 8], r_cut=6.0, n_max=8, l_max=6, sigma=1.0, average="off",
                         periodic=True),
    "cluster1M": dict(species=[1, 8], r_cut=6.0, n_max=8, l_max=4, sigma=1.0, average="off"),
}


def make(name: str):
    """The structure(s) of a named workload."""
    if name == "cluster192":
        return water_cluster(4, 4, 4, seed=0)
    if name == "cluster3000":
        return water_cluster(10, 10, 10, seed=0)
    if name == "cells512":
        return random_cells(512, seed=0)
    if name == "waterbox2001":
        return water_box(667, 27.1, seed=0)
    if name == "cluster1M":
        return water_cluster(70, 70, 69, n_mol=333_334, seed=0)
    raise KeyError(name)
