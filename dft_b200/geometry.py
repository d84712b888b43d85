"""Seeded synthetic molecules for the integral / Fock-build path.

All coordinates are in bohr.  Atoms are given as strings of the nuclear charge,
the way the reference lists them (``atoms = ["64", "9", ...]``, shelled.py:37),
and centres as an ``(n_atoms, 3)`` float64 array (shelled.py:38, :79).

Workloads:

* ``water()`` -- one H2O, O at (0, 0, 0.2217), H at (0, +-1.4309, -0.8867).
* ``alkane(10)`` -- all-trans C10H22 built from C-C 1.54 A, C-H 1.09 A and
  tetrahedral angles, carbon zigzag in the xy plane.
* ``water_cluster((4, 4, 4))`` -- (H2O)_64: the water monomer on a cubic
  lattice with 5.5 bohr spacing, each monomer rotated by a uniform random
  SO(3) rotation about the coordinate origin of the monomer frame, and every
  atom jittered by U(-0.3, 0.3) bohr per coordinate.  Random numbers come from
  ``numpy.random.default_rng(seed)``: first all rotations
  (``scipy.spatial.transform.Rotation.random(n, random_state=rng)``), then all
  jitters (``rng.uniform(-0.3, 0.3, (n, 3, 3))``).
* ``water_cluster_batch(count, n_max, seed)`` -- ``count`` clusters with
  ``n ~ U{1..n_max}`` monomers each, from one generator: the sizes are drawn
  first, then each cluster in turn is built as above on the smallest cube
  lattice holding it (first ``n`` sites in lattice order).
"""
from __future__ import annotations

import math
from typing import List, Sequence, Tuple

import numpy as np

ANGSTROM_TO_BOHR = 1.8897261246

WATER_ATOMS = ["8", "1", "1"]
WATER_CENTERS = np.array(
    [[0.0, 0.0, 0.2217], [0.0, 1.4309, -0.8867], [0.0, -1.4309, -0.8867]], dtype=np.float64
)

Molecule = Tuple[List[str], np.ndarray]


def water() -> Molecule:
    return list(WATER_ATOMS), WATER_CENTERS.copy()


def alkane(n_carbon: int = 10, cc: float = 1.54, ch: float = 1.09) -> Molecule:
    """All-trans CnH(2n+2); carbons first, then hydrogens carbon by carbon.

    The chain runs along x with carbon k at x = k*b and y = +h/2 (k even) or
    -h/2 (k odd), b = d_CC sin(theta/2), h = d_CC cos(theta/2), theta the
    tetrahedral angle, so every C-C-C angle is theta.  Each carbon's two
    out-of-plane hydrogens sit at d_CH (cos(theta/2) u +- sin(theta/2) z),
    u = +y for even k and -y for odd k (the outward bisector); the end
    carbons get a third, in-plane hydrogen where the next chain carbon
    would be.
    """
    if n_carbon < 2:
        raise ValueError("alkane needs at least two carbons")
    theta = math.acos(-1.0 / 3.0)
    dcc = cc * ANGSTROM_TO_BOHR
    dch = ch * ANGSTROM_TO_BOHR
    s, c = math.sin(theta / 2.0), math.cos(theta / 2.0)
    b, h = dcc * s, dcc * c
    carbons = []
    for k in range(n_carbon):
        carbons.append([k * b, (h / 2.0) if k % 2 == 0 else (-h / 2.0), 0.0])
    carbons = np.array(carbons)
    hydrogens = []
    for k in range(n_carbon):
        u = 1.0 if k % 2 == 0 else -1.0
        ck = carbons[k]
        for sz in (1.0, -1.0):
            hydrogens.append(ck + dch * np.array([0.0, c * u, s * sz]))
        if k == 0 or k == n_carbon - 1:
            direction = -1.0 if k == 0 else 1.0
            # the missing neighbour lies at x -+ b with y flipped
            hydrogens.append(ck + dch * np.array([direction * s, -u * c, 0.0]))
    atoms = ["6"] * n_carbon + ["1"] * len(hydrogens)
    centers = np.vstack([carbons, np.array(hydrogens)])
    return atoms, centers.astype(np.float64)


def _lattice_sites(shape: Sequence[int]) -> np.ndarray:
    nx, ny, nz = shape
    sites = [(i, j, k) for i in range(nx) for j in range(ny) for k in range(nz)]
    return np.array(sites, dtype=np.float64)


def _place_waters(sites: np.ndarray, spacing: float, jitter: float, rng) -> Molecule:
    from scipy.spatial.transform import Rotation

    n = sites.shape[0]
    rot = Rotation.random(n, random_state=rng).as_matrix()  # (n, 3, 3)
    shake = rng.uniform(-jitter, jitter, size=(n, 3, 3))
    monomer = WATER_CENTERS
    coords = np.einsum("nij,aj->nai", rot, monomer) + sites[:, None, :] * spacing + shake
    atoms = WATER_ATOMS * n
    return atoms, coords.reshape(-1, 3).astype(np.float64)


def water_cluster(shape: Sequence[int] = (4, 4, 4), spacing: float = 5.5,
                  jitter: float = 0.3, seed: int = 0) -> Molecule:
    rng = np.random.default_rng(seed)
    return _place_waters(_lattice_sites(shape), spacing, jitter, rng)


def water_cluster_batch(count: int = 512, n_max: int = 24, seed: int = 0,
                        spacing: float = 5.5, jitter: float = 0.3) -> List[Molecule]:
    rng = np.random.default_rng(seed)
    sizes = rng.integers(1, n_max + 1, size=count)
    out = []
    for n in sizes:
        side = 1
        while side ** 3 < n:
            side += 1
        sites = _lattice_sites((side, side, side))[: int(n)]
        out.append(_place_waters(sites, spacing, jitter, rng))
    return out


def nuclear_repulsion(atoms: Sequence[str], centers: np.ndarray) -> float:
    """E_NN = sum_{i<j} Z_i Z_j / |R_i - R_j| (shelled.py:157-163)."""
    z = np.array([int(a) for a in atoms], dtype=np.float64)
    d = centers[:, None, :] - centers[None, :, :]
    r = np.sqrt((d * d).sum(-1))
    iu = np.triu_indices(len(z), 1)
    return float((z[:, None] * z[None, :])[iu].dot(1.0 / r[iu]))


def nuclear_repulsion_gradient(atoms: Sequence[str], centers: np.ndarray) -> np.ndarray:
    """dE_NN/dR_A = -sum_{B != A} Z_A Z_B (R_A - R_B) / |R_A - R_B|^3."""
    z = np.array([int(a) for a in atoms], dtype=np.float64)
    d = centers[:, None, :] - centers[None, :, :]
    r = np.sqrt((d * d).sum(-1))
    np.fill_diagonal(r, np.inf)
    return -np.einsum("ab,abx->ax", (z[:, None] * z[None, :]) / r ** 3, d)
