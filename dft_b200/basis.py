"""Basis files and shell construction.

Basis files use the reference's JSON layout (``STO-3G.json``; generator
compile.py:1-23): ``{"Z": [[[l, ...], [exponents], [[coefficients], ...]], ...]}``.
The package ships the public STO-3G set (elements 1-54) as
``data/sto-3g.json``, identical in content to the reference's file.

Shells are dicts with the reference's keys (shelled.py:49-77, :934-952):
``atom_idx, atom_pos, angular_momentum, exponents, coefficients, components,
n_components, n_contractions, n_ao, n_exponents, ao_start, ao_stop,
sphere_n_ao, sphere_ao_start, sphere_ao_stop, normalization``.  Entries that
list several momenta with one coefficient row each (sp shells) are split
into one shell per momentum, as the reference does.
"""
from __future__ import annotations

import json
import math
import os
from typing import Dict, List, Sequence

import numpy as np

DATA_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")
STO3G_PATH = os.path.join(DATA_DIR, "sto-3g.json")


class UnsupportedBasis(ValueError):
    """The basis needs something the kernels do not provide (momenta beyond f)."""


def load_basis(path: str = STO3G_PATH) -> Dict:
    with open(path) as fh:
        return json.load(fh)


def combinations(l: int) -> List[List[int]]:
    """Cartesian powers of angular momentum l in the reference order
    (shelled.py:15-23): loop z, then y, then x power."""
    out = []
    for n in range(l + 1):
        for m in range(l + 1):
            for k in range(l + 1):
                if k + m + n == l:
                    out.append([k, m, n])
    return out


def _double_factorial(n: int) -> float:
    r = 1.0
    while n > 1:
        r *= n
        n -= 2
    return r


def normal(alpha: np.ndarray, powers: np.ndarray) -> np.ndarray:
    """Primitive normalisation sqrt((4a)^L / prod (2l_i - 1)!!) (2a/pi)^{3/4}
    (normal(), shelled.py:95-101).  Contracted functions are not renormalised."""
    alpha = np.asarray(alpha, dtype=np.float64)
    powers = np.asarray(powers)
    L = powers.sum(axis=1)
    df = np.array([_double_factorial(2 * a - 1) * _double_factorial(2 * b - 1) * _double_factorial(2 * c - 1)
                   for a, b, c in powers])
    return np.sqrt(np.power(4.0 * alpha, L) / df) * np.power(2.0 * alpha / math.pi, 0.75)


def build_shells(basis: Dict, atoms: Sequence[str], centers) -> List[Dict]:
    centers = np.asarray(centers, dtype=np.float64)
    shells: List[Dict] = []
    for i, atom in enumerate(atoms):
        key = str(atom)
        if key not in basis:
            raise UnsupportedBasis(f"element {key} not in basis")
        for ls, exps, coefs in basis[key]:
            if len(ls) == 1:
                parts = [(ls[0], coefs)]
            elif len(ls) == len(coefs):
                parts = [(m, [row]) for m, row in zip(ls, coefs)]
            else:
                raise ValueError("basis entry with mismatched momenta and coefficient rows")
            for m, rows in parts:
                shells.append({
                    "atom_idx": i,
                    "atom_pos": centers[i].copy(),
                    "angular_momentum": int(m),
                    "exponents": np.array(exps, dtype=np.float64),
                    "coefficients": np.array(rows, dtype=np.float64),
                })
    ao = 0
    sph = 0
    for sh in shells:
        l = sh["angular_momentum"]
        sh["components"] = np.array(combinations(l), dtype=np.int32)
        sh["n_components"] = len(sh["components"])
        sh["n_contractions"] = sh["coefficients"].shape[0]
        sh["n_ao"] = sh["n_components"] * sh["n_contractions"]
        sh["sphere_n_ao"] = sh["n_contractions"] * (2 * l + 1)
        sh["n_exponents"] = int(sh["exponents"].size)
        sh["ao_start"] = ao
        sh["sphere_ao_start"] = sph
        sh["ao_stop"] = ao + sh["n_ao"]
        sh["sphere_ao_stop"] = sph + sh["sphere_n_ao"]
        e = np.tile(sh["exponents"], sh["n_components"])
        pw = np.repeat(sh["components"], sh["n_exponents"], axis=0).reshape(-1, 3)
        sh["normalization"] = normal(e, pw)
        ao = sh["ao_stop"]
        sph = sh["sphere_ao_stop"]
    return shells


def molecule_shells(atoms: Sequence[str], centers, basis: Dict = None) -> List[Dict]:
    return build_shells(basis if basis is not None else load_basis(), atoms, centers)


def n_electrons(atoms: Sequence[str], charge: int = 0) -> int:
    return sum(int(a) for a in atoms) - charge


LMAX = 3  # f shells: the largest momentum the integral kernels take


def check_supported(shells: List[Dict]) -> None:
    """The integral kernels take s, p, d and f shells, generally contracted or not."""
    for k, sh in enumerate(shells):
        if sh["angular_momentum"] > LMAX:
            raise UnsupportedBasis(f"shell {k}: l = {sh['angular_momentum']} (kernels cover s, p, d and f)")


def check_sp(shells: List[Dict], what: str) -> None:
    """Paths built on the s/p classes only (batches, gradients) take s and p
    shells with one contraction each."""
    for k, sh in enumerate(shells):
        if sh["angular_momentum"] > 1 or np.atleast_2d(sh["coefficients"]).shape[0] != 1:
            raise UnsupportedBasis(f"{what}: shell {k} (l = {sh['angular_momentum']}, "
                                   f"{np.atleast_2d(sh['coefficients']).shape[0]} contractions) needs s/p shells "
                                   "with one contraction")


def radial_norm(alpha: np.ndarray, l: int) -> np.ndarray:
    """sqrt((4a)^l) (2a/pi)^{3/4}: normal() of component (l, 0, 0) times
    sqrt((2l - 1)!!).  The kernels apply each Cartesian component's remaining
    factor 1/sqrt(prod (2 l_i - 1)!!) themselves (1 for s and p)."""
    alpha = np.asarray(alpha, dtype=np.float64)
    return np.sqrt(np.power(4.0 * alpha, l)) * np.power(2.0 * alpha / math.pi, 0.75)


def segments(shells: List[Dict]) -> List[Dict]:
    """One integral shell per contraction row of each shell.

    A generally contracted shell (coefficient matrix with n rows,
    shelled.py:49-64) becomes n shells that share its centre and momentum, keep
    the primitives with a non-zero coefficient in their row, and take the AO
    offsets ao_start + r * n_components: the reference's AO order within a
    shell is contraction-major (the einsum of shelled.py:663-691), so the
    integrals of the segments fill exactly the shell's rows.  Each segment
    carries ``cn`` = coefficient x radial_norm per kept primitive."""
    out = []
    for idx, sh in enumerate(shells):
        l = int(sh["angular_momentum"])
        nc = int(sh["n_components"])
        exps = np.asarray(sh["exponents"], dtype=np.float64)
        for r, row in enumerate(np.atleast_2d(np.asarray(sh["coefficients"], dtype=np.float64))):
            keep = np.nonzero(row != 0.0)[0]
            if keep.size == 0:
                raise UnsupportedBasis(f"shell {idx}: contraction row {r} is all zero")
            out.append({
                "shell": idx,
                "atom_idx": int(sh["atom_idx"]),
                "atom_pos": np.asarray(sh["atom_pos"], dtype=np.float64),
                "l": l,
                "exponents": exps[keep],
                "cn": row[keep] * radial_norm(exps[keep], l),
                "ao_start": int(sh["ao_start"]) + r * nc,
                "n_ao": nc,
            })
    return out


def spherical_transform(shells: List[Dict]) -> np.ndarray:
    """The reference's (sphere_total_ao x total_ao) matrix A =
    independent(shells, sphere_total_ao, I) (shelled.py:878-920, :1071): s and
    p rows copied, each d contraction's six Cartesian rows (xx, xy, yy, xz, yz,
    zz) mapped to xy, xz, yz, sqrt(3)/2 (xx - yy), zz - (xx + yy)/2, and f
    likewise to its seven combinations."""
    n_cart = int(shells[-1]["ao_stop"]) if shells else 0
    n_sph = int(shells[-1]["sphere_ao_stop"]) if shells else 0
    A = np.zeros((n_sph, n_cart))
    s2, s3, s5, s6, s10, s30 = (math.sqrt(x) for x in (2.0, 3.0, 5.0, 6.0, 10.0, 30.0))
    rows = {
        2: [{1: 1.0}, {3: 1.0}, {4: 1.0}, {0: s3 / 2, 2: -s3 / 2}, {5: 1.0, 0: -0.5, 2: -0.5}],
        3: [{4: -3 * s5 / 10, 6: -3 * s5 / 10, 9: 1.0},
            {0: -s6 / 4, 2: -s30 / 20, 7: s30 / 5},
            {1: -s30 / 20, 3: -s6 / 4, 8: s30 / 5},
            {4: s3 / 2, 6: -s3 / 2},
            {5: 1.0},
            {0: s10 / 4, 2: -3 * s2 / 4},
            {1: 3 * s2 / 4, 3: -s10 / 4}],
    }
    for sh in shells:
        l = int(sh["angular_momentum"])
        c0, s0 = int(sh["ao_start"]), int(sh["sphere_ao_start"])
        if l <= 1:
            for k in range(int(sh["n_ao"])):
                A[s0 + k, c0 + k] = 1.0
            continue
        if l not in rows:
            raise UnsupportedBasis(f"spherical transform for l = {l}")
        nc, ns = int(sh["n_components"]), 2 * l + 1
        for r in range(int(sh["n_contractions"])):
            for i, row in enumerate(rows[l]):
                for k, v in row.items():
                    A[s0 + r * ns + i, c0 + r * nc + k] = v
    return A
