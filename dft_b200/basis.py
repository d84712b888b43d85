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
    """The basis needs something the s/p kernels do not provide."""


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


def check_supported(shells: List[Dict]) -> None:
    """The ERI/J-K kernels handle s and p shells with one contraction."""
    for k, sh in enumerate(shells):
        if sh["angular_momentum"] > 1:
            raise UnsupportedBasis(f"shell {k}: l = {sh['angular_momentum']} (kernels cover s and p)")
        if sh["n_contractions"] != 1:
            raise UnsupportedBasis(f"shell {k}: {sh['n_contractions']} contractions (kernels need 1)")
