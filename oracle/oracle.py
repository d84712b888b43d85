"""CPU oracle for the integral / Fock-build path -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` leg of
``bench.py`` may import this module, and only as the checker.  The product
(``dft_b200``) never imports it; its CUDA path fails loudly without its own
library instead of falling back here.

It restates the reference (yegor-gondhal/DFT, ``shelled.py``) on the CPU:

* host logic in NumPy -- shell construction and normalisation
  (shelled.py:49-77, :88-101, :934-952), pair and quartet enumeration
  (shelled.py:599-603, :962-964, :1059), the class sort of ``process_eri``
  (shelled.py:727-762) and the UHF SCF loop with damping and DIIS
  (shelled.py:1079-1293);
* the arithmetic in plain C (``oracle.c``): Boys, Hermite E/R, primitive and
  contracted ERIs, one-electron S/T/V, and J/K digestion.

* orbital densities on a grid of points (the reference's evaluation script,
  shelled_eval.py:88-131) in NumPy: ``grid_ao``, ``grid_densities``.

Pinned by ``tests/test_oracle_golden.py`` and ``tests/test_oracle_grid.py``
against fixtures generated by running the reference itself
(``tests/golden/make_golden.py``).
"""
from __future__ import annotations

import ctypes
import json
import math
import os
import subprocess
from typing import Callable, Dict, List, Sequence, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_LIB_PATH = os.path.join(HERE, "_ref", "libref.so")

_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = ctypes.CDLL(LIB_PATH)
        for name in ("orc_boys", "orc_hermite_E", "orc_hermite_R", "orc_pair_prims",
                     "orc_eri_prims", "orc_eri_quartets", "orc_fill_matrices",
                     "orc_direct_jk", "orc_one_electron"):
            getattr(_lib, name).restype = None
        _lib.orc_num_threads.restype = ctypes.c_int
    return _lib


def _p(a: np.ndarray):
    return ctypes.c_void_p(a.ctypes.data)


# --------------------------------------------------------------------------- shells
def combinations(l: int) -> List[List[int]]:
    """Cartesian components in the reference's order (shelled.py:15-23)."""
    out = []
    for n in range(l + 1):
        for m in range(l + 1):
            for i in range(l + 1):
                if i + m + n == l:
                    out.append([i, m, n])
    return out


def double_factorial(x: np.ndarray) -> np.ndarray:
    """(x)!! through the Gamma function (shelled.py:88-92)."""
    x = np.asarray(x, dtype=np.float64)
    term = np.power(2.0, x / 2.0) * np.array([math.gamma(v / 2.0 + 1.0) for v in x.ravel()]).reshape(x.shape)
    odd = (x % 2.0) != 0.0
    term[odd] *= math.sqrt(2.0 / math.pi)
    return term


def normal(alpha: np.ndarray, pow_: np.ndarray) -> np.ndarray:
    """Primitive normalisation (shelled.py:95-101)."""
    term = np.power(4.0 * alpha, pow_.sum(axis=1))
    for k in range(3):
        term = term / double_factorial(2 * pow_[:, k] - 1)
    return np.sqrt(term) * np.power(2.0 * alpha / math.pi, 0.75)


def load_basis(path: str) -> Dict:
    with open(path) as fh:
        return json.load(fh)


def build_shells(basis: Dict, atoms: Sequence[str], centers: np.ndarray) -> List[Dict]:
    """Shell dicts with the reference's keys (shelled.py:49-77, :934-952)."""
    shells = []
    for i, atom in enumerate(atoms):
        for entry in basis[str(atom)]:
            ls, exps, coefs = entry
            if len(ls) == 1:
                parts = [(ls[0], coefs)]
            elif len(ls) == len(coefs):
                parts = [(m, [row]) for m, row in zip(ls, coefs)]
            else:
                raise ValueError("basis entry with mismatched momenta/coefficients")
            for m, rows in parts:
                shells.append({
                    "atom_idx": i,
                    "atom_pos": np.array(centers[i], dtype=np.float64),
                    "angular_momentum": int(m),
                    "exponents": np.array(exps, dtype=np.float64),
                    "coefficients": np.array(rows, dtype=np.float64),
                })
    total = 0
    for sh in shells:
        sh["components"] = np.array(combinations(sh["angular_momentum"]), dtype=np.int32)
        sh["n_components"] = len(sh["components"])
        sh["n_contractions"] = sh["coefficients"].shape[0]
        sh["n_ao"] = sh["n_components"] * sh["n_contractions"]
        sh["n_exponents"] = sh["exponents"].size
        sh["ao_start"] = total
        sh["ao_stop"] = total + sh["n_ao"]
        e = np.tile(sh["exponents"], sh["n_components"])
        pw = np.repeat(sh["components"], sh["n_exponents"], axis=0).reshape(-1, 3)
        sh["normalization"] = normal(e, pw)
        total = sh["ao_stop"]
    return shells


class ShellArrays:
    """Flat shell arrays in the layout ``oracle.c`` reads."""

    def __init__(self, shells: List[Dict]):
        self.ns = len(shells)
        self.center = np.ascontiguousarray([s["atom_pos"] for s in shells], dtype=np.float64).reshape(-1)
        self.l = np.array([s["angular_momentum"] for s in shells], dtype=np.int32)
        self.nexp = np.array([s["n_exponents"] for s in shells], dtype=np.int32)
        self.ncontr = np.array([s["n_contractions"] for s in shells], dtype=np.int32)
        self.ao = np.array([s["ao_start"] for s in shells], dtype=np.int32)
        self.nao = np.array([s["n_ao"] for s in shells], dtype=np.int32)
        self.exps = np.concatenate([s["exponents"] for s in shells]).astype(np.float64)
        self.coefs = np.concatenate([s["coefficients"].ravel() for s in shells]).astype(np.float64)
        self.exp_off = np.concatenate([[0], np.cumsum(self.nexp)[:-1]]).astype(np.int32)
        sizes = self.nexp * self.ncontr
        self.coef_off = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int32)
        self.N = int(shells[-1]["ao_stop"]) if shells else 0

    def args(self):
        return (ctypes.c_int(self.ns), _p(self.center), _p(self.l), _p(self.nexp), _p(self.ncontr),
                _p(self.exp_off), _p(self.coef_off), _p(self.ao), _p(self.exps), _p(self.coefs))


# --------------------------------------------------------------------------- enumeration
def pair_list(n_shells: int) -> List[Tuple[int, int]]:
    """Shell pairs (i, j), j <= i, row-major lower triangle (shelled.py:962-964, :1059)."""
    return [(i, j) for i in range(n_shells) for j in range(i + 1)]


def quartet_list(n_shells: int) -> np.ndarray:
    """Unique quartets (a, b, c, d) in calc_eri order: cd_idx <= ab_idx (shelled.py:634-638)."""
    pl = np.array(pair_list(n_shells), dtype=np.int32)
    npair = pl.shape[0]
    ab = np.repeat(np.arange(npair), np.arange(1, npair + 1))
    cd = np.concatenate([np.arange(k + 1) for k in range(npair)]) if npair else np.zeros(0, int)
    return np.ascontiguousarray(np.hstack([pl[ab], pl[cd]]).astype(np.int32))


def quartet_offsets(shells: List[Dict], quads: np.ndarray) -> np.ndarray:
    nao = np.array([s["n_ao"] for s in shells], dtype=np.int64)
    sizes = nao[quads[:, 0]] * nao[quads[:, 1]] * nao[quads[:, 2]] * nao[quads[:, 3]]
    return np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)


def process_order(shells: List[Dict], quads: np.ndarray) -> np.ndarray:
    """Stable lexsort by (n_ao_a, n_ao_b, n_ao_c, n_ao_d) (shelled.py:727)."""
    nao = np.array([s["n_ao"] for s in shells])
    shp = nao[quads]
    return np.lexsort((shp[:, 3], shp[:, 2], shp[:, 1], shp[:, 0]))


# --------------------------------------------------------------------------- arithmetic
def boys(n: int, T: float) -> np.ndarray:
    F = np.zeros(max(n, 1))
    lib().orc_boys(ctypes.c_int(n), ctypes.c_double(T), _p(F))
    return F[:n]


def eri_quartets(shells: List[Dict], quads: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
    """Contracted ERI blocks, block t at values[offsets[t]:offsets[t+1]]."""
    sa = ShellArrays(shells)
    quads = np.ascontiguousarray(quads, dtype=np.int32)
    off = quartet_offsets(shells, quads)
    out = np.zeros(int(off[-1]))
    lib().orc_eri_quartets(*sa.args(), ctypes.c_long(quads.shape[0]), _p(quads), _p(off), _p(out))
    return out, off


def one_electron(shells: List[Dict], atoms: Sequence[str], centers: np.ndarray):
    sa = ShellArrays(shells)
    Z = np.array([int(a) for a in atoms], dtype=np.int32)
    xyz = np.ascontiguousarray(centers, dtype=np.float64).reshape(-1)
    N = sa.N
    S, T, V = (np.zeros((N, N)) for _ in range(3))
    lib().orc_one_electron(*sa.args(), ctypes.c_int(len(Z)), _p(Z), _p(xyz), ctypes.c_int(N),
                           _p(S), _p(T), _p(V))
    return S, T, V


def fill_matrices(shells, quads, values, offsets, P, P_a, P_b):
    """J, K_a, K_b from stored blocks (fill_matrices, shelled.py:770-877)."""
    sa = ShellArrays(shells)
    N = sa.N
    J, Ka, Kb = (np.zeros((N, N)) for _ in range(3))
    P, P_a, P_b = (np.ascontiguousarray(x, dtype=np.float64) for x in (P, P_a, P_b))
    quads = np.ascontiguousarray(quads, dtype=np.int32)
    offsets = np.ascontiguousarray(offsets, dtype=np.int64)
    values = np.ascontiguousarray(values, dtype=np.float64)
    lib().orc_fill_matrices(*sa.args(), ctypes.c_long(quads.shape[0]), _p(quads), _p(offsets),
                            _p(values), ctypes.c_int(N), _p(P), _p(P_a), _p(P_b), _p(J), _p(Ka), _p(Kb))
    return J, Ka, Kb


def direct_jk(shells, quads, P, P_a, P_b, sa=None):
    """Integral-direct J, K_a, K_b over the given unique quartets (``sa``: the
    molecule's ShellArrays, built here when not given)."""
    sa = sa if sa is not None else ShellArrays(shells)
    N = sa.N
    J, Ka, Kb = (np.zeros((N, N)) for _ in range(3))
    P, P_a, P_b = (np.ascontiguousarray(x, dtype=np.float64) for x in (P, P_a, P_b))
    quads = np.ascontiguousarray(quads, dtype=np.int32)
    lib().orc_direct_jk(*sa.args(), ctypes.c_long(quads.shape[0]), _p(quads), ctypes.c_int(N),
                        _p(P), _p(P_a), _p(P_b), _p(J), _p(Ka), _p(Kb))
    return J, Ka, Kb


def direct_jk_reference_kernel(shells, quads, P, P_a, P_b, ref=None, sa=None):
    """direct_jk with the primitive ERIs from the reference's own eri_kernel
    (oracle/_ref), contraction and digestion from the restatement."""
    ref = ref if ref is not None else ref_lib()
    if ref is None:
        raise RuntimeError("oracle/_ref/libref.so not built")
    sa = sa if sa is not None else ShellArrays(shells)
    N = sa.N
    J, Ka, Kb = (np.zeros((N, N)) for _ in range(3))
    P, P_a, P_b = (np.ascontiguousarray(x, dtype=np.float64) for x in (P, P_a, P_b))
    quads = np.ascontiguousarray(quads, dtype=np.int32)
    fn = ctypes.cast(ref.ref_run_eri_kernel, ctypes.c_void_p)
    lib().orc_direct_jk_fn.restype = None
    lib().orc_direct_jk_fn(*sa.args(), ctypes.c_long(quads.shape[0]), _p(quads), ctypes.c_int(N),
                           _p(P), _p(P_a), _p(P_b), _p(J), _p(Ka), _p(Kb), fn)
    return J, Ka, Kb


def full_eri_tensor(shells: List[Dict]) -> np.ndarray:
    """Dense (N,N,N,N) ERI tensor from the unique quartets (small N only)."""
    quads = quartet_list(len(shells))
    vals, off = eri_quartets(shells, quads)
    N = shells[-1]["ao_stop"]
    eri = np.zeros((N, N, N, N))
    for t, (a, b, c, d) in enumerate(quads):
        sl = [slice(shells[k]["ao_start"], shells[k]["ao_stop"]) for k in (a, b, c, d)]
        blk = vals[off[t]:off[t + 1]].reshape([shells[k]["n_ao"] for k in (a, b, c, d)])
        for perm, arr in (((0, 1, 2, 3), blk), ((1, 0, 2, 3), blk.transpose(1, 0, 2, 3)),
                          ((0, 1, 3, 2), blk.transpose(0, 1, 3, 2)),
                          ((1, 0, 3, 2), blk.transpose(1, 0, 3, 2)),
                          ((2, 3, 0, 1), blk.transpose(2, 3, 0, 1)),
                          ((3, 2, 0, 1), blk.transpose(3, 2, 0, 1)),
                          ((2, 3, 1, 0), blk.transpose(2, 3, 1, 0)),
                          ((3, 2, 1, 0), blk.transpose(3, 2, 1, 0))):
            eri[sl[perm[0]], sl[perm[1]], sl[perm[2]], sl[perm[3]]] = arr
    return eri


# --------------------------------------------------------------------------- SCF
def spherical_transform(shells: List[Dict]) -> np.ndarray:
    """The reference's A = independent(shells, sphere_total_ao, I)
    (shelled.py:878-920, :1071), restated row by row for s, p, d and f."""
    n_cart = sum(int(s["n_ao"]) for s in shells)
    n_sph = sum(int(s["n_contractions"]) * (2 * int(s["angular_momentum"]) + 1) for s in shells)
    A = np.zeros((n_sph, n_cart))
    r = 0
    for sh in shells:
        l, c0 = int(sh["angular_momentum"]), int(sh["ao_start"])
        for k in range(int(sh["n_contractions"])):
            c = c0 + k * int(sh["n_components"])
            if l <= 1:
                for m in range(2 * l + 1):
                    A[r + m, c + m] = 1.0
            elif l == 2:
                A[r, c + 1] = 1.0
                A[r + 1, c + 3] = 1.0
                A[r + 2, c + 4] = 1.0
                A[r + 3, c] = np.sqrt(3) / 2
                A[r + 3, c + 2] = -np.sqrt(3) / 2
                A[r + 4, c + 5] = 1.0
                A[r + 4, c] = -0.5
                A[r + 4, c + 2] = -0.5
            elif l == 3:
                s2, s3, s5, s6, s10, s30 = (np.sqrt(x) for x in (2.0, 3.0, 5.0, 6.0, 10.0, 30.0))
                A[r, c + 4] = -3 * s5 / 10
                A[r, c + 6] = -3 * s5 / 10
                A[r, c + 9] = 1.0
                A[r + 1, c] = -s6 / 4
                A[r + 1, c + 2] = -s30 / 20
                A[r + 1, c + 7] = s30 / 5
                A[r + 2, c + 1] = -s30 / 20
                A[r + 2, c + 3] = -s6 / 4
                A[r + 2, c + 8] = s30 / 5
                A[r + 3, c + 4] = s3 / 2
                A[r + 3, c + 6] = -s3 / 2
                A[r + 4, c + 5] = 1.0
                A[r + 5, c] = s10 / 4
                A[r + 5, c + 2] = -3 * s2 / 4
                A[r + 6, c + 1] = 3 * s2 / 4
                A[r + 6, c + 3] = -s10 / 4
            else:
                raise ValueError("oracle spherical transform: s, p, d and f")
            r += 2 * l + 1
    return A


def scf_uhf(H: np.ndarray, S: np.ndarray, jk: Callable, n_alpha: int, n_beta: int, e_nn: float,
            etol: float = 1e-8, ptol: float = 1e-6, max_iter: int = 500, history: int = 10,
            A: np.ndarray = None):
    """The reference's UHF loop (shelled.py:1079-1293).

    With A (d shells) the loop runs in the spherical basis as the reference's
    does: S, H, J and K as A M A^T and the densities handed to jk as A^T P A
    (shelled.py:1071-1074, :1166-1176); without it A is the identity.
    Core-H guess, damping from rate 0.4 (divided by 1.1 after 4 strikes),
    DIIS on the commutator FPS - SPF once |dE| < 1e-3, convergence at
    |dE| < etol and max|dP| < ptol, then one rebuild with the last density.
    Returns a dict with the energy, densities and iteration count.
    """
    if A is not None:
        H, S = A @ H @ A.T, A @ S @ A.T
        jk_cart = jk

        def jk(P, Pa, Pb):
            out = jk_cart(A.T @ P @ A, A.T @ Pa @ A, A.T @ Pb @ A)
            return tuple(A @ M @ A.T for M in out)

    w, U = np.linalg.eigh(S)
    X = U @ np.diag(w ** -0.5) @ U.T
    _, Cp = np.linalg.eigh(X.T @ H @ X)
    C = X @ Cp
    P_a = C[:, :n_alpha] @ C[:, :n_alpha].T
    P_b = C[:, :n_beta] @ C[:, :n_beta].T
    N = H.shape[0]
    hist = {k: np.zeros((history, N, N)) for k in ("Pa", "Pb", "Fa", "Fb", "Ra", "Rb")}
    E_total, prev_dE, prev_dP = None, np.inf, np.inf
    rate, strikes, use_diis, count = 0.4, 0, False, 0
    while True:
        if count > max_iter:
            raise RuntimeError("oracle SCF did not converge")
        P = P_a + P_b
        J, Ka, Kb = jk(P, P_a, P_b)
        Fa, Fb = H + J - Ka, H + J - Kb
        for key, val in (("Pa", P_a), ("Pb", P_b), ("Fa", Fa), ("Fb", Fb),
                         ("Ra", Fa @ P_a @ S - S @ P_a @ Fa), ("Rb", Fb @ P_b @ S - S @ P_b @ Fb)):
            hist[key][1:] = hist[key][:-1].copy()
            hist[key][0] = val
        if use_diis:
            B = (np.einsum("iab,jab->ij", hist["Ra"], hist["Ra"]) +
                 np.einsum("iab,jab->ij", hist["Rb"], hist["Rb"]))
            lim = min(count + 1, history)
            try:
                c = np.linalg.solve(B[:lim, :lim], np.ones(lim))
            except np.linalg.LinAlgError:
                # exactly singular history (tight thresholds, nearly equal error
                # vectors): the reference would stop here; continue with the
                # least-squares coefficients
                c = np.linalg.lstsq(B[:lim, :lim], np.ones(lim), rcond=None)[0]
            c /= c.sum()
            Fa = np.einsum("i,iab->ab", c, hist["Fa"][:lim])
            Fb = np.einsum("i,iab->ab", c, hist["Fb"][:lim])
        E_new = 0.5 * np.sum(P * H + P_a * Fa + P_b * Fb) + e_nn
        dE = np.inf if E_total is None else abs(E_new - E_total)
        _, Ca = np.linalg.eigh(X.T @ Fa @ X)
        _, Cb = np.linalg.eigh(X.T @ Fb @ X)
        Ca, Cb = X @ Ca, X @ Cb
        Pa_new = rate * (Ca[:, :n_alpha] @ Ca[:, :n_alpha].T) + (1 - rate) * P_a
        Pb_new = rate * (Cb[:, :n_beta] @ Cb[:, :n_beta].T) + (1 - rate) * P_b
        dP = np.max(np.maximum(np.abs(Pa_new - P_a), np.abs(Pb_new - P_b)))
        if (dE > prev_dE or dP > prev_dP) and not use_diis:
            if strikes == 3:
                rate /= 1.1
                strikes = 0
            else:
                strikes += 1
        if dE < 1e-3:
            use_diis = True
        if dE < etol and dP < ptol:
            J, Ka, Kb = jk(P, P_a, P_b)
            Fa, Fb = H + J - Ka, H + J - Kb
            E_new = 0.5 * np.sum(P * H + P_a * Fa + P_b * Fb) + e_nn
            return {"energy": float(E_new), "P_a": P_a, "P_b": P_b, "iterations": count,
                    "J": J, "K_a": Ka, "K_b": Kb}
        E_total, prev_dE, prev_dP = E_new, dE, dP
        P_a, P_b = Pa_new, Pb_new
        count += 1


def electron_counts(atoms: Sequence[str], charge: int = 0, mult: int = 1) -> Tuple[int, int]:
    """N_a, N_b from the electron count and multiplicity (shelled.py:1081, :1099-1100)."""
    n = sum(int(a) for a in atoms) - charge
    return (n + mult - 1) // 2, (n - mult + 1) // 2


def ref_lib():
    """The reference's kernels compiled as host code (oracle/_ref), or None."""
    if not os.path.exists(REF_LIB_PATH):
        return None
    lib_ = ctypes.CDLL(REF_LIB_PATH)
    for n in ("ref_run_nuclear_kernel", "ref_run_eri_kernel", "ref_run_eri_batch"):
        getattr(lib_, n).restype = None
    return lib_


# --------------------------------------------------------------------------- gradients
def nuclear_repulsion(atoms: Sequence[str], centers: np.ndarray) -> float:
    z = [int(a) for a in atoms]
    e = 0.0
    for i in range(len(z)):
        for j in range(i):
            e += z[i] * z[j] / float(np.linalg.norm(centers[i] - centers[j]))
    return e


def nuclear_repulsion_gradient(atoms: Sequence[str], centers: np.ndarray) -> np.ndarray:
    z = [int(a) for a in atoms]
    g = np.zeros((len(z), 3))
    for i in range(len(z)):
        for j in range(len(z)):
            if i != j:
                d = centers[i] - centers[j]
                g[i] -= z[i] * z[j] * d / float(np.linalg.norm(d)) ** 3
    return g


def gradient(shells: List[Dict], atoms: Sequence[str], centers: np.ndarray, D, Da, Db, W) -> np.ndarray:
    """Total nuclear gradient (n_atoms, 3): electronic part from orc_gradient
    (explicit derivative integrals on every centre) plus nuclear repulsion."""
    sa = ShellArrays(shells)
    Z = np.array([int(a) for a in atoms], dtype=np.int32)
    xyz = np.ascontiguousarray(centers, dtype=np.float64).reshape(-1)
    shell_atom = np.array([s["atom_idx"] for s in shells], dtype=np.int32)
    D, Da, Db, W = (np.ascontiguousarray(x, dtype=np.float64) for x in (D, Da, Db, W))
    g = np.zeros(3 * len(Z))
    lib().orc_gradient(*sa.args(), _p(shell_atom), ctypes.c_int(len(Z)), _p(Z), _p(xyz), ctypes.c_int(sa.N),
                       _p(D), _p(Da), _p(Db), _p(W), _p(g))
    return g.reshape(-1, 3) + nuclear_repulsion_gradient(atoms, np.asarray(centers, dtype=np.float64))


def scf_energy_gradient(basis_path: str, atoms: Sequence[str], centers: np.ndarray, etol: float = 1e-12,
                        ptol: float = 1e-10, with_gradient: bool = True):
    """Oracle SCF (the reference's loop with oracle J/K) and, optionally, its
    analytic gradient with W = P_a F_a P_a + P_b F_b P_b (valid at convergence)."""
    centers = np.asarray(centers, dtype=np.float64)
    sh = build_shells(load_basis(basis_path), list(atoms), centers)
    S, T, V = one_electron(sh, atoms, centers)
    H = T + V
    q = quartet_list(len(sh))
    na, nb = electron_counts(atoms)
    r = scf_uhf(H, S, lambda P, Pa, Pb: direct_jk(sh, q, P, Pa, Pb), na, nb, nuclear_repulsion(atoms, centers),
                etol=etol, ptol=ptol)
    if not with_gradient:
        return r["energy"], None
    Pa, Pb = r["P_a"], r["P_b"]
    Fa, Fb = H + r["J"] - r["K_a"], H + r["J"] - r["K_b"]
    W = Pa @ Fa @ Pa + Pb @ Fb @ Pb
    return r["energy"], gradient(sh, atoms, centers, Pa + Pb, Pa, Pb, W)


# ------------------------------------------------------------------ grid
def grid_ao(shells: List[Dict], points: np.ndarray) -> np.ndarray:
    """AO values (total_ao, n_points) at FP32 points (shelled_eval.py:91-107):
    per shell, Cartesian component (i, j, k), primitive p and contraction c,
    coefficient[c, p] * normalization[comp, p] * x^i y^j z^k exp(-alpha_p r^2)
    summed over p, with (x, y, z) the FP64 difference of the FP32 point and
    the shell centre."""
    pts = np.asarray(points, dtype=np.float32)
    n_ao = int(shells[-1]["ao_stop"]) if shells else 0
    out = np.empty((n_ao, pts.shape[0]))
    for sh in shells:
        d = pts.astype(np.float64) - np.asarray(sh["atom_pos"], dtype=np.float64)
        r2 = d[:, 0] ** 2 + d[:, 1] ** 2 + d[:, 2] ** 2
        nexp = int(sh["n_exponents"])
        comps = np.asarray(sh["components"])
        norm = np.asarray(sh["normalization"]).reshape(len(comps), nexp)
        coef = np.asarray(sh["coefficients"]).reshape(-1, nexp)
        gauss = np.exp(-np.asarray(sh["exponents"], dtype=np.float64)[:, None] * r2[None, :])  # (nexp, n)
        row = int(sh["ao_start"])
        for c in range(coef.shape[0]):
            for a, (i, j, k) in enumerate(comps):
                poly = d[:, 0] ** i * d[:, 1] ** j * d[:, 2] ** k
                out[row] = ((coef[c] * norm[a])[:, None] * gauss).sum(axis=0) * poly
                row += 1
    return out


def grid_densities(ckpt: Dict, points: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
    """(total, phase), each (max(N_a, N_b), n_points) FP32, from an evaluation
    checkpoint (shelled_eval.py:108-131): psi_s = C_s[:, :n]^T (rounded to
    FP32, applied in FP64) A ao; total = [k < N_a] psi_a^2 + [k < N_b] psi_b^2;
    phase = psi_a in rows k < N_a, zero elsewhere."""
    n_a, n_b = int(ckpt["N_a"]), int(ckpt["N_b"])
    n = max(n_a, n_b)
    ao = np.asarray(ckpt["A"], dtype=np.float64) @ grid_ao(ckpt["shells"], points)
    psi = [np.asarray(ckpt[k]).astype(np.float32)[:, :n].T.astype(np.float64) @ ao for k in ("C_a", "C_b")]
    occ_a = (np.arange(n) < n_a)[:, None]
    occ_b = (np.arange(n) < n_b)[:, None]
    total = (np.where(occ_a, psi[0] ** 2, 0.0) + np.where(occ_b, psi[1] ** 2, 0.0)).astype(np.float32)
    phase = np.zeros((n, ao.shape[1]), dtype=np.float32)
    phase[:n_a] = psi[0][:n_a]
    return total, phase
