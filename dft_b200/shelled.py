"""Drop-in for the integral path of the reference's ``shelled.py``.

Same names, argument meanings and in-place semantics as the reference's
functions, backed by ``libdftk.so``:

=====================================  ====================================================
this module                             reference (shelled.py)
=====================================  ====================================================
``combinations``, ``normal``            :15-23, :95-101
``build_shells(basis, atoms, centers)`` shell construction and metadata :49-77, :934-952
``nuclear_repulsion(Z, centers)``       :157-163
``one_electron(shells, atoms, centers)`` S, T, V block loop :961-1069
``pair_data(shells, atoms, centers)``   ``pair_list`` / ``pair_cache`` :958-1059
``nuclear_kernel``, ``eri_kernel``      RawKernels :350-532 (launch :1015, :642)
``calc_eri(pair_list, pair_cache, shells)``  :596-700 (returns the arrays; writes the .npy files if asked)
``process_eri(...)``                    :702-768
``fill_matrices(shells, P, P_a, P_b, J, K_a, K_b)``  :770-877 (integral-direct, in place)
``independent(shells, sphere_total_ao, C)``  :878-920
``UHF_density``, ``init_UHF_density``   :549-574
``scf(...)``                            the SCF loop :1079-1293
=====================================  ====================================================

Densities and Fock blocks may be NumPy arrays or CUDA tensors; results come
back in the same kind.  Nothing here runs on the CPU except host bookkeeping
(quartet ordering, the class sort of ``process_eri``).
"""
from __future__ import annotations

import os
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch

from . import _lib, basis as _basis, geometry as _geometry
from .basis import build_shells, combinations, load_basis, normal  # noqa: F401  (re-exported API)
from .engine import IntegralEngine
from .scf import SCFResult, scf_reference, scf_rhf

_ENGINES: Dict[Tuple, IntegralEngine] = {}


def _fingerprint(shells: List[Dict]) -> Tuple:
    """Value key of a shell list (momenta, AO offsets, centres to 1e-12,
    exponents, coefficients): a call with equal shells finds the cached engine,
    a changed geometry or basis builds a new one."""
    meta = tuple((s["angular_momentum"], s["ao_start"]) for s in shells)
    pos = np.round(np.array([np.ravel(s["atom_pos"]) for s in shells], dtype=np.float64), 12).tobytes()
    ex = tuple(tuple(np.asarray(s["exponents"], dtype=np.float64).tolist()) for s in shells)
    co = tuple(tuple(np.asarray(s["coefficients"], dtype=np.float64).ravel().tolist()) for s in shells)
    return (meta, pos, ex, co)


def get_engine(shells: List[Dict], tau_schwarz: float = 1e-12) -> IntegralEngine:
    """The cached engine for this shell list (built on first use)."""
    key = (_fingerprint(shells), tau_schwarz, torch.cuda.current_device() if torch.cuda.is_available() else -1)
    eng = _ENGINES.get(key)
    if eng is None:
        eng = IntegralEngine(shells, tau_schwarz=tau_schwarz)
        _ENGINES[key] = eng
    return eng


def nuclear_repulsion(Z, centers) -> float:
    """sum_{i<j} Z_i Z_j / |R_i - R_j| (shelled.py:157-163)."""
    return _geometry.nuclear_repulsion([str(int(z)) for z in np.asarray(Z).ravel()], np.asarray(centers))


def one_electron(shells: List[Dict], atoms: Sequence[str], centers):
    """(S, T, V) as CUDA tensors for all shell pairs (shelled.py:961-1069)."""
    return get_engine(shells).one_electron(atoms, centers)


# ------------------------------------------------------------------ RawKernels
class _DropInKernel:
    """Callable as ``kernel((blocks,), (threads,), args)`` like a CuPy RawKernel.

    The launch shape is chosen by the library (it covers exactly the threads
    the reference's grid guard keeps); ``args`` are CUDA tensors and ints in
    the reference's order."""

    def __init__(self, name: str, n_ptr_args: Sequence[bool]):
        self.name = name
        self.kinds = n_ptr_args

    def __call__(self, grid, block, args):
        if len(args) != len(self.kinds):
            raise _lib.DftkError(self.name, _lib.ERR_ARG, f"expected {len(self.kinds)} arguments")
        conv = [(_lib.ptr(a) if is_ptr else int(a)) for a, is_ptr in zip(args, self.kinds)]
        _lib.call(self.name, *conv, _lib.stream_handle())


# nuclear_kernel(exp_a, exp_b, cen_a, cen_b, pow_a, pow_b, atoms, atom_centers, num_atoms,
#                num_funcs_a, num_funcs_b, V, Ex, Ey, Ez, p, P, nx, ny, nz)   (shelled.py:350-371)
nuclear_kernel = _DropInKernel("dftk_nuclear_kernel", [True] * 8 + [False] * 3 + [True] * 9)
# eri_kernel(K_ab, p, P, Ex, Ey, Ez, nx, ny, nz, K_cd, p, P, Ex, Ey, Ez, nx, ny, nz, out)  (:452-473)
eri_kernel = _DropInKernel("dftk_eri_kernel", [False] + [True] * 8 + [False] + [True] * 9)


# ----------------------------------------------------------------- pair data
class PairCache(dict):
    """``pair_cache[(i, j)]`` of the reference (shelled.py:1047-1058), filled
    lazily through the drop-in nuclear_kernel: keys K, p, P, Ex, Ey, Ez, nx,
    ny, nz (and V, the primitive nuclear attraction)."""

    def __init__(self, shells, atoms, centers, pair_list):
        super().__init__()
        self._shells = shells
        self._Z = torch.as_tensor(np.array([int(a) for a in atoms], dtype=np.int32)).cuda()
        self._centers = torch.as_tensor(np.asarray(centers, dtype=np.float64)).cuda()
        self._keys = set(pair_list)

    def __contains__(self, key):
        return key in self._keys

    def __missing__(self, key):
        if key not in self._keys:
            raise KeyError(key)
        i, j = key
        sa, sb = self._shells[i], self._shells[j]
        dev = self._Z.device
        ea = torch.as_tensor(np.tile(sa["exponents"], sa["n_components"]), device=dev)
        eb = torch.as_tensor(np.tile(sb["exponents"], sb["n_components"]), device=dev)
        pa = torch.as_tensor(np.repeat(sa["components"], sa["n_exponents"], axis=0).reshape(-1, 3).astype(np.int32), device=dev)
        pb = torch.as_tensor(np.repeat(sb["components"], sb["n_exponents"], axis=0).reshape(-1, 3).astype(np.int32), device=dev)
        ca = torch.as_tensor(np.asarray(sa["atom_pos"], dtype=np.float64), device=dev)
        cb = torch.as_tensor(np.asarray(sb["atom_pos"], dtype=np.float64), device=dev)
        na, nb = int(ea.numel()), int(eb.numel())
        K = na * nb
        f64 = dict(dtype=torch.float64, device=dev)
        rec = {"K": K, "V": torch.empty(K, **f64), "Ex": torch.empty(K * 7, **f64), "Ey": torch.empty(K * 7, **f64),
               "Ez": torch.empty(K * 7, **f64), "p": torch.empty(K, **f64), "P": torch.empty(K * 3, **f64),
               "nx": torch.empty(K, dtype=torch.int32, device=dev), "ny": torch.empty(K, dtype=torch.int32, device=dev),
               "nz": torch.empty(K, dtype=torch.int32, device=dev)}
        nuclear_kernel(None, None, (ea, eb, ca, cb, pa, pb, self._Z, self._centers, int(self._Z.numel()), na, nb,
                                    rec["V"], rec["Ex"], rec["Ey"], rec["Ez"], rec["p"], rec["P"], rec["nx"],
                                    rec["ny"], rec["nz"]))
        self[key] = rec
        return rec


def pair_data(shells: List[Dict], atoms: Sequence[str], centers) -> Tuple[List[Tuple[int, int]], PairCache]:
    """``pair_list`` (i, j), j <= i in row-major order, and a lazy ``pair_cache``."""
    pair_list = [(i, j) for i in range(len(shells)) for j in range(i + 1)]
    return pair_list, PairCache(shells, atoms, centers, pair_list)


# ------------------------------------------------------------------ ERIs
def quartet_list(pair_list: Sequence[Tuple[int, int]]) -> np.ndarray:
    """Quartets (a, b, c, d) in calc_eri order: cd_idx <= ab_idx (shelled.py:599-603, :634-638)."""
    pl = np.asarray(pair_list, dtype=np.int64).reshape(-1, 2)
    n = pl.shape[0]
    ab = np.repeat(np.arange(n), np.arange(1, n + 1))
    cd = np.concatenate([np.arange(k + 1) for k in range(n)]) if n else np.zeros(0, dtype=np.int64)
    return np.hstack([pl[ab], pl[cd]])


def calc_eri(pair_list, pair_cache, shells, out_dir: Optional[str] = None, quads: Optional[np.ndarray] = None):
    """Contracted ERI blocks of every unique quartet of ``pair_list``.

    Returns a dict with the reference's four arrays (``eri_values`` flat in
    quartet order, ``eri_indices`` [start, stop), ``eri_quads``,
    ``eri_quads_shapes``); with ``out_dir`` also writes them as
    ``out_dir/compute_eri/*.npy`` like the reference.  ``pair_cache`` is
    accepted for call-shape compatibility; the blocks come from the
    class-sorted engine data."""
    eng = get_engine(shells)
    if quads is None:
        quads = quartet_list(pair_list)
    vals, off = eng.eri_blocks(quads)
    nao = eng.nao_sh
    res = {
        "eri_values": vals.cpu().numpy(),
        "eri_indices": np.stack([off[:-1], off[1:]], axis=1).astype(np.int32),
        "eri_quads": quads.astype(np.int16),
        "eri_quads_shapes": nao[quads].astype(np.int16),
    }
    if out_dir is not None:
        d = os.path.join(out_dir, "compute_eri")
        os.makedirs(d, exist_ok=True)
        for k, v in res.items():
            np.save(os.path.join(d, k + ".npy"), v)
    return res


def process_eri(eri: Optional[dict] = None, out_dir: Optional[str] = None):
    """Stable class sort of the quartets by (n_ao_a, n_ao_b, n_ao_c, n_ao_d)
    and the block table (shelled.py:702-768)."""
    if eri is None:
        d = os.path.join(out_dir or ".", "compute_eri")
        eri = {k: np.load(os.path.join(d, k + ".npy")) for k in
               ("eri_values", "eri_indices", "eri_quads", "eri_quads_shapes")}
    shp = eri["eri_quads_shapes"]
    order = np.lexsort((shp[:, 3], shp[:, 2], shp[:, 1], shp[:, 0]))
    idx = eri["eri_indices"][order].astype(np.int64)
    sizes = idx[:, 1] - idx[:, 0]
    new_off = np.concatenate([[0], np.cumsum(sizes)])
    gather = np.concatenate([np.arange(s, e) for s, e in idx]) if idx.shape[0] else np.zeros(0, dtype=np.int64)
    shp_sorted = shp[order]
    change = np.nonzero(np.any(np.diff(shp_sorted, axis=0) != 0, axis=1))[0] + 1 if shp_sorted.shape[0] > 1 else \
        np.zeros(0, dtype=np.int64)
    starts = np.concatenate([[0], change])
    stops = np.concatenate([change, [shp_sorted.shape[0]]])
    res = {
        "processed_eri_values": eri["eri_values"][gather],
        "processed_eri_indices": np.stack([new_off[:-1], new_off[1:]], axis=1).astype(np.int32),
        "processed_eri_quads": eri["eri_quads"][order].astype(np.int32),
        "block_idxs": np.stack([starts, stops], axis=1),
        "chunked_quad_shape": shp_sorted[starts],
    }
    if out_dir is not None:
        d = os.path.join(out_dir, "compute_eri")
        os.makedirs(d, exist_ok=True)
        for k, v in res.items():
            np.save(os.path.join(d, k + ".npy"), v)
    return res


# --------------------------------------------------------------------- J / K
def fill_matrices(shells, P, P_a, P_b, J_matrix, K_a, K_b, tau: float = 0.0):
    """Add the Coulomb and exchange matrices of (P, P_a, P_b) into J_matrix,
    K_a and K_b in place (shelled.py:770-877), integral-direct on the GPU.

    tau is the density-weighted Schwarz cut (0 keeps every quartet the
    engine's Schwarz prefix holds, like the reference's stored ERIs)."""
    eng = get_engine(shells)
    same = (P_a is P_b) or (np.shares_memory(P_a, P_b) if isinstance(P_a, np.ndarray) and isinstance(P_b, np.ndarray)
                            else False)
    J, Ka, Kb = eng.jk(P, P_a, None if same else P_b, uhf=not same, tau=tau)
    pairs = ((J_matrix, J), (K_a, Ka), (K_b, Kb))
    # host destinations: one device-to-host copy of the distinct results
    srcs = []
    for dst, src in pairs:
        if not isinstance(dst, torch.Tensor) and not any(src is x for x in srcs):
            srcs.append(src)
    host = torch.stack(srcs).cpu().numpy() if srcs else None
    for dst, src in pairs:
        if isinstance(dst, torch.Tensor):
            dst += src.to(dst.device, dst.dtype)
        else:
            dst += host[next(i for i, x in enumerate(srcs) if x is src)]


def independent(shells, sphere_total_ao, C):
    """Cartesian-to-spherical row transform (shelled.py:878-920): A @ C with
    the reference's A (s/p rows copied; d and f contractions mapped to their
    five and seven combinations, basis.spherical_transform)."""
    A = _basis.spherical_transform(shells)
    if A.shape[0] != int(sphere_total_ao):
        raise ValueError(f"sphere_total_ao {sphere_total_ao} != {A.shape[0]}")
    return A @ np.asarray(C, dtype=np.float64)


def init_UHF_density(C_a, C_b, N_a, N_b):
    """P_s = C_s[:, :N_s] C_s[:, :N_s]^T (shelled.py:549-559)."""
    return C_a[:, :int(N_a)] @ C_a[:, :int(N_a)].T, C_b[:, :int(N_b)] @ C_b[:, :int(N_b)].T


def UHF_density(C_a, C_b, N_a, N_b, old_P_a, old_P_b, rate):
    """Damped density rate * new + (1 - rate) * old (shelled.py:561-574)."""
    P_a, P_b = init_UHF_density(C_a, C_b, N_a, N_b)
    return rate * P_a + (1 - rate) * old_P_a, rate * P_b + (1 - rate) * old_P_b


# ------------------------------------------------------------------------ SCF
def scf(atoms: Sequence[str], centers, charge: int = 0, mult: int = 1, basis: Optional[dict] = None,
        method: str = "reference", **kw) -> SCFResult:
    """Integrals + SCF for a molecule.  method "reference" runs the reference's
    UHF loop; "rhf" runs the closed-shell DIIS(8) incremental driver."""
    shells = build_shells(basis if basis is not None else load_basis(), atoms, centers)
    eng = get_engine(shells)
    S, T, V = eng.one_electron(atoms, centers)
    H = T + V
    e_nn = _geometry.nuclear_repulsion(atoms, np.asarray(centers))
    n = _basis.n_electrons(atoms, charge)
    n_a, n_b = (n + mult - 1) // 2, (n - mult + 1) // 2
    if method == "reference":
        return scf_reference(eng, H, S, n_a, n_b, e_nn, **kw)
    if method == "rhf":
        if n_a != n_b:
            raise ValueError("rhf needs a closed shell")
        return scf_rhf(eng, H, S, n_a, e_nn, **kw)
    raise ValueError(f"unknown method {method}")
