"""Many molecules through one shell set: batched J/K builds, SCF and gradients.

The molecules' shells are concatenated into one ``dftk_shells_t`` with a
molecule table (``mol``, ``mol_mat``, ...): AO indices stay molecule-local and
every N x N matrix is the concatenation of the molecules' own n x n blocks
("packed" storage, block m at element offset ``mol_mat[m]``).  Shell pairs of
each pair class are grouped by molecule and sorted by descending Schwarz
factor within it; the candidate queue gives every bra row the ket segment of
its own molecule (``ket_base``), so one selection pass and one launch per
quartet class cover every molecule, and quartets never mix molecules.

:func:`scf_rhf_batch` iterates all molecules together on padded
(B, Nmax, Nmax) tensors (padding: identity overlap and zero coupling, so
padded functions never mix in).  Each iteration's Fock build is one replay of
a CUDA graph captured once (memset, shell-block density maxima, selection,
six class kernels, symmetrisation).  The new density comes from canonical
purification of the DIIS-extrapolated Fock matrix in the Cholesky-orthogonal
basis (Palser and Manolopoulos, Phys. Rev. B 58, 12704 (1998)): batched
matrix products only, no per-molecule eigensolver, with the padded levels
put at the top of each molecule's Gershgorin interval so they end up empty.
Molecules converge individually: a converged molecule's flag in
``mol_active`` (read by the selection pass inside the graph) drops its
quartets from later builds.
"""
from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch

from . import _lib
from . import basis as _basis
from . import geometry as _geometry
from .engine import QCLASS_PAIRS, IntegralEngine, _dev, candidate_offsets


def _prefix(x: np.ndarray) -> np.ndarray:
    return np.concatenate([[0], np.cumsum(x)[:-1]]).astype(np.int64)


def batch_row_offsets(q_bra: np.ndarray, seg_bra: np.ndarray, q_ket: np.ndarray, seg_ket: np.ndarray,
                      same_class: bool, tau: float) -> Tuple[np.ndarray, np.ndarray]:
    """Candidate row offsets and per-row ket bases of one quartet class of a
    batch.  Both pair lists hold each molecule's pairs contiguously
    (molecule m at seg[m]:seg[m+1]), sorted by descending Schwarz factor
    within the molecule; bra row r of molecule m pairs with the Schwarz-kept
    prefix of molecule m's ket segment, ket k of that row being ket pair
    ket_base[r] + k."""
    counts, kb = [], []
    for m in range(seg_bra.size - 1):
        qx = q_bra[seg_bra[m]:seg_bra[m + 1]]
        qy = q_ket[seg_ket[m]:seg_ket[m + 1]]
        if qx.size == 0:
            continue
        counts.append(np.diff(candidate_offsets(qx, qy, same_class, tau)))
        kb.append(np.full(qx.size, seg_ket[m], dtype=np.int32))
    cnt = np.concatenate(counts) if counts else np.zeros(0, dtype=np.int64)
    off = np.concatenate([[0], np.cumsum(cnt)]).astype(np.int64)
    kbase = np.concatenate(kb) if kb else np.zeros(0, dtype=np.int32)
    return off, kbase


def pack_index(mol_nao: np.ndarray, n_max: int) -> np.ndarray:
    """Position in the padded (B, n_max, n_max) layout of every element of
    the packed per-molecule blocks (block m: n_m x n_m row-major)."""
    idx = []
    for m, n in enumerate(np.asarray(mol_nao, dtype=np.int64)):
        r, c = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
        idx.append(m * n_max * n_max + r.reshape(-1) * n_max + c.reshape(-1))
    return np.concatenate(idx) if idx else np.zeros(0, dtype=np.int64)


class BatchEngine(IntegralEngine):
    """Integral engine over a batch of molecules given as (atoms, centres) pairs."""

    def __init__(self, molecules: Sequence[Tuple[Sequence[str], np.ndarray]], basis_data: Optional[Dict] = None,
                 tau_schwarz: float = 1e-12, tau_prim: float = 1e-15, device=None):
        _lib.load()
        self.device = _dev(device)
        basis_data = basis_data if basis_data is not None else _basis.load_basis()
        self.molecules = [([str(a) for a in atoms], np.asarray(c, dtype=np.float64).reshape(-1, 3))
                          for atoms, c in molecules]
        if not self.molecules:
            raise _lib.DftkError("batch", _lib.ERR_ARG, "empty batch")
        per = [_basis.build_shells(basis_data, a, c) for a, c in self.molecules]
        for sh in per:
            _basis.check_sp(sh, "batch")
        self.n_mol = len(per)
        self.mol_ns = np.array([len(s) for s in per], dtype=np.int64)
        self.mol_nao = np.array([int(s[-1]["ao_stop"]) for s in per], dtype=np.int64)
        self.mol_natom = np.array([len(a) for a, _ in self.molecules], dtype=np.int64)
        self.mol_shell0 = _prefix(self.mol_ns)
        self.mol_atom0 = _prefix(self.mol_natom)
        self.mol_mat = _prefix(self.mol_nao ** 2)
        self.mol_dsh = _prefix(self.mol_ns ** 2)
        self.mat_elems = int((self.mol_nao ** 2).sum())
        self.shells = [s for sh in per for s in sh]
        self.segs = _basis.segments(self.shells)  # s/p shells, one contraction each: one segment per shell
        self.general = False
        self.has_hl = False
        self.shell_mol = np.repeat(np.arange(self.n_mol), self.mol_ns)
        self.shell_atom = np.array([s["atom_idx"] for s in self.shells], dtype=np.int64) + \
            self.mol_atom0[self.shell_mol]
        self.ns = len(self.shells)
        self.n_ao = int(self.mol_nao.max())
        self.n_max = self.n_ao
        self.tau_schwarz = float(tau_schwarz)
        self.tau_prim = float(tau_prim)
        self.l = np.array([s["angular_momentum"] for s in self.shells], dtype=np.int32)
        self.nao_sh = np.array([s["n_ao"] for s in self.shells], dtype=np.int64)
        self.atoms = [a for atoms, _ in self.molecules for a in atoms]
        self.centers = np.concatenate([c for _, c in self.molecules], axis=0)
        with torch.cuda.device(self.device):
            _lib.call("dftk_init")
            self._upload_shells()
            self._upload_batch()
            self._build_pairs()
            self._build_queue()
            nbytes = _lib.load().dftk_workspace_bytes(ctypes.byref(self.c_shells), ctypes.byref(self.c_queue))
            self.workspace = torch.empty(int(nbytes), dtype=torch.uint8, device=self.device)
            self.workspace_bytes = int(nbytes)
            self.base_workspace_bytes = int(_lib.load().dftk_workspace_bytes(ctypes.byref(self.c_shells), None))
            self._build_packing()
        self.d_atom_xyz = self._t(self.centers.reshape(-1), torch.float64)
        self.d_atom_z = self._t(np.array([float(int(a)) for a in self.atoms]), torch.float64)
        self.d_shell_atom = self._t(self.shell_atom.astype(np.int32), torch.int32)

    # ------------------------------------------------------------------ setup
    def _upload_batch(self):
        self.d_mol = self._t(self.shell_mol.astype(np.int32), torch.int32)
        self.d_mol_mat = self._t(self.mol_mat, torch.int64)
        self.d_mol_nao = self._t(self.mol_nao.astype(np.int32), torch.int32)
        self.d_mol_shell0 = self._t(self.mol_shell0.astype(np.int32), torch.int32)
        self.d_mol_ns = self._t(self.mol_ns.astype(np.int32), torch.int32)
        self.d_mol_dsh = self._t(self.mol_dsh, torch.int64)
        self.d_mol_atom0 = self._t(self.mol_atom0.astype(np.int32), torch.int32)
        self.d_mol_natom = self._t(self.mol_natom.astype(np.int32), torch.int32)
        self.mol_active = torch.ones(self.n_mol, dtype=torch.uint8, device=self.device)
        c = self.c_shells
        c.n_ao = self.n_ao
        c.n_mol = self.n_mol
        c.max_ns = int(self.mol_ns.max())
        c.max_natom = int(self.mol_natom.max())
        c.mat_elems = self.mat_elems
        c.dsh_elems = int((self.mol_ns ** 2).sum())
        for name in ("mol", "mol_mat", "mol_nao", "mol_shell0", "mol_ns", "mol_dsh", "mol_atom0", "mol_natom"):
            setattr(c, name, _lib.ptr(getattr(self, "d_" + name)).value)

    def _build_pairs(self):
        ii_l, jj_l = [], []
        for m in range(self.n_mol):
            i, j = np.tril_indices(int(self.mol_ns[m]))
            ii_l.append(i + self.mol_shell0[m])
            jj_l.append(j + self.mol_shell0[m])
        ii = np.concatenate(ii_l).astype(np.int64)
        jj = np.concatenate(jj_l).astype(np.int64)
        swap = self.l[ii] < self.l[jj]
        a = np.where(swap, jj, ii)
        b = np.where(swap, ii, jj)
        pclass = self.l[a] + self.l[b]
        pmol = self.shell_mol[a]
        stream = _lib.stream_handle()
        self.pair_bufs, self.c_pairs_list, self.q_sorted, self.pair_seg = [], [], [], []
        for pc in range(3):
            sel = np.nonzero(pclass == pc)[0]
            ab = np.stack([a[sel], b[sel]], axis=1)
            mol = pmol[sel]
            bufs, st = self._alloc_class(pc, ab)
            if ab.shape[0]:
                _lib.call("dftk_pair_data", ctypes.byref(self.c_shells), pc, ctypes.byref(st), stream)
                _lib.call("dftk_schwarz", ctypes.byref(self.c_shells), pc, ctypes.byref(st), stream)
                q = bufs["q"][: ab.shape[0]].cpu().numpy()
                order = np.lexsort((-q, mol))  # by molecule, then descending Q
                ab, mol = ab[order], mol[order]
                bufs, st = self._alloc_class(pc, ab)
                _lib.call("dftk_pair_data", ctypes.byref(self.c_shells), pc, ctypes.byref(st), stream)
                _lib.call("dftk_schwarz", ctypes.byref(self.c_shells), pc, ctypes.byref(st), stream)
                self.q_sorted.append(bufs["q"][: ab.shape[0]].cpu().numpy())
            else:
                self.q_sorted.append(np.zeros(0))
            # first pair of each molecule in this class (n_mol + 1 entries)
            self.pair_seg.append(np.searchsorted(mol, np.arange(self.n_mol + 1)).astype(np.int64))
            self.pair_bufs.append(bufs)
            self.c_pairs_list.append(st)
        self.c_pairs = _lib.PairsArray(*self.c_pairs_list)
        self.n_pairs = [int(x.shape[0]) for x in self.q_sorted]

    def _build_queue(self):
        self.row_off, self.totals, self.ket_base = [], [], []
        q = _lib.Queue()
        for c, (X, Y) in enumerate(QCLASS_PAIRS):
            off, kbase = batch_row_offsets(self.q_sorted[X], self.pair_seg[X], self.q_sorted[Y], self.pair_seg[Y],
                                           X == Y, self.tau_schwarz)
            n_rows = off.size - 1
            if kbase.size == 0:
                kbase = np.zeros(1, dtype=np.int32)
            d_off = self._t(off, torch.int64)
            d_kb = self._t(kbase.astype(np.int32), torch.int32)
            self.row_off.append(d_off)
            self.ket_base.append(d_kb)
            self.totals.append(int(off[-1]))
            q.n_rows[c] = n_rows if off[-1] > 0 else 0
            q.total[c] = int(off[-1])
            q.row_off[c] = _lib.ptr(d_off).value
            q.ket_base[c] = _lib.ptr(d_kb).value
        q.tau_prim = self.tau_prim
        q.mol_active = _lib.ptr(self.mol_active).value
        self.c_queue = q

    def _build_packing(self):
        """Index of every packed element in the padded (B, Nmax, Nmax) layout."""
        B, Nm = self.n_mol, self.n_max
        self.pack_index = self._t(pack_index(self.mol_nao, Nm), torch.int64)
        self.packed_mol = self._t(np.repeat(np.arange(B), self.mol_nao ** 2), torch.int64)
        ar = np.arange(Nm)
        self.pad_mask = self._t((ar[None, :] >= self.mol_nao[:, None]).astype(np.float64), torch.float64)

    # ---------------------------------------------------------------- packing
    def to_padded(self, packed: torch.Tensor) -> torch.Tensor:
        out = torch.zeros(self.n_mol * self.n_max * self.n_max, dtype=packed.dtype, device=self.device)
        out[self.pack_index] = packed
        return out.view(self.n_mol, self.n_max, self.n_max)

    def to_packed(self, padded: torch.Tensor) -> torch.Tensor:
        return padded.reshape(-1)[self.pack_index]

    def block(self, packed: torch.Tensor, m: int) -> torch.Tensor:
        """Molecule m's n x n view of a packed matrix."""
        n = int(self.mol_nao[m])
        o = int(self.mol_mat[m])
        return packed[o:o + n * n].view(n, n)

    # ---------------------------------------------------------------- compute
    def one_electron(self, atoms=None, centers=None):
        """Packed S, T, V of every molecule."""
        S, T, V = (torch.empty(self.mat_elems, dtype=torch.float64, device=self.device) for _ in range(3))
        _lib.call("dftk_one_electron", ctypes.byref(self.c_shells), len(self.atoms), _lib.ptr(self.d_atom_xyz),
                  _lib.ptr(self.d_atom_z), _lib.ptr(S), _lib.ptr(T), _lib.ptr(V), _lib.stream_handle())
        return S, T, V

    def _square(self, M) -> torch.Tensor:
        if not isinstance(M, torch.Tensor):
            M = torch.as_tensor(np.asarray(M, dtype=np.float64))
        M = M.to(device=self.device, dtype=torch.float64).contiguous()
        if M.numel() != self.mat_elems:
            raise _lib.DftkError("batch", _lib.ERR_ARG, f"packed matrix of {M.numel()} != {self.mat_elems} elements")
        return M

    def jk(self, D, D_a=None, D_b=None, uhf=False, mixed=False, tau=1e-14, tau_fp32=1e-6, out=None, counts=None,
           scan=False, persist=False):
        """Packed J, K_a (, K_b) of every active molecule (see IntegralEngine.jk)."""
        D = self._square(D)
        D_a = self._square(D_a) if D_a is not None else (0.5 * D).contiguous()
        if uhf:
            D_b = self._square(D_b)
        if out is None:
            J = torch.empty(self.mat_elems, dtype=torch.float64, device=self.device)
            Ka = torch.empty_like(J)
            Kb = torch.empty_like(J) if uhf else None
        else:
            J, Ka, Kb = out
        flags = (_lib.JK_UHF if uhf else 0) | (_lib.JK_MIXED if mixed else 0) | (_lib.JK_PERSIST if persist else 0)
        _lib.call("dftk_jk", ctypes.byref(self.c_shells), self.c_pairs, ctypes.byref(self.c_queue),
                  _lib.ptr(D), _lib.ptr(D_a), _lib.ptr(D_b if uhf else None), _lib.ptr(J), _lib.ptr(Ka),
                  _lib.ptr(Kb if uhf else None), flags, float(tau), float(tau_fp32 if mixed else tau),
                  _lib.ptr(self.workspace), self.base_workspace_bytes if scan else self.workspace_bytes,
                  _lib.ptr(counts), _lib.stream_handle())
        return J, Ka, (Kb if uhf else Ka)

    def gradient(self, D, D_a, D_b, W, tau: float = 1e-14, tau_fp32: float = 0.0) -> torch.Tensor:
        """Electronic gradient of every atom of the batch, (total atoms, 3), on the device."""
        n = len(self.atoms)
        g = torch.zeros(3 * n, dtype=torch.float64, device=self.device)
        _lib.call("dftk_grad", ctypes.byref(self.c_shells), _lib.ptr(self.d_shell_atom), n,
                  _lib.ptr(self.d_atom_xyz), _lib.ptr(self.d_atom_z), self.c_pairs, ctypes.byref(self.c_queue),
                  _lib.ptr(self._square(D)), _lib.ptr(self._square(D_a)), _lib.ptr(self._square(D_b)),
                  _lib.ptr(self._square(W)), float(tau), float(tau_fp32), _lib.ptr(g), _lib.ptr(self.workspace),
                  self.workspace_bytes, _lib.stream_handle())
        return g.view(n, 3)

    def nuclear_repulsion(self) -> np.ndarray:
        return np.array([_geometry.nuclear_repulsion(a, c) for a, c in self.molecules])

    def nuclear_repulsion_gradient(self) -> np.ndarray:
        return np.concatenate([_geometry.nuclear_repulsion_gradient(a, c) for a, c in self.molecules], axis=0)


class _FockGraph:
    """The packed J/K build of a batch captured once as a CUDA graph: static
    density input, static J and K outputs."""

    def __init__(self, eng: BatchEngine, tau: float, persist: bool = False):
        self.eng = eng
        self.D = torch.zeros(eng.mat_elems, dtype=torch.float64, device=eng.device)
        self.Dh = torch.zeros_like(self.D)
        self.J = torch.zeros_like(self.D)
        self.K = torch.zeros_like(self.D)
        self.tau = tau
        # warm-up on a side stream, then capture
        s = torch.cuda.Stream(device=eng.device)
        s.wait_stream(torch.cuda.current_stream(eng.device))
        with torch.cuda.stream(s):
            eng.jk(self.D, self.Dh, tau=tau, out=(self.J, self.K, None), persist=persist)
        torch.cuda.current_stream(eng.device).wait_stream(s)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            eng.jk(self.D, self.Dh, tau=tau, out=(self.J, self.K, None), persist=persist)

    def run(self, D_alpha_packed: torch.Tensor):
        """G = J - K for the RHF alpha density (J from 2 D_alpha, K from D_alpha)."""
        self.D.copy_(2.0 * D_alpha_packed)
        self.Dh.copy_(D_alpha_packed)
        self.graph.replay()
        return self.J - self.K


@dataclass
class BatchSCFResult:
    energy: np.ndarray           # per molecule
    converged: np.ndarray        # bool per molecule
    iterations: np.ndarray       # SCF iterations per molecule
    D: torch.Tensor              # packed alpha densities (converged molecules: of their final full build)
    F: torch.Tensor              # packed Fock matrices of those builds
    n_occ: np.ndarray
    fock_builds: int
    seconds: float
    fock_seconds: float
    history: List[int] = field(default_factory=list)  # active molecules per iteration


def _cholesky_orthogonalizer(S: torch.Tensor) -> torch.Tensor:
    """X = L^{-T} with S = L L^T, so X^T S X = I (batched)."""
    L = torch.linalg.cholesky(S)
    eye = torch.eye(S.shape[-1], dtype=S.dtype, device=S.device).expand_as(S)
    return torch.linalg.solve_triangular(L, eye, upper=False).transpose(-1, -2)


def _purify(Fo: torch.Tensor, n_occ: torch.Tensor, real: torch.Tensor, tol: float = 1e-10,
            max_iter: int = 200) -> torch.Tensor:
    """Density D' = sum of the n_occ lowest eigenvectors' projectors of the
    symmetric Fo (B, N, N), by canonical purification.  Padded levels (real
    == 0) are placed above the Gershgorin interval of the real block, by its
    width (at least 1), so they stay apart from the real levels even when
    every real level is occupied (a single-function atom).  Stops when every
    molecule's tr(D - D^2) (the summed deviation of its eigenvalues from 0 or
    1) is below tol, or, once below 1e-6, stops halving; the closing McWeeny step
    D <- 3D^2 - 2D^3 then squares the remaining deviations."""
    B, N, _ = Fo.shape
    diag = Fo.diagonal(dim1=1, dim2=2)
    rad = Fo.abs().sum(dim=2) - diag.abs()
    e_max = torch.where(real > 0, diag + rad, torch.full_like(diag, -torch.inf)).amax(dim=1)
    e_min = torch.where(real > 0, diag - rad, torch.full_like(diag, torch.inf)).amin(dim=1)
    e_max = e_max + (e_max - e_min).clamp_min(1.0)
    F = Fo + torch.diag_embed((1.0 - real) * e_max[:, None])
    mu = F.diagonal(dim1=1, dim2=2).sum(dim=1) / N
    n = n_occ.to(F.dtype)
    lam = torch.minimum(n / (e_max - mu), (N - n) / (mu - e_min))
    eye = torch.eye(N, dtype=F.dtype, device=F.device)
    D = (lam / N)[:, None, None] * (mu[:, None, None] * eye - F) + (n / N)[:, None, None] * eye
    last = float("inf")
    for it in range(max_iter):
        D2 = D @ D
        D3 = D2 @ D
        t1 = (D - D2).diagonal(dim1=1, dim2=2).sum(dim=1)
        t2 = (D2 - D3).diagonal(dim1=1, dim2=2).sum(dim=1)
        ok = t1.abs() > 1e-300
        c = torch.where(ok, t2 / torch.where(ok, t1, torch.ones_like(t1)), torch.full_like(t1, 0.5))
        up = ((1.0 + c)[:, None, None] * D2 - D3) / c.clamp_min(1e-300)[:, None, None]
        lo = ((1.0 - 2.0 * c)[:, None, None] * D + (1.0 + c)[:, None, None] * D2 - D3) / \
            (1.0 - c).clamp_min(1e-300)[:, None, None]
        Dn = torch.where((c >= 0.5)[:, None, None], up, lo)
        D = torch.where(ok[:, None, None], Dn, D)
        if it % 4 == 3:
            err = float(t1.abs().max())
            # in the quadratic end phase a deviation that stops halving is round-off
            if err < tol or (err < 1e-6 and err > 0.5 * last):
                break
            last = err
    # one McWeeny step, then symmetrise
    D2 = D @ D
    D = 3.0 * D2 - 2.0 * (D2 @ D)
    return 0.5 * (D + D.transpose(1, 2))


def _batched_diis(Fh: torch.Tensor, Eh: torch.Tensor, n: int) -> torch.Tensor:
    """Pulay extrapolation for every molecule from the last n entries of the
    history (hist, B, N, N); bordered system solved through its eigenvectors
    with eigenvalues below 1e-14 of the largest dropped."""
    F, E = Fh[:n], Eh[:n]
    B = F.shape[1]
    Ev = E.permute(1, 0, 2, 3).reshape(B, n, -1)
    Bm = Ev @ Ev.transpose(1, 2)
    scale = Bm.diagonal(dim1=1, dim2=2).amax(dim=1).clamp_min(1e-300)
    M = torch.zeros((B, n + 1, n + 1), dtype=torch.float64, device=F.device)
    M[:, :n, :n] = Bm / scale[:, None, None]
    M[:, n, :n] = -1.0
    M[:, :n, n] = -1.0
    rhs = torch.zeros((B, n + 1), dtype=torch.float64, device=F.device)
    rhs[:, n] = -1.0
    w, v = torch.linalg.eigh(M)
    keep = w.abs() > 1e-14 * w.abs().amax(dim=1, keepdim=True)
    winv = torch.where(keep, 1.0 / torch.where(keep, w, torch.ones_like(w)), torch.zeros_like(w))
    c = v @ (winv * (v.transpose(1, 2) @ rhs.unsqueeze(-1)).squeeze(-1)).unsqueeze(-1)
    c = c.squeeze(-1)[:, :n]
    return torch.einsum("bi,ibxy->bxy", c, F)


def scf_rhf_batch(eng: BatchEngine, charges: Optional[Sequence[int]] = None, diis: int = 8, etol: float = 1e-10,
                  dtol: float = 1e-8, max_iter: int = 100, tau: float = 1e-12, rebuild_every: int = 12,
                  finish_factor: float = 100.0, use_graph: bool = True, autotune: bool = False,
                  persist: bool = False) -> BatchSCFResult:
    """Closed-shell SCF of every molecule of the batch at once (same criteria
    as scf.scf_rhf: DIIS(8), |dE| < etol and RMS(dD) < dtol on a full FP64
    Fock build, incremental builds F_k = F_{k-1} + G(D_k - D_{k-1}) in between,
    full builds every ``rebuild_every`` iterations and once RMS(dD) <
    finish_factor x dtol).  ``persist``: each Fock build is one selection
    launch plus one persistent launch over every molecule's quartet tiles of
    every class (DFTK_JK_PERSIST) instead of a selection and a class kernel per
    class."""
    dev = eng.device
    t_start = time.perf_counter()
    B, Nm = eng.n_mol, eng.n_max
    charges = [0] * B if charges is None else list(charges)
    n_el = np.array([_basis.n_electrons(a, q) for (a, _), q in zip(eng.molecules, charges)])
    if np.any(n_el % 2):
        raise ValueError("closed-shell SCF needs even electron counts")
    n_occ = n_el // 2
    e_nn = torch.as_tensor(eng.nuclear_repulsion(), dtype=torch.float64, device=dev)
    eng.mol_active.fill_(1)
    S_p, T_p, V_p = eng.one_electron()
    S = eng.to_padded(S_p) + torch.diag_embed(eng.pad_mask)
    H = eng.to_padded(T_p + V_p)
    X = _cholesky_orthogonalizer(S)
    nn = torch.as_tensor(eng.mol_nao.astype(np.float64) ** 2, device=dev)
    Xt = X.transpose(1, 2)
    real = 1.0 - eng.pad_mask
    rmask = real[:, :, None] * real[:, None, :]
    n_occ_t = torch.as_tensor(n_occ, device=dev)

    def density(Fm):
        """AO density of the n_occ lowest orbitals of Fm (padded, real block)."""
        Dp = _purify(Xt @ Fm @ X, n_occ_t, real)
        return (X @ Dp @ Xt) * rmask

    D = density(H)
    if autotune:
        # launch shapes per class measured on this batch's first (full) build,
        # fixed before the graph captures them
        from . import autotune as _autotune

        Dp0 = eng.to_packed(D)
        _autotune.tune(eng, lambda: eng.jk(2.0 * Dp0, Dp0, tau=tau), _autotune.FAMILY_JK, repeats=1)
    graph = _FockGraph(eng, tau, persist) if use_graph else None

    def build(Dp):
        if graph is not None:
            return graph.run(Dp)
        J, K, _ = eng.jk(2.0 * Dp, Dp, tau=tau, persist=persist)
        return J - K

    Fh = torch.zeros((diis, B, Nm, Nm), dtype=torch.float64, device=dev)
    Eh = torch.zeros_like(Fh)
    n_hist = 0
    G = torch.zeros(eng.mat_elems, dtype=torch.float64, device=dev)
    D_ref = torch.zeros_like(D)
    D_fin = torch.zeros(eng.mat_elems, dtype=torch.float64, device=dev)
    F_fin = torch.zeros_like(D_fin)
    since_full = np.full(B, rebuild_every, dtype=np.int64)  # first build is full
    finishing = np.zeros(B, dtype=bool)
    active = np.ones(B, dtype=bool)
    E_prev = np.full(B, np.inf)
    E_fin = np.zeros(B)
    iters = np.zeros(B, dtype=np.int64)
    conv = np.zeros(B, dtype=bool)
    builds, t_fock = 0, 0.0
    hist_active: List[int] = []
    for it in range(max_iter + 1):
        full = (since_full >= rebuild_every) | finishing
        full_t = torch.as_tensor(full, device=dev)
        Din = torch.where(full_t[:, None, None], D, D - D_ref)
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        Gb = build(eng.to_packed(Din))
        torch.cuda.synchronize(dev)
        t_fock += time.perf_counter() - t0
        builds += 1
        hist_active.append(int(active.sum()))
        fp = full_t[eng.packed_mol]
        G = torch.where(fp, Gb, G + Gb)
        since_full = np.where(full, 1, since_full + 1)
        D_ref = D
        F = H + eng.to_padded(G)
        E = ((D * (H + F)).sum(dim=(1, 2)) + e_nn).cpu().numpy()
        err = Xt @ (F @ D @ S - S @ D @ F) @ X
        Fh = torch.roll(Fh, 1, dims=0)
        Eh = torch.roll(Eh, 1, dims=0)
        Fh[0] = F
        Eh[0] = err
        n_hist = min(n_hist + 1, diis)
        Fx = _batched_diis(Fh, Eh, n_hist) if n_hist >= 2 else F
        D_new = density(Fx)
        rms = torch.sqrt(((D_new - D) ** 2).sum(dim=(1, 2)) / nn).cpu().numpy()
        dE = np.abs(E - E_prev)
        finishing |= rms < finish_factor * dtol
        done = active & (dE < etol) & (rms < dtol) & full
        if done.any():
            idx = np.nonzero(done)[0]
            E_fin[idx] = E[idx]
            iters[idx] = it
            conv[idx] = True
            active[idx] = False
            sel = torch.as_tensor(idx, device=dev)
            pm = torch.zeros(B, dtype=torch.bool, device=dev)
            pm[sel] = True
            pm = pm[eng.packed_mol]
            D_fin = torch.where(pm, eng.to_packed(D), D_fin)
            F_fin = torch.where(pm, eng.to_packed(F), F_fin)
            eng.mol_active[sel] = 0
        if not active.any():
            break
        E_prev = np.where(active, E, E_prev)
        keep = torch.as_tensor(active, device=dev)[:, None, None]
        D = torch.where(keep, D_new, D)
    if active.any():
        E_fin[active] = E_prev[active]
        iters[active] = max_iter
        pm = torch.as_tensor(active, device=dev)[eng.packed_mol]
        D_fin = torch.where(pm, eng.to_packed(D), D_fin)
        F_fin = torch.where(pm, eng.to_packed(F), F_fin)
    eng.mol_active.fill_(1)
    torch.cuda.synchronize(dev)
    return BatchSCFResult(E_fin, conv, iters, D_fin, F_fin, n_occ, builds, time.perf_counter() - t_start,
                          t_fock, hist_active)


def rhf_gradient_batch(eng: BatchEngine, res: BatchSCFResult, tau: float = 1e-14,
                       tau_fp32: float = 0.0) -> List[np.ndarray]:
    """Analytic RHF gradients of every molecule of a converged batch, one
    dftk_grad call for the whole batch: per molecule an (n_atoms, 3) array.
    With D_alpha = C_occ C_occ^T of a converged F, the energy-weighted
    density C_occ diag(eps) C_occ^T equals D_alpha F D_alpha."""
    Da = eng.to_padded(res.D)
    Fp = eng.to_padded(res.F)
    Dp = eng.to_packed(2.0 * Da)
    Wp = eng.to_packed(2.0 * (Da @ Fp @ Da))
    Dh = (0.5 * Dp).contiguous()
    g = eng.gradient(Dp, Dh, Dh, Wp, tau=tau, tau_fp32=tau_fp32).cpu().numpy() + eng.nuclear_repulsion_gradient()
    return [g[int(eng.mol_atom0[m]):int(eng.mol_atom0[m] + eng.mol_natom[m])] for m in range(eng.n_mol)]
