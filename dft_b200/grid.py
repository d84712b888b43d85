"""Orbitals on a grid of points: the evaluation checkpoint the reference's SCF
writes (shelled.py:1296) and the orbital densities its evaluation script
computes from it (shelled_eval.py:11-131), on the GPU.

Per chunk of points: ``dftk_grid_ao`` evaluates every AO at every point (FP32
points, FP64 arithmetic, like the reference), the MO values
psi_s = C_s[:, :n]^T A ao are one FP64 GEMM per spin (the library GEMM; the
coefficients are rounded to FP32 first, as the reference does), and
``dftk_grid_density`` writes the per-orbital total density
[k < N_a] psi_a^2 + [k < N_b] psi_b^2 and the alpha phase psi_a (rows
k < N_a) in FP32.  When C_b equals C_a (closed shell) the beta GEMM is reused.
"""
from __future__ import annotations

import ctypes
import math
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch

from . import _lib

CHECKPOINT_KEYS = ("centers", "N_a", "N_b", "C_a", "C_b", "total_ao", "shells", "A")


def _host(x):
    return x.detach().cpu().numpy() if isinstance(x, torch.Tensor) else x


def save_eval_checkpoint(path: str, centers, N_a, N_b, C_a, C_b, total_ao, shells: List[Dict], A) -> None:
    """Write the evaluation checkpoint with the reference's keys and layout
    (``savez``; the shell dicts are stored as an object array)."""
    np.savez(path, centers=_host(centers), N_a=_host(N_a), N_b=_host(N_b), C_a=_host(C_a), C_b=_host(C_b),
             total_ao=_host(total_ao), shells=np.asarray(shells, dtype=object), A=_host(A))


def load_eval_checkpoint(path: str) -> Dict:
    """Read an evaluation checkpoint (the reference's or ``save_eval_checkpoint``'s)."""
    data = np.load(path, allow_pickle=True)
    missing = [k for k in CHECKPOINT_KEYS if k not in data.files]
    if missing:
        raise KeyError(f"evaluation checkpoint {path} lacks {missing}")
    out = {k: data[k] for k in CHECKPOINT_KEYS}
    out["shells"] = data["shells"].tolist()
    return out


def reference_grid(centers, spacing: float = 0.008, pad_lo: Sequence[float] = (0.0, -0.75, 1.0),
                   pad_hi: Sequence[float] = (-1.0, -0.75, 1.0)) -> Tuple[np.ndarray, Tuple[int, int, int]]:
    """The evaluation script's grid (shelled_eval.py:27-56): along each axis
    ``linspace(min - pad_lo, max + pad_hi, ceil(range / spacing) + 1)`` over
    the centres, points ordered x slowest, z fastest, stored FP32.  The
    defaults are the script's own bounds (x up to max - 1, y inset by 0.75,
    z padded by 1).  Returns (points (n, 3) float32, (nx, ny, nz))."""
    c = np.asarray(centers, dtype=np.float64).reshape(-1, 3)
    axes = []
    for k in range(3):
        lo = float(c[:, k].min()) - float(pad_lo[k])
        hi = float(c[:, k].max()) + float(pad_hi[k])
        n = math.ceil((hi - lo) / spacing) + 1
        if n < 1:
            raise ValueError(f"empty grid along axis {'xyz'[k]} ({lo} .. {hi})")
        axes.append(np.linspace(lo, hi, n))
    shape = tuple(len(a) for a in axes)
    g = np.stack(np.meshgrid(*axes, indexing="ij"), axis=-1).astype(np.float32)
    return g.reshape(-1, 3), shape


class OrbitalGrid:
    """Orbital densities of one evaluation checkpoint at arbitrary points."""

    def __init__(self, ckpt: Dict, device=None):
        from . import shelled

        self.ckpt = ckpt
        self.shells = ckpt["shells"]
        with torch.cuda.device(torch.device(device) if device is not None else torch.cuda.current_device()):
            self.engine = shelled.get_engine(self.shells)
        self.device = self.engine.device
        self.n_a, self.n_b = int(ckpt["N_a"]), int(ckpt["N_b"])
        self.n_mo = max(self.n_a, self.n_b)
        A = np.asarray(ckpt["A"], dtype=np.float64)
        identity = A.shape[0] == A.shape[1] and np.array_equal(A, np.eye(A.shape[0]))

        def coeffs(C):
            C32 = np.asarray(C).astype(np.float32)[:, :self.n_mo].T  # the reference's FP32 rounding
            M = torch.as_tensor(C32.astype(np.float64), device=self.device)
            if not identity:
                M = M @ torch.as_tensor(A, device=self.device)
            return C32, M.contiguous()

        Ca32, self.Ca = coeffs(ckpt["C_a"])
        Cb32, self.Cb = coeffs(ckpt["C_b"])
        self.same_spin = np.array_equal(Ca32, Cb32)
        if self.Ca.shape[1] != self.engine.n_ao:
            raise _lib.DftkError("grid", _lib.ERR_ARG,
                                 f"coefficients cover {self.Ca.shape[1]} AOs, the shells {self.engine.n_ao}")

    def chunk(self, points: torch.Tensor, total: torch.Tensor, phase: torch.Tensor) -> None:
        """Densities of the FP32 device points (m, 3) into the device tensors
        total (n_mo, ld) and phase (N_a, ld), columns 0 .. m - 1."""
        m = int(points.shape[0])
        if points.dtype != torch.float32 or tuple(points.shape[1:]) != (3,):
            raise _lib.DftkError("grid", _lib.ERR_ARG, "points must be an (m, 3) float32 tensor")
        if total.shape[0] != self.n_mo or total.shape[1] < m or (self.n_a > 0 and (phase.shape[0] < self.n_a
                                                                                   or phase.shape[1] < m)):
            raise _lib.DftkError("grid", _lib.ERR_ARG, "total (n_mo, >= m) and phase (N_a, >= m) expected")
        eng = self.engine
        ao = torch.empty((eng.n_ao, m), dtype=torch.float64, device=self.device)
        _lib.call("dftk_grid_ao", ctypes.byref(eng.c_shells), m, _lib.ptr(points), _lib.ptr(ao), m,
                  _lib.stream_handle())
        psi_a = self.Ca @ ao
        psi_b = psi_a if self.same_spin else self.Cb @ ao
        if self.n_a > 0 and phase.stride(0) != total.stride(0):
            raise _lib.DftkError("grid", _lib.ERR_ARG, "total and phase need the same leading dimension")
        _lib.call("dftk_grid_density", self.n_mo, self.n_a, self.n_b, m, _lib.ptr(psi_a), _lib.ptr(psi_b), m,
                  _lib.row_ptr(total), _lib.row_ptr(phase) if self.n_a > 0 else None, int(total.stride(0)),
                  _lib.stream_handle())

    def evaluate(self, points, chunk_size: int = 1_000_000, total: Optional[np.ndarray] = None,
                 phase: Optional[np.ndarray] = None) -> Tuple[np.ndarray, np.ndarray]:
        """Total and phase densities (n_mo, n_points) FP32 on the host, filled
        chunk by chunk like the evaluation script (into ``total``/``phase``
        when given, e.g. memory-mapped files; else new zeroed arrays)."""
        pts = np.asarray(points, dtype=np.float32).reshape(-1, 3)
        n = pts.shape[0]
        if total is None:
            total = np.zeros((self.n_mo, n), dtype=np.float32)
        if phase is None:
            phase = np.zeros((self.n_mo, n), dtype=np.float32)
        if total.shape != (self.n_mo, n) or phase.shape != (self.n_mo, n):
            raise _lib.DftkError("grid", _lib.ERR_ARG, f"outputs must be ({self.n_mo}, {n})")
        if chunk_size < 1:
            raise _lib.DftkError("grid", _lib.ERR_ARG, "chunk_size must be positive")
        m_max = min(chunk_size, max(n, 1))
        d_tot = torch.empty((self.n_mo, m_max), dtype=torch.float32, device=self.device)
        d_ph = torch.empty((max(self.n_a, 1), m_max), dtype=torch.float32, device=self.device)
        # pinned staging, kept for the next call: one device-to-host copy per
        # output and chunk
        key = (self.n_mo, max(self.n_a, 1), m_max)
        if getattr(self, "_staging_key", None) != key:
            self._staging = (torch.empty((self.n_mo, m_max), dtype=torch.float32, pin_memory=True),
                             torch.empty((max(self.n_a, 1), m_max), dtype=torch.float32, pin_memory=True))
            self._staging_key = key
        h_tot, h_ph = self._staging
        for w in range(0, n, chunk_size):
            m = min(chunk_size, n - w)
            d_pts = torch.as_tensor(pts[w:w + m]).to(self.device)
            self.chunk(d_pts, d_tot[:, :m], d_ph[:, :m])
            h_tot[:, :m].copy_(d_tot[:, :m], non_blocking=True)
            if self.n_a > 0:
                h_ph[:, :m].copy_(d_ph[:, :m], non_blocking=True)
            torch.cuda.current_stream(self.device).synchronize()
            total[:, w:w + m] = h_tot[:, :m].numpy()
            if self.n_a > 0:
                phase[:self.n_a, w:w + m] = h_ph[:self.n_a, :m].numpy()
        return total, phase
