"""ctypes binding of libdftk.so (declared in include/dftk.h).

The library is built in-tree (``dft_b200/libdftk.so``) by
``dft_b200/csrc/build.py``.  There is no fallback: if the shared object is
missing or a call fails, a :class:`DftkError` is raised.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

HERE = os.path.dirname(os.path.abspath(__file__))
# DFTK_LIB selects another build of the same library (e.g. a tuning variant)
LIB_PATH = os.environ.get("DFTK_LIB") or os.path.join(HERE, "libdftk.so")

N_QCLASS = 6
N_PCLASS = 3
JK_UHF = 1
JK_MIXED = 2
JK_PERSIST = 4
PCLASS_GENERIC = 3  # dftk_pair_data: the 13-field record layout of the d-shell path

OK, ERR_ARG, ERR_CUDA, ERR_UNSUPPORTED, ERR_WORKSPACE, ERR_SIZE = range(6)

# Exported symbols (every one declared in include/dftk.h).
SYMBOLS = (
    "dftk_version", "dftk_last_error", "dftk_init", "dftk_boys", "dftk_boys32",
    "dftk_pair_data", "dftk_schwarz", "dftk_one_electron", "dftk_eri_blocks",
    "dftk_jk_workspace_bytes", "dftk_jk_workspace_bytes_queue", "dftk_jk", "dftk_nuclear_kernel", "dftk_eri_kernel",
    "dftk_fma_burn", "dftk_jk_timing", "dftk_jk_timing_read", "dftk_jk_noalloc", "dftk_grad", "dftk_workspace_bytes",
    "dftk_set_launch", "dftk_get_launch", "dftk_grid_ao", "dftk_grid_density", "dftk_prepare_bytes", "dftk_prepare",
    "dftk_hl_schwarz", "dftk_jk_hl", "dftk_hl_eri_blocks", "dftk_set_tile", "dftk_get_tile",
    "dftk_prepare_hl_bytes", "dftk_prepare_hl",
)


class DftkError(RuntimeError):
    """A libdftk call returned a non-zero status."""

    def __init__(self, name: str, status: int, message: str):
        super().__init__(f"{name} failed with status {status}: {message}")
        self.status = status


class Shells(ctypes.Structure):
    _fields_ = [
        ("n_shells", ctypes.c_int),
        ("n_ao", ctypes.c_int),
        ("xyz", ctypes.c_void_p),
        ("l", ctypes.c_void_p),
        ("nprim", ctypes.c_void_p),
        ("prim_off", ctypes.c_void_p),
        ("ao", ctypes.c_void_p),
        ("prim_exp", ctypes.c_void_p),
        ("prim_cn", ctypes.c_void_p),
        # batch description (zero / NULL for one molecule)
        ("n_mol", ctypes.c_int),
        ("max_ns", ctypes.c_int),
        ("max_natom", ctypes.c_int),
        ("mat_elems", ctypes.c_longlong),
        ("dsh_elems", ctypes.c_longlong),
        ("mol", ctypes.c_void_p),
        ("mol_mat", ctypes.c_void_p),
        ("mol_nao", ctypes.c_void_p),
        ("mol_shell0", ctypes.c_void_p),
        ("mol_ns", ctypes.c_void_p),
        ("mol_dsh", ctypes.c_void_p),
        ("mol_atom0", ctypes.c_void_p),
        ("mol_natom", ctypes.c_void_p),
    ]


class Pairs(ctypes.Structure):
    _fields_ = [
        ("n_pairs", ctypes.c_int),
        ("kmax", ctypes.c_int),
        ("ab", ctypes.c_void_p),
        ("nprim", ctypes.c_void_p),
        ("rec64", ctypes.c_void_p),
        ("rec32", ctypes.c_void_p),
        ("q", ctypes.c_void_p),
        ("qp", ctypes.c_void_p),
        ("core64", ctypes.c_void_p),
        ("core32", ctypes.c_void_p),
    ]


class Queue(ctypes.Structure):
    _fields_ = [
        ("n_rows", ctypes.c_longlong * N_QCLASS),
        ("total", ctypes.c_longlong * N_QCLASS),
        ("row_off", ctypes.c_void_p * N_QCLASS),
        ("tau_prim", ctypes.c_double),
        ("ket_base", ctypes.c_void_p * N_QCLASS),
        ("mol_active", ctypes.c_void_p),
        ("bucket_kets", ctypes.c_int),
    ]


# thread-per-quartet d classes: (bra pair kind, ket pair kind), kinds 0 ss,
# 1 ps, 2 pp, 3 ds, 4 dp, 5 dd (the table of hl_classes.cuh)
HLC_CLASS_KINDS = [(3, 0), (3, 1), (3, 2), (4, 0), (4, 1), (4, 2), (5, 0), (5, 1), (3, 3), (4, 3), (4, 4), (5, 2),
                   (5, 3), (5, 4), (5, 5)]
HLC_N_CLASSES = len(HLC_CLASS_KINDS)
# primitive-pair-count buckets of the class ket lists (DFTK_HLC_BUCKET_BOUNDS)
HLC_BUCKET_BOUNDS = [1, 4, 9, 16, 36, 1 << 30]
HLC_NB = len(HLC_BUCKET_BOUNDS)


class HlSet(ctypes.Structure):
    """dftk_hl_t: the pair sets and candidate spaces of the quartets with a d shell."""
    _fields_ = [
        ("hi", Pairs),
        ("lo", Pairs),
        ("n_rows", ctypes.c_longlong),
        ("total", ctypes.c_longlong * 2),
        ("row_off", ctypes.c_void_p * 2),
        ("tau_prim", ctypes.c_double),
        ("lmax", ctypes.c_int),
        ("cls_rows", ctypes.c_void_p * 3),
        ("n_cls_rows", ctypes.c_longlong * 3),
        ("cls_kets", ctypes.c_void_p * 6),
        ("cls_ket_seg", (ctypes.c_longlong * (HLC_NB + 1)) * 6),
        ("cls_off", ctypes.c_void_p * HLC_N_CLASSES),
        ("cls_total", ctypes.c_longlong * HLC_N_CLASSES),
    ]


PairsArray = Pairs * N_PCLASS

_lib: Optional[ctypes.CDLL] = None


def load() -> ctypes.CDLL:
    """Load libdftk.so (building it first when nvcc is present and it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        from .csrc import build as _build

        try:
            _build.build()
        except Exception as exc:  # pragma: no cover - build environment specific
            raise DftkError("load", -1, f"libdftk.so missing and build failed: {exc}") from exc
    lib = ctypes.CDLL(LIB_PATH)
    vp, i, ll, d, sz = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, ctypes.c_double, ctypes.c_size_t
    sig = {
        "dftk_version": ([], i),
        "dftk_last_error": ([], ctypes.c_char_p),
        "dftk_init": ([], i),
        "dftk_boys": ([i, ll, vp, vp, vp], i),
        "dftk_boys32": ([i, ll, vp, vp, vp], i),
        "dftk_pair_data": ([ctypes.POINTER(Shells), i, ctypes.POINTER(Pairs), vp], i),
        "dftk_schwarz": ([ctypes.POINTER(Shells), i, ctypes.POINTER(Pairs), vp], i),
        "dftk_one_electron": ([ctypes.POINTER(Shells), i, vp, vp, vp, vp, vp, vp], i),
        "dftk_eri_blocks": ([ctypes.POINTER(Shells), ctypes.POINTER(Pairs), ll, vp, vp, vp, vp], i),
        "dftk_jk_workspace_bytes": ([i, i], sz),
        "dftk_jk_workspace_bytes_queue": ([i, i, ctypes.POINTER(Queue)], sz),
        "dftk_workspace_bytes": ([ctypes.POINTER(Shells), ctypes.POINTER(Queue)], sz),
        "dftk_set_launch": ([i, i, i, i, i], i),
        "dftk_get_launch": ([i, i, i, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)], i),
        "dftk_set_tile": ([i, i, i], i),
        "dftk_prepare_hl_bytes": ([ctypes.POINTER(Shells), ctypes.POINTER(ctypes.c_size_t)], i),
        "dftk_prepare_hl": ([ctypes.POINTER(Shells), d, d, vp, sz, ctypes.POINTER(HlSet), vp], i),
        "dftk_get_tile": ([i, i, ctypes.POINTER(ctypes.c_int)], i),
        "dftk_jk": ([ctypes.POINTER(Shells), ctypes.POINTER(Pairs), ctypes.POINTER(Queue), vp, vp, vp,
                     vp, vp, vp, i, d, d, vp, sz, vp, vp], i),
        "dftk_nuclear_kernel": ([vp] * 8 + [i, i, i] + [vp] * 9 + [vp], i),
        "dftk_eri_kernel": ([i] + [vp] * 8 + [i] + [vp] * 8 + [vp, vp], i),
        "dftk_fma_burn": ([i, i, i, i, vp, vp], i),
        "dftk_jk_noalloc": ([ctypes.POINTER(Shells), ctypes.POINTER(Pairs), ctypes.POINTER(Queue), vp, vp, vp,
                             vp, vp, vp, i, d, d, vp, vp], i),
        "dftk_grad": ([ctypes.POINTER(Shells), vp, i, vp, vp, ctypes.POINTER(Pairs), ctypes.POINTER(Queue), vp, vp,
                       vp, vp, d, d, vp, vp, sz, vp], i),
        "dftk_jk_timing": ([i], i),
        "dftk_jk_timing_read": ([vp, i], i),
        "dftk_grid_ao": ([ctypes.POINTER(Shells), ll, vp, vp, ll, vp], i),
        "dftk_grid_density": ([i, i, i, ll, vp, vp, ll, vp, vp, ll, vp], i),
        "dftk_prepare_bytes": ([ctypes.POINTER(Shells), ctypes.POINTER(ctypes.c_size_t)], i),
        "dftk_prepare": ([ctypes.POINTER(Shells), d, d, vp, sz, ctypes.POINTER(Pairs), ctypes.POINTER(Queue), vp], i),
        "dftk_hl_schwarz": ([ctypes.POINTER(Shells), ctypes.POINTER(Pairs), i, vp], i),
        "dftk_jk_hl": ([ctypes.POINTER(Shells), ctypes.POINTER(HlSet), vp, vp, vp, vp, vp, vp, i, d, vp, sz, vp, vp], i),
        "dftk_hl_eri_blocks": ([ctypes.POINTER(Shells), ctypes.POINTER(HlSet), ll, vp, vp, vp, vp], i),
    }
    missing = set(SYMBOLS) - set(sig)
    if missing:  # every entry point gets explicit argument types (64-bit sizes)
        raise DftkError("load", -1, f"no argument types for {sorted(missing)}")
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def call(name: str, *args) -> None:
    lib = load()
    st = getattr(lib, name)(*args)
    if st != OK:
        msg = lib.dftk_last_error()
        raise DftkError(name, st, msg.decode() if msg else "")


def stream_handle(stream=None) -> ctypes.c_void_p:
    import torch

    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def row_ptr(t) -> ctypes.c_void_p:
    """Device pointer of a CUDA matrix whose rows are contiguous (a column
    slice of a wider matrix; the leading dimension is t.stride(0))."""
    if not t.is_cuda or t.dim() != 2 or t.stride(1) != 1:
        raise DftkError("ptr", ERR_ARG, "expected a CUDA matrix with contiguous rows")
    return ctypes.c_void_p(t.data_ptr())


def ptr(t) -> ctypes.c_void_p:
    """Device pointer of a CUDA tensor (None -> NULL)."""
    if t is None:
        return ctypes.c_void_p(0)
    if not t.is_cuda:
        raise DftkError("ptr", ERR_ARG, "expected a CUDA tensor")
    if not t.is_contiguous():
        raise DftkError("ptr", ERR_ARG, "expected a contiguous tensor")
    return ctypes.c_void_p(t.data_ptr())
