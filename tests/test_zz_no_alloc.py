"""dftk_jk_noalloc: the J/K build for callers that cannot allocate device memory.

Such callers (a host program running inside a device-memory budget it has
already divided up, or a plugin host whose pool must account for every byte)
cannot hand dftk_jk a workspace.  dftk_jk_noalloc uses a fixed array inside
the library instead.  These tests call it through the C-ABI and check it
against dftk_jk with a caller workspace, on two calls in a row (the second
call sees the scratch the first one left behind).  This file is collected last
so that a run stopping at the first failure has already run everything else.
"""
import ctypes

import numpy as np
import pytest

from dft_b200 import _lib, basis, geometry

# J/K tolerance of the FP64 path (elements are sums of ~1e8 atomically added terms)
TOL = 1e-12


def _noalloc(eng, D, Da, Db, uhf, tau, mixed=False, tau_fp32=1e-6):
    import torch

    N = eng.n_ao
    J, Ka = (torch.full((N, N), np.nan, dtype=torch.float64, device=eng.device) for _ in range(2))
    Kb = torch.full((N, N), np.nan, dtype=torch.float64, device=eng.device) if uhf else None
    flags = (_lib.JK_UHF if uhf else 0) | (_lib.JK_MIXED if mixed else 0)
    _lib.call("dftk_jk_noalloc", ctypes.byref(eng.c_shells), eng.c_pairs, ctypes.byref(eng.c_queue),
              _lib.ptr(D), _lib.ptr(Da), _lib.ptr(Db if uhf else None), _lib.ptr(J), _lib.ptr(Ka),
              _lib.ptr(Kb), flags, tau, tau_fp32 if mixed else tau, None, _lib.stream_handle())
    return J, Ka, Kb


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [None, (2, 2, 2)])
def test_noalloc_matches_workspace_jk(shape):
    import torch

    from dft_b200.engine import IntegralEngine

    atoms, centers = geometry.water() if shape is None else geometry.water_cluster(shape, seed=5)
    eng = IntegralEngine(basis.build_shells(basis.load_basis(), atoms, centers), tau_schwarz=1e-12)
    N = eng.n_ao
    rng = np.random.default_rng(4)
    A, B = rng.normal(size=(N, N)), rng.normal(size=(N, N))
    Da = torch.as_tensor(0.05 * (A + A.T)).cuda()
    Db = torch.as_tensor(0.05 * (B + B.T)).cuda()
    D = Da + Db
    J0, Ka0, Kb0 = eng.jk(D, Da, Db, uhf=True, tau=0.0)
    for _ in range(2):
        J, Ka, Kb = _noalloc(eng, D, Da, Db, uhf=True, tau=0.0)
        torch.cuda.synchronize()
        assert (J - J0).abs().max().item() < TOL
        assert (Ka - Ka0).abs().max().item() < TOL
        assert (Kb - Kb0).abs().max().item() < TOL
    # closed-shell call shape, also twice
    J1, K1, _ = eng.jk(D, 0.5 * D, tau=1e-14)
    for _ in range(2):
        J, Ka, _ = _noalloc(eng, D, (0.5 * D).contiguous(), None, uhf=False, tau=1e-14)
        torch.cuda.synchronize()
        assert (J - J1).abs().max().item() < TOL and (Ka - K1).abs().max().item() < TOL


@pytest.mark.gpu
def test_noalloc_mixed_and_scan_path_near_limit():
    """(H2O)_64 (448 basis functions, 320 shells) is near the 512 limit: its
    selection lists (about 0.9 GB) do not fit the fixed scratch, so the call
    takes the direct path, where the class kernels scan the candidates
    themselves.  Checked against dftk_jk with a full workspace, FP64 and mixed
    FP32/FP64 (same thresholds, so the same quartets run in FP32), twice each."""
    import torch

    from dft_b200.engine import IntegralEngine

    atoms, centers = geometry.water_cluster((4, 4, 4))
    eng = IntegralEngine(basis.build_shells(basis.load_basis(), atoms, centers), tau_schwarz=1e-12)
    N = eng.n_ao
    assert N == 448
    rng = np.random.default_rng(6)
    A = rng.normal(size=(N, N))
    D = torch.as_tensor(0.01 * (A + A.T)).cuda()
    Dh = (0.5 * D).contiguous()
    for mixed in (False, True):
        J0, K0, _ = eng.jk(D, Dh, mixed=mixed, tau=1e-12, tau_fp32=1e-6)
        # the two paths add the same terms in different orders: FP64 atomics
        # over ~1e8 terms per build, so compare relative to the largest element
        tol = 1e-12 * max(1.0, J0.abs().max().item())
        for _ in range(2):
            J, Ka, _ = _noalloc(eng, D, Dh, None, uhf=False, tau=1e-12, mixed=mixed, tau_fp32=1e-6)
            torch.cuda.synchronize()
            assert (J - J0).abs().max().item() < tol, mixed
            assert (Ka - K0).abs().max().item() < tol, mixed


@pytest.mark.gpu
def test_noalloc_mixed_small():
    """Mixed FP32/FP64 call on a small cluster, against dftk_jk, twice."""
    import torch

    from dft_b200.engine import IntegralEngine

    atoms, centers = geometry.water_cluster((2, 2, 2), seed=5)
    eng = IntegralEngine(basis.build_shells(basis.load_basis(), atoms, centers), tau_schwarz=1e-12)
    N = eng.n_ao
    rng = np.random.default_rng(8)
    A = rng.normal(size=(N, N))
    D = torch.as_tensor(1e-4 * (A + A.T)).cuda()  # small, so many quartets fall below tau_fp32
    Dh = (0.5 * D).contiguous()
    counts = torch.zeros(24, dtype=torch.int64, device="cuda")
    J0, K0, _ = eng.jk(D, Dh, mixed=True, tau=1e-14, tau_fp32=1e-6, counts=counts)
    torch.cuda.synchronize()
    assert counts[6:12].sum().item() > 0  # some quartets did run in FP32
    for _ in range(2):
        J, Ka, _ = _noalloc(eng, D, Dh, None, uhf=False, tau=1e-14, mixed=True, tau_fp32=1e-6)
        torch.cuda.synchronize()
        assert (J - J0).abs().max().item() < TOL and (Ka - K0).abs().max().item() < TOL


@pytest.mark.gpu
def test_noalloc_rejects_oversize_molecule():
    """Sizes beyond the fixed scratch are refused before any device work."""
    lib = _lib.load()
    sh = _lib.Shells(600, 800, None, None, None, None, None, None, None)
    pairs = _lib.PairsArray()
    q = _lib.Queue()
    st = lib.dftk_jk_noalloc(ctypes.byref(sh), pairs, ctypes.byref(q), None, None, None, None, None, None,
                             0, 0.0, 0.0, None, None)
    assert st == _lib.ERR_SIZE
    msg = lib.dftk_last_error().decode()
    assert "exceed" in msg and "512" in msg
