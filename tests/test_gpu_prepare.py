"""dftk_prepare: the C-ABI's one-call setup of pairs and queue (what a C host
uses instead of the Python engine) gives the engine's pair counts, quartet
counts and J/K (needs a GPU)."""
import ctypes

import numpy as np
import pytest
import torch

from dft_b200 import _lib, basis, geometry
from dft_b200.engine import IntegralEngine

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape,tau", [((2, 2, 2), 1e-12), ((1, 1, 2), 0.0)])
def test_prepare_matches_engine(shape, tau):
    atoms, centers = geometry.water_cluster(shape)
    shells = basis.build_shells(basis.load_basis(), atoms, centers)
    eng = IntegralEngine(shells, tau_schwarz=tau)
    nbytes = ctypes.c_size_t()
    _lib.call("dftk_prepare_bytes", ctypes.byref(eng.c_shells), ctypes.byref(nbytes))
    storage = torch.empty(nbytes.value, dtype=torch.uint8, device=eng.device)
    pairs, queue = _lib.PairsArray(), _lib.Queue()
    _lib.call("dftk_prepare", ctypes.byref(eng.c_shells), tau, eng.tau_prim, _lib.ptr(storage), nbytes.value,
              pairs, ctypes.byref(queue), _lib.stream_handle())
    assert [pairs[pc].n_pairs for pc in range(3)] == eng.n_pairs
    assert [pairs[pc].kmax for pc in range(3)] == [eng.kmax] * 3
    assert [queue.total[c] for c in range(6)] == eng.quartet_totals()
    assert queue.tau_prim == eng.tau_prim
    # J/K through the C-ABI's pairs and queue
    N = eng.n_ao
    g = torch.Generator(device="cpu").manual_seed(2)
    A = torch.randn(N, N, generator=g, dtype=torch.float64)
    Da = (0.05 * (A + A.T)).to(eng.device)
    J0, K0, _ = eng.jk(2 * Da, Da, tau=1e-14)
    ws_bytes = _lib.load().dftk_jk_workspace_bytes_queue(eng.ns, N, ctypes.byref(queue))
    ws = torch.empty(int(ws_bytes), dtype=torch.uint8, device=eng.device)
    J, K = torch.empty_like(J0), torch.empty_like(K0)
    D = (2 * Da).contiguous()
    _lib.call("dftk_jk", ctypes.byref(eng.c_shells), pairs, ctypes.byref(queue), _lib.ptr(D), _lib.ptr(Da), None,
              _lib.ptr(J), _lib.ptr(K), None, 0, 1e-14, 1e-14, _lib.ptr(ws), int(ws_bytes), None,
              _lib.stream_handle())
    torch.cuda.synchronize()
    assert (J - J0).abs().max().item() < 1e-12
    assert (K - K0).abs().max().item() < 1e-12
    # too little storage is refused before any work
    with pytest.raises(_lib.DftkError) as ei:
        _lib.call("dftk_prepare", ctypes.byref(eng.c_shells), tau, eng.tau_prim, _lib.ptr(storage),
                  nbytes.value - 1, pairs, ctypes.byref(queue), _lib.stream_handle())
    assert ei.value.status == _lib.ERR_WORKSPACE


def test_prepare_hl_d_shells_through_the_c_abi():
    """A C host's whole d-shell path with no Python setup: dftk_prepare (s/p
    part) and dftk_prepare_hl (d part) fill the pair sets and candidate
    spaces; dftk_jk then dftk_jk_hl give the engine's J/K (HBr / STO-3G, and
    the generally contracted d-polarised test basis on H2O)."""
    import json
    import os

    from conftest import GOLDEN

    with open(os.path.join(GOLDEN, "dz_gc_test.json")) as fh:
        gc = json.load(fh)
    cases = [(basis.load_basis(), ["35", "1"], np.array([[0.0, 0.0, 0.0], [0.3, 0.1, 2.7]])),
             (gc,) + tuple(geometry.water())]
    for data, atoms, centers in cases:
        sh = basis.build_shells(data, atoms, centers)
        eng = IntegralEngine(sh, tau_schwarz=1e-12)
        N = eng.n_ao
        rng = np.random.default_rng(2)
        M = rng.normal(size=(N, N))
        D = torch.as_tensor(0.05 * (M + M.T), device=eng.device)
        Da = (0.5 * D).contiguous()
        J0, K0, _ = eng.jk(D, Da, tau=1e-14)
        stream = _lib.stream_handle()
        nbytes = ctypes.c_size_t()
        _lib.call("dftk_prepare_bytes", ctypes.byref(eng.c_shells), ctypes.byref(nbytes))
        storage = torch.empty(nbytes.value, dtype=torch.uint8, device=eng.device)
        pairs = _lib.PairsArray()
        queue = _lib.Queue()
        _lib.call("dftk_prepare", ctypes.byref(eng.c_shells), 1e-12, eng.tau_prim, _lib.ptr(storage), nbytes.value,
                  pairs, ctypes.byref(queue), stream)
        hbytes = ctypes.c_size_t()
        _lib.call("dftk_prepare_hl_bytes", ctypes.byref(eng.c_shells), ctypes.byref(hbytes))
        hstore = torch.empty(hbytes.value, dtype=torch.uint8, device=eng.device)
        hl = _lib.HlSet()
        _lib.call("dftk_prepare_hl", ctypes.byref(eng.c_shells), 1e-12, eng.tau_prim, _lib.ptr(hstore), hbytes.value,
                  ctypes.byref(hl), stream)
        assert hl.n_rows == eng.c_hl.n_rows and list(hl.total) == list(eng.c_hl.total) and hl.lmax == 2
        assert queue.bucket_kets == eng.c_queue.bucket_kets
        assert list(hl.cls_total) == list(eng.c_hl.cls_total)
        assert list(hl.n_cls_rows) == list(eng.c_hl.n_cls_rows)
        assert [list(x) for x in hl.cls_ket_seg] == [list(x) for x in eng.c_hl.cls_ket_seg]
        ws_bytes = _lib.load().dftk_jk_workspace_bytes_queue(eng.ns, N, ctypes.byref(queue))
        ws = torch.empty(ws_bytes, dtype=torch.uint8, device=eng.device)
        J = torch.empty((N, N), dtype=torch.float64, device=eng.device)
        K = torch.empty_like(J)
        _lib.call("dftk_jk", ctypes.byref(eng.c_shells), pairs, ctypes.byref(queue), _lib.ptr(D), _lib.ptr(Da),
                  None, _lib.ptr(J), _lib.ptr(K), None, 0, 1e-14, 1e-14, _lib.ptr(ws), ws_bytes, None, stream)
        _lib.call("dftk_jk_hl", ctypes.byref(eng.c_shells), ctypes.byref(hl), _lib.ptr(D), _lib.ptr(Da), None,
                  _lib.ptr(J), _lib.ptr(K), None, 0, 1e-14, _lib.ptr(ws), ws_bytes, None, stream)
        assert torch.abs(J - J0).max().item() < 1e-12 and torch.abs(K - K0).max().item() < 1e-12
