"""d and f shells and general contractions on the GPU against the reference's
own outputs (tests/golden/make_golden.py br2 / gc / gcf) and the oracle.

* Br2 / STO-3G (3d shells on both atoms): every processed ERI at 1e-12
  absolute, S/T/V in the reference's spherical basis, J/K at the reference's
  converged densities, and the SCF energy of the reference loop at 1e-8 Eh.
* H2O with a generally contracted, d-polarised test basis, and the same with
  an f shell on O and a d shell on H: S/T/V, J/K and the energy (reference
  loop and the RHF/DIIS driver) at 1e-8 Eh.
* J/K with random densities against the oracle's direct J/K (1e-11).
"""
import ctypes
import json
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN, load_golden
from dft_b200 import _lib, basis, geometry, shelled
from dft_b200.engine import IntegralEngine
from dft_b200.scf import scf_reference, scf_rhf

pytestmark = pytest.mark.gpu

ERI_TOL = 1e-12
GC_BASIS = os.path.join(GOLDEN, "dz_gc_test.json")
GCF_BASIS = os.path.join(GOLDEN, "dzf_gc_test.json")
CASES = {"br2": ("br2.npz", None), "gc": ("h2o_gc.npz", GC_BASIS), "gcf": ("h2o_gcf.npz", GCF_BASIS)}


def _mol(g):
    return [str(a) for a in g["atoms"]], np.asarray(g["centers"])


def _gc_basis(path=GC_BASIS):
    with open(path) as fh:
        return json.load(fh)


def _case(case):
    name, path = CASES[case]
    g = load_golden(name)
    return g, (basis.load_basis() if path is None else _gc_basis(path))


def _sph(A, M):
    return A @ M @ A.T


def test_br2_all_eris_match_reference(tmp_path):
    g = load_golden("br2.npz")
    atoms, centers = _mol(g)
    sh = basis.build_shells(basis.load_basis(), atoms, centers)
    pair_list, pair_cache = shelled.pair_data(sh, atoms, centers)
    eri = shelled.calc_eri(pair_list, pair_cache, sh, out_dir=str(tmp_path))
    np.testing.assert_array_equal(eri["eri_quads"], g["eri_quads"])
    np.testing.assert_array_equal(eri["eri_indices"], g["eri_indices"])
    proc = shelled.process_eri(out_dir=str(tmp_path))
    np.testing.assert_array_equal(proc["processed_eri_quads"], g["processed_eri_quads"])
    err = np.abs(proc["processed_eri_values"] - g["processed_eri_values"])
    assert err.max() < ERI_TOL, err.max()


@pytest.mark.parametrize("case", ["br2", "gc", "gcf"])
def test_one_electron_spherical_match_reference(case):
    g, data = _case(case)
    atoms, centers = _mol(g)
    sh = basis.build_shells(data, atoms, centers)
    A = basis.spherical_transform(sh)
    np.testing.assert_allclose(A, g["A"], atol=1e-15, rtol=0)
    S, T, V = shelled.one_electron(sh, atoms, centers)
    for M, key in ((S, "overlaps"), (T, "T_matrix"), (V, "V_matrix")):
        ref = g[key]
        err = np.abs(_sph(A, M.cpu().numpy()) - ref).max()
        assert err < 1e-12 * max(1.0, np.abs(ref).max()), (key, err)


@pytest.mark.parametrize("case", ["br2", "gc", "gcf"])
def test_jk_at_reference_density(case):
    """fill_matrices at the reference's converged densities (UHF call shape),
    compared in the reference's spherical basis."""
    g, data = _case(case)
    atoms, centers = _mol(g)
    sh = basis.build_shells(data, atoms, centers)
    A = g["A"]
    Pa_c, Pb_c = A.T @ g["P_a"] @ A, A.T @ g["P_b"] @ A
    N = A.shape[1]
    J, Ka, Kb = np.zeros((N, N)), np.zeros((N, N)), np.zeros((N, N))
    shelled.fill_matrices(sh, Pa_c + Pb_c, Pa_c, Pb_c.copy(), J, Ka, Kb)
    for M, key in ((J, "J_matrix"), (Ka, "K_a"), (Kb, "K_b")):
        ref = g[key]
        err = np.abs(_sph(A, M) - ref).max()
        assert err < 1e-11 * max(1.0, np.abs(ref).max()), (key, err)


@pytest.mark.parametrize("case", ["br2", "gc", "gcf"])
def test_scf_energy_matches_reference(case):
    g, data = _case(case)
    atoms, centers = _mol(g)
    sh = basis.build_shells(data, atoms, centers)
    eng = IntegralEngine(sh, tau_schwarz=0.0)
    S, T, V = eng.one_electron(atoms, centers)
    n = basis.n_electrons(atoms)
    e_nn = geometry.nuclear_repulsion(atoms, centers)
    r = scf_reference(eng, T + V, S, n // 2, n // 2, e_nn, etol=1e-11, ptol=1e-8)
    assert abs(r.energy - g["energy"]) < 1e-8, (r.energy, g["energy"])
    r2 = scf_rhf(eng, T + V, S, n // 2, e_nn, tau=1e-13)
    assert abs(r2.energy - g["energy"]) < 1e-8, (r2.energy, g["energy"])


@pytest.mark.parametrize("case", ["br2", "gc"])
def test_jk_random_density_vs_oracle(oracle_mod, case):
    """Every quartet, UHF densities with no structure: the d path and the
    segmented general contractions against the oracle's direct J/K."""
    if case == "br2":
        atoms, centers = ["35", "1"], np.array([[0.0, 0.0, 0.0], [0.3, 0.1, 2.7]])
        data = basis.load_basis()
    else:
        atoms, centers = geometry.water()
        data = _gc_basis()
    sh = basis.build_shells(data, atoms, centers)
    eng = IntegralEngine(sh, tau_schwarz=0.0)
    N = eng.n_ao
    rng = np.random.default_rng(7)
    M1, M2 = rng.normal(size=(N, N)), rng.normal(size=(N, N))
    Pa, Pb = 0.1 * (M1 + M1.T), 0.1 * (M2 + M2.T)
    dev = eng.device
    J, Ka, Kb = eng.jk(torch.as_tensor(Pa + Pb, device=dev), torch.as_tensor(Pa, device=dev),
                       torch.as_tensor(Pb, device=dev), uhf=True, tau=0.0)
    osh = oracle_mod.build_shells(data, atoms, centers)
    q = oracle_mod.quartet_list(len(osh))
    J0, Ka0, Kb0 = oracle_mod.direct_jk(osh, q, Pa + Pb, Pa, Pb)
    for M, M0 in ((J, J0), (Ka, Ka0), (Kb, Kb0)):
        err = np.abs(M.cpu().numpy() - M0).max()
        assert err < 1e-11 * max(1.0, np.abs(M0).max()), err


def test_br2_eri_blocks_vs_oracle(oracle_mod):
    """HBr quartets through dftk_hl_eri_blocks / dftk_eri_blocks against the
    oracle's contracted blocks, every quartet."""
    atoms, centers = ["35", "1"], np.array([[0.0, 0.0, 0.0], [0.3, 0.1, 2.7]])
    sh = basis.build_shells(basis.load_basis(), atoms, centers)
    eng = IntegralEngine(sh, tau_schwarz=0.0)
    q = shelled.quartet_list([(i, j) for i in range(len(sh)) for j in range(i + 1)])
    vals, off = eng.eri_blocks(q)
    osh = oracle_mod.build_shells(basis.load_basis(), atoms, centers)
    v0, off0 = oracle_mod.eri_quartets(osh, q)
    np.testing.assert_array_equal(off, off0)
    assert np.abs(vals.cpu().numpy() - v0).max() < ERI_TOL


def test_f_shell_eris_and_jk_vs_oracle(oracle_mod):
    """HF with STO-3G plus an f shell on each atom (single contractions): every
    ERI block through dftk_hl_eri_blocks against the oracle at 1e-12, and J/K
    with random densities at 1e-11 relative."""
    data = basis.load_basis()
    data = {"1": data["1"] + [[[3], [0.8], [[1.0]]]], "9": data["9"] + [[[3], [1.1], [[1.0]]]]}
    atoms, centers = ["9", "1"], np.array([[0.0, 0.0, 0.0], [0.2, -0.1, 1.75]])
    sh = basis.build_shells(data, atoms, centers)
    eng = IntegralEngine(sh, tau_schwarz=0.0)
    assert eng.hl_lmax == 3
    q = shelled.quartet_list([(i, j) for i in range(len(sh)) for j in range(i + 1)])
    vals, off = eng.eri_blocks(q)
    osh = oracle_mod.build_shells(data, atoms, centers)
    v0, off0 = oracle_mod.eri_quartets(osh, q)
    np.testing.assert_array_equal(off, off0)
    assert np.abs(vals.cpu().numpy() - v0).max() < ERI_TOL
    N = eng.n_ao
    rng = np.random.default_rng(3)
    M = rng.normal(size=(N, N))
    P = 0.1 * (M + M.T)
    dev = eng.device
    J, K, _ = eng.jk(torch.as_tensor(2 * P, device=dev), torch.as_tensor(P, device=dev), tau=0.0)
    J0, K0, _ = oracle_mod.direct_jk(osh, q, 2 * P, P, P)
    for A_, B_ in ((J, J0), (K, K0)):
        assert np.abs(A_.cpu().numpy() - B_).max() < 1e-11 * max(1.0, np.abs(B_).max())


def test_thread_classes_match_warp_path_and_oracle(oracle_mod):
    """(H2O)_2 with the generally contracted d-polarised basis: the generated
    thread-per-quartet kernels of the fifteen generated d classes (every d
    class, no warp kernel) give the warp kernel's J/K alone (1e-12) and the
    oracle's direct J/K (1e-11 relative), UHF densities with no structure."""
    atoms, centers = geometry.water_cluster((1, 1, 2))
    data = _gc_basis()
    sh = basis.build_shells(data, atoms, centers)
    eng = IntegralEngine(sh, tau_schwarz=0.0)
    warp = IntegralEngine(sh, tau_schwarz=0.0, hl_classes=False)
    assert all(t > 0 for t in eng.hlc_totals)
    # with no f shells every d quartet belongs to a class: the warp kernel's
    # spaces are empty, and the class spaces hold exactly its candidates
    lo_classes = [c for c, (bk, kk) in enumerate(_lib.HLC_CLASS_KINDS) if kk < 3]
    hi_classes = [c for c, (bk, kk) in enumerate(_lib.HLC_CLASS_KINDS) if kk >= 3]
    assert eng.hl_totals == [0, 0] and sum(warp.hlc_totals) == 0
    assert sum(eng.hlc_totals[c] for c in lo_classes) == warp.hl_totals[0]
    assert sum(eng.hlc_totals[c] for c in hi_classes) == warp.hl_totals[1]
    N = eng.n_ao
    rng = np.random.default_rng(17)
    M1, M2 = rng.normal(size=(N, N)), rng.normal(size=(N, N))
    Pa, Pb = 0.1 * (M1 + M1.T), 0.1 * (M2 + M2.T)
    dev = eng.device
    args = [torch.as_tensor(x, device=dev) for x in (Pa + Pb, Pa, Pb)]
    J, Ka, Kb = eng.jk(*args, uhf=True, tau=0.0)
    J1, Ka1, Kb1 = warp.jk(*args, uhf=True, tau=0.0)
    for A_, B_ in ((J, J1), (Ka, Ka1), (Kb, Kb1)):
        assert torch.abs(A_ - B_).max().item() < 1e-12 * max(1.0, torch.abs(B_).max().item())
    osh = oracle_mod.build_shells(data, atoms, centers)
    q = oracle_mod.quartet_list(len(osh))
    J0, Ka0, Kb0 = oracle_mod.direct_jk(osh, q, Pa + Pb, Pa, Pb)
    for M, M0 in ((J, J0), (Ka, Ka0), (Kb, Kb0)):
        err = np.abs(M.cpu().numpy() - M0).max()
        assert err < 1e-11 * max(1.0, np.abs(M0).max()), err


def test_thread_classes_screened_density_counts():
    """Screening through the class kernels: at a tau that cuts part of the
    d quartets the J/K still equal the warp kernel's at the same tau, and the
    evaluated-quartet counters of both paths agree (every quartet is
    evaluated by exactly one kernel)."""
    atoms, centers = geometry.water_cluster((1, 2, 2))
    sh = basis.build_shells(_gc_basis(), atoms, centers)
    eng = IntegralEngine(sh, tau_schwarz=1e-12)
    warp = IntegralEngine(sh, tau_schwarz=1e-12, hl_classes=False)
    N = eng.n_ao
    rng = np.random.default_rng(5)
    M = rng.normal(size=(N, N)) * np.exp(-0.3 * np.abs(np.subtract.outer(np.arange(N), np.arange(N))))
    D = torch.as_tensor(0.05 * (M + M.T), device=eng.device)
    Dh = (0.5 * D).contiguous()
    out = []
    for e in (eng, warp):
        counts = torch.zeros(2, dtype=torch.int64, device=e.device)
        J = torch.zeros((N, N), dtype=torch.float64, device=e.device)
        K = torch.zeros_like(J)
        _lib.call("dftk_jk_hl", ctypes.byref(e.c_shells), ctypes.byref(e.c_hl), _lib.ptr(D), _lib.ptr(Dh), None,
                  _lib.ptr(J), _lib.ptr(K), None, 0, 1e-9, _lib.ptr(e.workspace), e.workspace_bytes,
                  _lib.ptr(counts), _lib.stream_handle())
        out.append((J, K, int(counts[0].item())))
    (J, K, n), (J1, K1, n1) = out
    assert n == n1 and n > 0
    assert torch.abs(J - J1).max().item() < 1e-12 and torch.abs(K - K1).max().item() < 1e-12
