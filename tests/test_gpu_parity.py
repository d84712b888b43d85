"""CUDA path vs the oracle and the reference's golden outputs (needs a GPU).

Tolerances: 1e-12 absolute per FP64 ERI and J/K element (the parity bar for
the FP64 path), 1e-8 Eh on total energies.
"""
import ctypes

import numpy as np
import pytest
import scipy.special
import torch

from dft_b200 import _lib, basis, geometry, shelled
from dft_b200.engine import IntegralEngine

pytestmark = pytest.mark.gpu

ERI_TOL = 1e-12


def _mol(g):
    return [str(a) for a in g["atoms"]], np.asarray(g["centers"])


def _shells(atoms, centers):
    return basis.build_shells(basis.load_basis(), atoms, centers)


def test_boys_fp64_fp32():
    """GPU Boys against 40-digit mpmath values (tests/golden/make_boys.py)."""
    from conftest import load_golden

    g = load_golden("boys_mpmath.npz")
    T, ref_all = g["T"], g["F"]
    d_T = torch.as_tensor(T, device="cuda")
    # 5e-15 relative through the orders the ERI kernels use (m <= 5); the
    # higher orders lose a little in the upward recursion beyond the table
    for mmax in (0, 1, 4, 5, 8):
        F = torch.empty(T.size * (mmax + 1), dtype=torch.float64, device="cuda")
        _lib.call("dftk_boys", mmax, T.size, _lib.ptr(d_T), _lib.ptr(F), _lib.stream_handle())
        F = F.cpu().numpy().reshape(-1, mmax + 1)
        for m in range(mmax + 1):
            ref = ref_all[:, m]
            err = np.abs(F[:, m] - ref) / np.maximum(np.abs(ref), 1e-300)
            tol = 5e-15 if m <= 5 else 1e-13
            assert err.max() < tol, (mmax, m, T[err.argmax()], err.max())
    T32 = torch.as_tensor(g["T32"], device="cuda")
    F32 = torch.empty(T.size * 5, dtype=torch.float32, device="cuda")
    _lib.call("dftk_boys32", 4, T.size, _lib.ptr(T32), _lib.ptr(F32), _lib.stream_handle())
    F32 = F32.cpu().numpy().reshape(-1, 5).astype(np.float64)
    for m in range(5):
        ref = g["F32"][:, m]
        ok = ref > 1e-30
        assert (np.abs(F32[ok, m] - ref[ok]) / ref[ok]).max() < 2e-6


def test_dropin_kernels_match_oracle(oracle_mod):
    """dftk_nuclear_kernel / dftk_eri_kernel against the oracle's restatement
    of the reference kernels, same arguments and layouts."""
    lib = oracle_mod.lib()
    rng = np.random.default_rng(11)
    p_ = lambda a: ctypes.c_void_p(a.ctypes.data)
    for trial in range(12):
        la, lb = (int(x) for x in rng.integers(0, 3, size=2))
        pa = np.array(basis.combinations(la), dtype=np.int32)
        pb = np.array(basis.combinations(lb), dtype=np.int32)
        ea, eb = rng.uniform(0.1, 40, size=3), rng.uniform(0.1, 40, size=2)
        exp_a, pow_a = np.tile(ea, len(pa)), np.repeat(pa, ea.size, axis=0).reshape(-1, 3).copy()
        exp_b, pow_b = np.tile(eb, len(pb)), np.repeat(pb, eb.size, axis=0).reshape(-1, 3).copy()
        ca, cb = rng.normal(size=3), rng.normal(size=3) * 2
        Z = np.array([1, 8, 6, 7], dtype=np.int32)
        xyz = rng.normal(size=(4, 3)) * 2.5
        na, nb = exp_a.size, exp_b.size
        K = na * nb
        host = [np.zeros(K), np.zeros(7 * K), np.zeros(7 * K), np.zeros(7 * K), np.zeros(K), np.zeros(3 * K),
                np.zeros(K, np.int32), np.zeros(K, np.int32), np.zeros(K, np.int32)]
        lib.orc_pair_prims(ctypes.c_int(na), p_(exp_a), p_(pow_a), p_(ca), ctypes.c_int(nb), p_(exp_b), p_(pow_b),
                           p_(cb), ctypes.c_int(4), p_(Z), p_(xyz), *[p_(h) for h in host])
        cu = lambda a: torch.as_tensor(a).cuda()
        dev = [torch.zeros_like(cu(h)) for h in host]
        shelled.nuclear_kernel(None, None, (cu(exp_a), cu(exp_b), cu(ca), cu(cb), cu(pow_a), cu(pow_b), cu(Z),
                                            cu(xyz), 4, na, nb, *dev))
        for h, d in zip(host, dev):
            np.testing.assert_allclose(d.cpu().numpy(), h, atol=1e-12, rtol=1e-12)
        V, Ex, Ey, Ez, p, P, nx, ny, nz = host
        out_h = np.zeros(K * K)
        pair = [p_(p), p_(P), p_(Ex), p_(Ey), p_(Ez), p_(nx), p_(ny), p_(nz)]
        lib.orc_eri_prims(ctypes.c_int(K), *pair, ctypes.c_int(K), *pair, p_(out_h))
        dpair = dev[4], dev[5], dev[1], dev[2], dev[3], dev[6], dev[7], dev[8]
        out_d = torch.zeros(K * K, dtype=torch.float64, device="cuda")
        shelled.eri_kernel(None, None, (K, *dpair, K, *dpair, out_d))
        np.testing.assert_allclose(out_d.cpu().numpy(), out_h, atol=1e-12, rtol=1e-12)


def test_h2o_calc_eri_process_eri_golden(golden_h2o, tmp_path):
    g = golden_h2o
    atoms, centers = _mol(g)
    sh = _shells(atoms, centers)
    pair_list, pair_cache = shelled.pair_data(sh, atoms, centers)
    eri = shelled.calc_eri(pair_list, pair_cache, sh, out_dir=str(tmp_path))
    np.testing.assert_array_equal(eri["eri_quads"], g["eri_quads"])
    np.testing.assert_array_equal(eri["eri_indices"], g["eri_indices"])
    proc = shelled.process_eri(out_dir=str(tmp_path))
    np.testing.assert_array_equal(proc["processed_eri_quads"], g["processed_eri_quads"])
    np.testing.assert_allclose(proc["processed_eri_values"], g["processed_eri_values"], atol=ERI_TOL, rtol=0)
    # the lazily filled pair cache carries the reference's pair records
    rec = pair_cache[(2, 1)]
    assert rec["K"] == 9 * 3 and rec["Ex"].numel() == 7 * rec["K"]


def test_one_electron_golden(golden_h2o, golden_c10h22):
    for g in (golden_h2o, golden_c10h22):
        atoms, centers = _mol(g)
        S, T, V = shelled.one_electron(_shells(atoms, centers), atoms, centers)
        np.testing.assert_allclose(S.cpu().numpy(), g["overlaps"], atol=1e-13, rtol=0)
        np.testing.assert_allclose(T.cpu().numpy(), g["T_matrix"], atol=1e-12, rtol=0)
        np.testing.assert_allclose(V.cpu().numpy(), g["V_matrix"], atol=1e-11, rtol=0)


def test_c10h22_all_eris_vs_oracle(oracle_mod, golden_c10h22):
    g = golden_c10h22
    atoms, centers = _mol(g)
    sh = _shells(atoms, centers)
    q = shelled.quartet_list([(i, j) for i in range(len(sh)) for j in range(i + 1)])
    assert q.shape[0] == 950131
    eng = shelled.get_engine(sh)
    vals, off = eng.eri_blocks(q)
    ref, ref_off = oracle_mod.eri_quartets(oracle_mod.build_shells(oracle_mod.load_basis(basis.STO3G_PATH), atoms,
                                                                   centers), q)
    np.testing.assert_array_equal(off, ref_off)
    diff = np.abs(vals.cpu().numpy() - ref)
    assert diff.max() < ERI_TOL, diff.max()
    # and the reference's own values on its sampled quartets
    sv, _ = eng.eri_blocks(g["sample_quads"])
    np.testing.assert_allclose(sv.cpu().numpy(), g["sample_values"], atol=ERI_TOL, rtol=0)


def test_h2o64_sample_golden(golden_h2o64):
    g = golden_h2o64
    atoms, centers = _mol(g)
    eng = shelled.get_engine(_shells(atoms, centers))
    v, off = eng.eri_blocks(g["sample_quads"])
    np.testing.assert_array_equal(off, g["sample_offsets"])
    np.testing.assert_allclose(v.cpu().numpy(), g["sample_values"], atol=ERI_TOL, rtol=0)


def test_jk_h2o_golden_uhf_and_rhf(golden_h2o):
    g = golden_h2o
    atoms, centers = _mol(g)
    sh = _shells(atoms, centers)
    Pa, Pb = g["P_a"], g["P_b"]
    N = Pa.shape[0]
    # the reference's in-place call shape with NumPy arrays (UHF path: distinct P_a, P_b objects)
    J, Ka, Kb = np.zeros((N, N)), np.zeros((N, N)), np.zeros((N, N))
    shelled.fill_matrices(sh, Pa + Pb, Pa, Pb.copy(), J, Ka, Kb)
    np.testing.assert_allclose(J, g["J_matrix"], atol=ERI_TOL)
    np.testing.assert_allclose(Ka, g["K_a"], atol=ERI_TOL)
    np.testing.assert_allclose(Kb, g["K_b"], atol=ERI_TOL)
    # in place: a second call accumulates
    shelled.fill_matrices(sh, Pa + Pb, Pa, Pb.copy(), J, Ka, Kb)
    np.testing.assert_allclose(J, 2 * g["J_matrix"], atol=2 * ERI_TOL)
    # RHF path (same density object) and CUDA tensors
    Pt = torch.as_tensor(Pa).cuda()
    Jt, Kat, Kbt = (torch.zeros((N, N), dtype=torch.float64, device="cuda") for _ in range(3))
    shelled.fill_matrices(sh, 2 * Pt, Pt, Pt, Jt, Kat, Kbt)
    np.testing.assert_allclose(Jt.cpu().numpy(), g["J_matrix"], atol=ERI_TOL)
    np.testing.assert_allclose(Kbt.cpu().numpy(), g["K_a"], atol=ERI_TOL)


def test_jk_c10h22_golden_unscreened(golden_c10h22):
    g = golden_c10h22
    atoms, centers = _mol(g)
    eng = shelled.get_engine(_shells(atoms, centers), tau_schwarz=0.0)
    # tau = 0 keeps every quartet except those of pairs whose Gaussian product
    # factor underflows to exactly zero
    assert 940000 < sum(eng.quartet_totals()) <= 950131
    Pa = torch.as_tensor(g["P_a"]).cuda()
    J, Ka, _ = eng.jk(2 * Pa, Pa, tau=0.0)
    np.testing.assert_allclose(J.cpu().numpy(), g["J_matrix"], atol=1e-11)
    np.testing.assert_allclose(Ka.cpu().numpy(), g["K_a"], atol=1e-11)
    # screened at 1e-12 the result moves by far less than 1e-8
    eng2 = shelled.get_engine(_shells(atoms, centers), tau_schwarz=1e-12)
    J2, K2, _ = eng2.jk(2 * Pa, Pa, tau=1e-14)
    assert (J2 - J).abs().max().item() < 1e-9 and (K2 - Ka).abs().max().item() < 1e-9


def test_jk_water8_vs_oracle_direct(oracle_mod):
    atoms, centers = geometry.water_cluster((2, 2, 2), seed=7)
    sh = _shells(atoms, centers)
    N = sh[-1]["ao_stop"]
    rng = np.random.default_rng(3)
    A = rng.normal(size=(N, N))
    Pa = (A + A.T) * 0.05
    B = rng.normal(size=(N, N))
    Pb = (B + B.T) * 0.05
    osh = oracle_mod.build_shells(oracle_mod.load_basis(basis.STO3G_PATH), atoms, centers)
    q = oracle_mod.quartet_list(len(osh))
    J0, Ka0, Kb0 = oracle_mod.direct_jk(osh, q, Pa + Pb, Pa, Pb)
    eng = IntegralEngine(sh, tau_schwarz=0.0)
    J, Ka, Kb = eng.jk(torch.as_tensor(Pa + Pb).cuda(), torch.as_tensor(Pa).cuda(), torch.as_tensor(Pb).cuda(),
                       uhf=True, tau=0.0)
    np.testing.assert_allclose(J.cpu().numpy(), J0, atol=1e-11)
    np.testing.assert_allclose(Ka.cpu().numpy(), Ka0, atol=1e-11)
    np.testing.assert_allclose(Kb.cpu().numpy(), Kb0, atol=1e-11)


def test_jk_screened_lanes_vs_oracle(oracle_mod):
    """Density screening and the FP32 split leave warps with skipped lanes;
    the result must still match the oracle's unscreened J/K to within what
    the skipped quartets can carry."""
    atoms, centers = geometry.water_cluster((2, 2, 2), seed=7)
    sh = _shells(atoms, centers)
    N = sh[-1]["ao_stop"]
    rng = np.random.default_rng(9)
    A = rng.normal(size=(N, N)) * (rng.random(size=(N, N)) < 0.15)
    Pa = 0.05 * (A + A.T)
    osh = oracle_mod.build_shells(oracle_mod.load_basis(basis.STO3G_PATH), atoms, centers)
    J0, K0, _ = oracle_mod.direct_jk(osh, oracle_mod.quartet_list(len(osh)), 2 * Pa, Pa, Pa)
    eng = IntegralEngine(sh, tau_schwarz=0.0)
    D = torch.as_tensor(2 * Pa).cuda()
    J, K, _ = eng.jk(D, 0.5 * D, tau=1e-9)
    assert np.abs(J.cpu().numpy() - J0).max() < 1e-6 and np.abs(K.cpu().numpy() - K0).max() < 1e-6
    counts = torch.zeros(24, dtype=torch.int64, device="cuda")
    Jm, Km, _ = eng.jk(D, 0.5 * D, mixed=True, tau=0.0, tau_fp32=1e-4, counts=counts)
    assert counts[6:12].sum().item() > 0 and counts[:6].sum().item() > 0
    assert np.abs(Jm.cpu().numpy() - J0).max() < 1e-8 and np.abs(Km.cpu().numpy() - K0).max() < 1e-8


def test_jk_properties_h2o64():
    """Full-size (H2O)_64: symmetry, linearity in D, run-to-run agreement,
    FP32/FP64 split accounting."""
    atoms, centers = geometry.water_cluster((4, 4, 4))
    eng = IntegralEngine(_shells(atoms, centers), tau_schwarz=1e-12)
    N = eng.n_ao
    assert N == 448
    rng = np.random.default_rng(0)
    A = torch.as_tensor(rng.normal(size=(N, N)) * 0.02).cuda()
    D1 = A + A.T
    B = torch.as_tensor(rng.normal(size=(N, N)) * 0.02).cuda()
    D2 = B + B.T
    J1, K1, _ = eng.jk(D1, 0.5 * D1, tau=0.0)
    J2, K2, _ = eng.jk(D2, 0.5 * D2, tau=0.0)
    J12, K12, _ = eng.jk(D1 + D2, 0.5 * (D1 + D2), tau=0.0)
    assert (J1 - J1.T).abs().max() < 1e-13 and (K1 - K1.T).abs().max() < 1e-13
    assert (J12 - J1 - J2).abs().max() < 1e-11 and (K12 - K1 - K2).abs().max() < 1e-11
    Jr, Kr, _ = eng.jk(D1, 0.5 * D1, tau=0.0)
    assert (Jr - J1).abs().max() < 1e-12
    counts = torch.zeros(24, dtype=torch.int64, device="cuda")
    eng.jk(D1, 0.5 * D1, tau=0.0, counts=counts)
    assert counts[:6].tolist() == eng.quartet_totals()
    counts.zero_()
    Jm, Km, _ = eng.jk(D1, 0.5 * D1, mixed=True, tau=0.0, tau_fp32=1e-5, counts=counts)
    c = counts.tolist()
    assert sum(c[:6]) + sum(c[6:12]) == sum(eng.quartet_totals()) and sum(c[6:12]) > 0
    assert (Jm - J1).abs().max() < 1e-7 and (Km - K1).abs().max() < 1e-7


def test_select_lists_match_direct_scan():
    """The selection pass + list kernels and the direct scan path agree, with
    density screening and the FP32 split active, and count the same quartets."""
    atoms, centers = geometry.water_cluster((2, 2, 2), seed=7)
    eng = IntegralEngine(_shells(atoms, centers), tau_schwarz=1e-12)
    N = eng.n_ao
    rng = np.random.default_rng(21)
    A = rng.normal(size=(N, N)) * (rng.random(size=(N, N)) < 0.2)
    D = torch.as_tensor(0.1 * (A + A.T)).cuda()
    for kw in (dict(tau=1e-10), dict(mixed=True, tau=1e-12, tau_fp32=1e-5)):
        c_list = torch.zeros(24, dtype=torch.int64, device="cuda")
        c_scan = torch.zeros(24, dtype=torch.int64, device="cuda")
        J1, K1, _ = eng.jk(D, 0.5 * D, counts=c_list, **kw)
        J2, K2, _ = eng.jk(D, 0.5 * D, counts=c_scan, scan=True, **kw)
        assert (J1 - J2).abs().max().item() < 1e-12 and (K1 - K2).abs().max().item() < 1e-12
        assert c_list.tolist() == c_scan.tolist()
        assert c_list[:6].sum().item() > 0


def test_h2o64_jk_rows_vs_oracle(oracle_mod):
    """Full-size digestion path: on (H2O)_64 (448 basis functions) a queue
    restricted to a few bra rows of every class (their whole Schwarz-kept ket
    prefix: strong, middle and weak bra pairs) against the oracle's direct J/K
    over exactly those quartets, at the converged-looking random density."""
    import ctypes

    from dft_b200 import _lib
    from dft_b200.engine import QCLASS_PAIRS

    atoms, centers = geometry.water_cluster((4, 4, 4))
    sh = _shells(atoms, centers)
    eng = IntegralEngine(sh, tau_schwarz=1e-12)
    N = eng.n_ao
    rng = np.random.default_rng(11)
    M = rng.normal(size=(N, N)) * np.exp(-0.05 * np.abs(np.subtract.outer(np.arange(N), np.arange(N))))
    P = 0.05 * (M + M.T)
    q = _lib.Queue()
    keep, quads = [], []
    for c, (X, Y) in enumerate(QCLASS_PAIRS):
        off = eng.row_off[c].cpu().numpy()
        n_rows = off.size - 1
        rows = sorted({0, 1, n_rows // 3, n_rows // 2, n_rows - 1} & set(range(n_rows)))
        cnt = np.zeros(n_rows, dtype=np.int64)
        for r in rows:
            cnt[r] = off[r + 1] - off[r]
        new = np.concatenate([[0], np.cumsum(cnt)]).astype(np.int64)
        d_off = torch.as_tensor(new, device=eng.device)
        keep.append(d_off)
        q.n_rows[c] = eng.c_queue.n_rows[c] if new[-1] > 0 else 0
        q.total[c] = int(new[-1])
        q.row_off[c] = _lib.ptr(d_off).value
        abx = eng.pair_bufs[X]["ab"].cpu().numpy().reshape(-1, 2)
        aby = eng.pair_bufs[Y]["ab"].cpu().numpy().reshape(-1, 2)
        for r in rows:
            k = np.arange(cnt[r])
            quads.append(np.hstack([np.repeat(abx[r][None], k.size, 0), aby[k]]))
    q.tau_prim = eng.c_queue.tau_prim
    quads = np.vstack(quads).astype(np.int32)
    assert quads.shape[0] > 10000
    dev = eng.device
    J, K, _ = eng.jk(torch.as_tensor(2 * P, device=dev), torch.as_tensor(P, device=dev), tau=0.0, queue=q)
    osh = oracle_mod.build_shells(oracle_mod.load_basis(basis.STO3G_PATH), atoms, centers)
    J0, K0, _ = oracle_mod.direct_jk(osh, quads, 2 * P, P, P)
    for A_, B_ in ((J, J0), (K, K0)):
        err = np.abs(A_.cpu().numpy() - B_).max()
        assert err < 1e-11, err
