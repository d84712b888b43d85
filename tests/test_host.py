"""Host logic and the C-ABI boundary, without a GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

from dft_b200 import _lib, basis, geometry, shelled
from dft_b200.engine import QCLASS_PAIRS, candidate_offsets

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_shells_match_oracle(oracle_mod):
    atoms, centers = geometry.alkane(10)
    mine = basis.build_shells(basis.load_basis(), atoms, centers)
    ref = oracle_mod.build_shells(oracle_mod.load_basis(basis.STO3G_PATH), atoms, centers)
    assert len(mine) == len(ref) == 52
    for a, b in zip(mine, ref):
        for k in ("angular_momentum", "n_components", "n_contractions", "n_ao", "n_exponents", "ao_start",
                  "ao_stop", "atom_idx"):
            assert a[k] == b[k], k
        np.testing.assert_allclose(a["normalization"], b["normalization"], rtol=1e-15)
        np.testing.assert_array_equal(a["components"], b["components"])
    assert mine[-1]["ao_stop"] == 72


def test_basis_file_matches_reference_format():
    data = basis.load_basis()
    assert set(data) >= {str(z) for z in range(1, 55)}
    o = data["8"]
    assert o[0][0] == [0] and o[1][0] == [0, 1] and len(o[1][2]) == 2


def test_combinations_order():
    assert basis.combinations(1) == [[1, 0, 0], [0, 1, 0], [0, 0, 1]]
    assert basis.combinations(2) == [[2, 0, 0], [1, 1, 0], [0, 2, 0], [1, 0, 1], [0, 1, 1], [0, 0, 2]]


def test_unsupported_basis_is_rejected():
    shells = basis.build_shells(basis.load_basis(), ["21"], np.zeros((1, 3)))  # Sc has d shells
    basis.check_supported(shells)  # d shells are covered
    with pytest.raises(basis.UnsupportedBasis):
        basis.check_sp(shells, "batch")  # the s/p-only paths refuse them
    g_basis = {"1": [[[4], [1.0], [[1.0]]]]}  # g shells are beyond the kernels
    with pytest.raises(basis.UnsupportedBasis):
        basis.check_supported(basis.build_shells(g_basis, ["1"], np.zeros((1, 3))))


def test_geometry_alkane():
    atoms, c = geometry.alkane(10)
    assert atoms.count("6") == 10 and atoms.count("1") == 22
    d = np.linalg.norm(c[:, None] - c[None], axis=-1)
    cc = d[:10, :10][np.triu_indices(10, 1)]
    bond = 1.54 * geometry.ANGSTROM_TO_BOHR
    assert np.sum(np.isclose(cc, bond, atol=1e-9)) == 9
    ch = d[:10, 10:]
    assert np.allclose(np.sort(ch, axis=0)[0], 1.09 * geometry.ANGSTROM_TO_BOHR)
    # every C-C-C and H-C-H angle is tetrahedral
    for k in range(1, 9):
        u, v = c[k - 1] - c[k], c[k + 1] - c[k]
        assert np.isclose(np.dot(u, v) / np.linalg.norm(u) / np.linalg.norm(v), -1 / 3)
    # the chain is planar (all carbons at z = 0)
    assert np.allclose(c[:10, 2], 0)


def test_geometry_clusters_deterministic():
    a1, c1 = geometry.water_cluster((4, 4, 4))
    a2, c2 = geometry.water_cluster((4, 4, 4))
    assert len(a1) == 192
    np.testing.assert_array_equal(c1, c2)
    # monomer O-H bond lengths preserved up to the +-0.3 bohr jitter
    oh = np.linalg.norm(c1[1::3] - c1[0::3], axis=1)
    assert np.all(np.abs(oh - 1.8089) < 0.3 * np.sqrt(3) * 2 + 1e-9)
    batch = geometry.water_cluster_batch(16, 24, seed=3)
    assert len(batch) == 16
    for atoms, cen in batch:
        assert 3 <= len(atoms) <= 72 and cen.shape == (len(atoms), 3)


def test_quartet_order_matches_reference(golden_h2o):
    n = 5
    pl = [(i, j) for i in range(n) for j in range(i + 1)]
    q = shelled.quartet_list(pl)
    np.testing.assert_array_equal(q, golden_h2o["eri_quads"])


def test_process_eri_matches_reference(golden_h2o):
    g = golden_h2o
    eri = {"eri_values": np.arange(int(g["eri_indices"][-1, 1]), dtype=np.float64),
           "eri_indices": g["eri_indices"], "eri_quads": g["eri_quads"], "eri_quads_shapes": g["eri_quads_shapes"]}
    res = shelled.process_eri(eri)
    np.testing.assert_array_equal(res["processed_eri_quads"], g["processed_eri_quads"])
    np.testing.assert_array_equal(res["processed_eri_indices"], g["processed_eri_indices"])
    np.testing.assert_array_equal(res["block_idxs"], g["block_idxs"])
    np.testing.assert_array_equal(res["chunked_quad_shape"], g["chunked_quad_shape"])
    assert g["block_idxs"].shape[0] == 13


def test_candidate_counts_c10h22(oracle_mod, golden_c10h22):
    """Schwarz-surviving unique quartets per class for C10H22 (tau = 1e-12)
    from the oracle's diagonal integrals, against a brute-force count."""
    g = golden_c10h22
    atoms, centers = [str(a) for a in g["atoms"]], g["centers"]
    sh = oracle_mod.build_shells(oracle_mod.load_basis(basis.STO3G_PATH), atoms, centers)
    l = np.array([s["angular_momentum"] for s in sh])
    ii, jj = np.tril_indices(len(sh))
    diag = np.stack([ii, jj, ii, jj], axis=1).astype(np.int32)
    vals, off = oracle_mod.eri_quartets(sh, diag)
    q = np.array([np.sqrt(np.abs(vals[off[t]:off[t + 1]]).max()) for t in range(len(ii))])
    pc = l[ii] + l[jj]
    qs = [np.sort(q[pc == c])[::-1] for c in range(3)]
    counts = []
    for X, Y in QCLASS_PAIRS:
        off_ = candidate_offsets(qs[X], qs[Y], X == Y, 1e-12)
        counts.append(int(off_[-1]))
    # brute force over unique pairs of pairs
    brute = [0] * 6
    from dft_b200.engine import QCLASS_OF
    for X in range(3):
        for Y in range(X + 1):
            prod = np.outer(qs[X], qs[Y]) >= 1e-12
            if X == Y:
                prod = np.tril(prod)
            brute[QCLASS_OF[(X, Y)]] = int(prod.sum())
    assert counts == brute
    assert sum(counts) <= 950131


def test_header_symbols_exported():
    """libdftk.so loads without a GPU and exports every symbol include/dftk.h declares."""
    header = open(os.path.join(REPO, "include", "dftk.h")).read()
    declared = set(re.findall(r"\b(dftk_\w+)\s*\(", header))
    assert declared == set(_lib.SYMBOLS)
    lib = _lib.load()
    for name in declared:
        assert hasattr(lib, name), name
    assert lib.dftk_version() == 100


def test_header_is_plain_c():
    """include/dftk.h and the C host example compile as C99 (no C++ in the ABI)."""
    import shutil
    import subprocess

    if shutil.which("gcc") is None:
        pytest.skip("gcc not found")
    cuda_inc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-fsyntax-only", "-I", os.path.join(REPO, "include"),
                    "-I", cuda_inc, os.path.join(REPO, "tests", "cabi", "jk_host.c")], check=True)


def test_every_symbol_has_argument_types():
    """ctypes passes undeclared integer arguments as 32-bit ints; every entry
    point (64-bit sizes among them) is declared."""
    lib = _lib.load()
    for name in _lib.SYMBOLS:
        assert getattr(lib, name).argtypes is not None, name


def test_cabi_argument_errors_without_gpu():
    """Argument validation happens before any CUDA call and reports through
    the status code and dftk_last_error()."""
    lib = _lib.load()
    st = lib.dftk_jk(None, None, None, None, None, None, None, None, None, 0, 0.0, 0.0, None, 0, None, None)
    assert st == _lib.ERR_ARG
    assert b"null" in lib.dftk_last_error()
    st = lib.dftk_boys(-1, 4, None, None, None)
    assert st == _lib.ERR_ARG
    st = lib.dftk_fma_burn(16, 1, 32, 1, None, None)
    assert st == _lib.ERR_ARG
    assert lib.dftk_prepare_bytes(None, None) == _lib.ERR_ARG
    assert lib.dftk_prepare(None, 1e-12, 1e-15, None, 0, None, None, None) == _lib.ERR_ARG
    assert lib.dftk_jk_workspace_bytes(10, 20) >= 3 * 20 * 20 * 8
    with pytest.raises(_lib.DftkError) as ei:
        _lib.call("dftk_boys", 99, 1, None, None, None)
    assert ei.value.status == _lib.ERR_ARG


def test_batched_purification_matches_eigh_projector():
    """The batched SCF's density step (canonical purification, CPU torch here)
    against the projector onto the n lowest eigenvectors, padded levels empty."""
    import torch

    from dft_b200.batch import _purify

    g = torch.Generator().manual_seed(0)
    B, N, n_real = 16, 40, 33
    A = torch.randn(B, N, N, dtype=torch.float64, generator=g)
    real = torch.ones(B, N, dtype=torch.float64)
    real[:, n_real:] = 0
    F = (A + A.transpose(1, 2)) * 2 * real[:, :, None] * real[:, None, :]
    n = torch.randint(3, 20, (B,), generator=g)
    D = _purify(F, n, real)
    w, U = torch.linalg.eigh(F[:, :n_real, :n_real])
    for b in range(B):
        Uo = U[b][:, : int(n[b])]
        assert (D[b, :n_real, :n_real] - Uo @ Uo.T).abs().max() < 1e-11
    assert D[:, n_real:, :].abs().max() < 1e-12


def test_purify_fully_occupied_blocks():
    """A molecule whose every real level is occupied (one function, or a
    closed shell filling its basis) next to padded levels: D is the identity
    on the real block and zero on the padding, never NaN."""
    import torch

    from dft_b200.batch import _purify

    F = torch.zeros(3, 4, 4, dtype=torch.float64)
    F[0, 0, 0] = -0.9
    F[1, :2, :2] = torch.tensor([[-1.0, 0.2], [0.2, 0.5]])
    F[2] = torch.diag(torch.tensor([-2.0, -1.0, 0.5, 0.7], dtype=torch.float64))
    real = torch.tensor([[1, 0, 0, 0], [1, 1, 0, 0], [1, 1, 1, 1]], dtype=torch.float64)
    D = _purify(F, torch.tensor([1, 2, 4]), real)
    expect = torch.diag_embed(real)
    assert torch.isfinite(D).all()
    assert (D - expect).abs().max() < 1e-12


def test_batched_diis_matches_single():
    import torch

    from dft_b200.batch import _batched_diis
    from dft_b200.scf import _Diis

    g = torch.Generator().manual_seed(1)
    hist, B, N = 5, 3, 6
    F = torch.randn(hist, B, N, N, dtype=torch.float64, generator=g)
    E = torch.randn(hist, B, N, N, dtype=torch.float64, generator=g)
    out = _batched_diis(F, E, hist)
    for b in range(B):
        d = _Diis(8)
        for k in reversed(range(hist)):  # history index 0 is the newest
            d.push(F[k, b], E[k, b])
        assert torch.allclose(out[b], d.extrapolate(), atol=1e-10)


def test_launch_shape_table_without_gpu():
    """dftk_set_launch / dftk_get_launch are host-side: validated and read back."""
    from dft_b200 import autotune

    before = autotune.get_shapes(autotune.FAMILY_JK)
    assert all(t in (64, 128) and 1 <= b <= 32 for t, b in before)
    autotune.set_shapes(autotune.FAMILY_JK, [(64, 8)] * 6)
    assert autotune.get_shapes(autotune.FAMILY_JK) == [(64, 8)] * 6
    autotune.set_shapes(autotune.FAMILY_JK, before)
    lib = _lib.load()
    assert lib.dftk_set_launch(0, 0, 0, 96, 4) == _lib.ERR_ARG
    assert lib.dftk_set_launch(0, 6, 0, 128, 4) == _lib.ERR_ARG
    assert lib.dftk_set_launch(2, 0, 0, 128, 4) == _lib.ERR_ARG
    assert lib.dftk_set_launch(1, 0, 0, 128, 33) == _lib.ERR_ARG
    t = ctypes.c_int()
    assert lib.dftk_set_tile(2, 1, 4) == _lib.OK
    assert lib.dftk_get_tile(2, 1, ctypes.byref(t)) == _lib.OK and t.value == 4
    assert lib.dftk_set_tile(2, 1, 3) == _lib.ERR_ARG
    assert lib.dftk_set_tile(6, 0, 1) == _lib.ERR_ARG
    assert lib.dftk_set_tile(2, 1, 1) == _lib.OK


def test_batch_queue_matches_per_molecule_queues():
    """The batch candidate space (row offsets + ket bases) enumerates exactly
    the union of the molecules' own candidate quartets, with kets indexing
    the concatenated ket list."""
    from dft_b200.batch import batch_row_offsets

    rng = np.random.default_rng(3)
    sizes_x = [5, 0, 9, 3]
    sizes_y = [4, 2, 7, 0]
    qx = [np.sort(rng.uniform(1e-9, 1, n))[::-1] for n in sizes_x]
    qy = [np.sort(rng.uniform(1e-9, 1, n))[::-1] for n in sizes_y]
    seg_x = np.concatenate([[0], np.cumsum(sizes_x)])
    seg_y = np.concatenate([[0], np.cumsum(sizes_y)])
    off, kb = batch_row_offsets(np.concatenate(qx), seg_x, np.concatenate(qy), seg_y, False, 1e-3)
    got = set()
    for r in range(off.size - 1):
        for k in range(off[r + 1] - off[r]):
            got.add((r, int(kb[r]) + k))
    want = set()
    for m in range(4):
        o = candidate_offsets(qx[m], qy[m], False, 1e-3)
        for rl in range(sizes_x[m]):
            for k in range(o[rl + 1] - o[rl]):
                want.add((seg_x[m] + rl, seg_y[m] + k))
    assert got == want and len(got) == off[-1]


def test_batch_pack_index_round_trip():
    import torch

    from dft_b200.batch import pack_index

    nao = np.array([3, 1, 4])
    idx = pack_index(nao, 4)
    assert idx.size == (nao ** 2).sum() and len(set(idx.tolist())) == idx.size
    blocks = [np.arange(n * n, dtype=float).reshape(n, n) + 100 * m for m, n in enumerate(nao)]
    packed = np.concatenate([b.reshape(-1) for b in blocks])
    padded = np.zeros(3 * 16)
    padded[idx] = packed
    padded = padded.reshape(3, 4, 4)
    for m, n in enumerate(nao):
        np.testing.assert_array_equal(padded[m, :n, :n], blocks[m])
        assert not padded[m, n:, :].any() and not padded[m, :, n:].any()


def test_generated_d_classes_are_current():
    """hl_classes.cuh (written by the build from gen_hl.py) is exactly what
    gen_hl.py renders, and the class kind table the host uses equals the one
    the kernels were generated with."""
    import os
    import sys

    from dft_b200 import _lib

    csrc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "dft_b200", "csrc")
    sys.path.insert(0, csrc)
    try:
        import gen_hl
    finally:
        sys.path.remove(csrc)
    path = os.path.join(csrc, "hl_classes.cuh")
    if os.path.exists(path):
        with open(path) as fh:
            assert fh.read() == gen_hl.render()
    kinds = [(gen_hl.kind(la, lb), gen_hl.kind(lc, ld)) for la, lb, lc, ld, _, _ in gen_hl.CLASSES]
    assert kinds == _lib.HLC_CLASS_KINDS


def test_hlc_spaces_enumerate_each_quartet_once():
    """The bucketed candidate spaces of the d classes hold exactly the
    quartets of their two pair kinds whose Schwarz product reaches tau, each
    once ((ds|ds): ket row <= bra row), and every (row, bucket) segment has
    kets of one primitive-count bucket only."""
    from dft_b200 import _lib
    from dft_b200.engine import hlc_bucket, hlc_spaces

    rng = np.random.default_rng(3)
    ns = 40
    l = rng.integers(0, 3, size=ns).astype(np.int32)
    nprim = rng.choice([1, 3, 4, 9], size=ns).astype(np.int32)
    ii, jj = np.tril_indices(ns)
    swap = l[ii] < l[jj]
    a, b = np.where(swap, jj, ii), np.where(swap, ii, jj)
    hi = l[a] >= 2
    sets = {}
    for name, m in (("hi", hi), ("lo", ~hi)):
        q = rng.uniform(1e-9, 1.0, size=int(m.sum()))
        order = np.argsort(-q, kind="stable")
        sets[name] = (a[m][order], b[m][order], q[order])
    tau = 1e-3
    rows, kets, seg, offs = hlc_spaces(l, nprim, sets["hi"][:2], sets["lo"][:2], sets["hi"][2], sets["lo"][2], tau)

    def kind(set_name, r):
        la, lb = l[sets[set_name][0][r]], l[sets[set_name][1][r]]
        return 0 if la == 0 else (1 + lb if la == 1 else 3 + lb)

    nb = _lib.HLC_NB
    for c, (bk, kk) in enumerate(_lib.HLC_CLASS_KINDS):
        kset = "lo" if kk < 3 else "hi"
        got = []
        for i, r in enumerate(rows[bk - 3]):
            for bb in range(nb):
                lo_, hi_ = offs[c][i * nb + bb], offs[c][i * nb + bb + 1]
                for t in range(hi_ - lo_):
                    k = kets[kk][seg[kk][bb] + t]
                    pa, pb = sets[kset][0][k], sets[kset][1][k]
                    assert hlc_bucket(np.array([int(nprim[pa]) * int(nprim[pb])]))[0] == bb
                    got.append((int(r), int(k)))
        want = []
        for r in range(sets["hi"][2].size):
            if kind("hi", r) != bk:
                continue
            for k in range(sets[kset][2].size):
                if kind(kset, k) != kk or sets["hi"][2][r] * sets[kset][2][k] < tau:
                    continue
                if bk == kk and k > r:
                    continue
                want.append((r, k))
        assert sorted(got) == sorted(want) and len(got) == len(set(got)), c


def test_bucket_flag_set_only_for_mixed_primitive_counts():
    """The s/p queue asks the selection pass to group by primitive-count
    bucket only when the s/p pairs span several buckets: never for STO-3G
    (3 x 3 primitives in every pair), always for the generally contracted
    test basis (pairs of 1 to 81 primitive pairs)."""
    import json
    import os

    from dft_b200 import basis
    from dft_b200.engine import hlc_bucket

    def buckets(data, atoms, centers):
        segs = basis.segments(basis.build_shells(data, atoms, centers))
        n = np.array([s["exponents"].size for s in segs])
        l = np.array([s["l"] for s in segs])
        sp = np.nonzero(l <= 1)[0]
        i, j = np.tril_indices(sp.size)
        return np.unique(hlc_bucket(n[sp[i]] * n[sp[j]])).size

    atoms, centers = ["8", "1", "1"], np.array([[0, 0, 0.22], [0, 1.43, -0.89], [0, -1.43, -0.89]])
    assert buckets(basis.load_basis(), atoms, centers) == 1
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "golden", "dz_gc_test.json")) as fh:
        assert buckets(json.load(fh), atoms, centers) > 1


def test_generated_hermite_coefficients_match_recursion():
    """The E^{ab}_t definitions gen_hl.py emits for the d classes (up to a = b
    = 2), evaluated here as Python, equal the McMurchie-Davidson recursion
    E^{a+1,b}_t = h E^{ab}_{t-1} + PA E^{ab}_t + (t+1) E^{ab}_{t+1} (b
    likewise with PB) computed directly."""
    import os
    import re
    import sys

    csrc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "dft_b200", "csrc")
    sys.path.insert(0, csrc)
    try:
        import gen_hl
    finally:
        sys.path.remove(csrc)
    rng = np.random.default_rng(8)
    vals = {"bh": rng.uniform(0.1, 2.0)}
    for x in "xyz":
        vals[f"bA{x}"], vals[f"bB{x}"] = rng.uniform(-2, 2, size=2)
    for line in gen_hl.e_defs("b", 2, 2):
        m = re.match(r"const T (\w+) = (.*);", line)
        expr = re.sub(r"T\((\d+)\)", r"\1", m.group(2))
        vals[m.group(1)] = eval(expr, {}, vals)

    def direct(a, b, pa, pb, h):
        E = {(0, 0): {0: 1.0}}
        for i in range(1, a + 1):
            lo = E[(i - 1, 0)]
            E[(i, 0)] = {t: h * lo.get(t - 1, 0) + pa * lo.get(t, 0) + (t + 1) * lo.get(t + 1, 0) for t in range(i + 1)}
        for i in range(a + 1):
            for j in range(1, b + 1):
                lo = E[(i, j - 1)]
                E[(i, j)] = {t: h * lo.get(t - 1, 0) + pb * lo.get(t, 0) + (t + 1) * lo.get(t + 1, 0)
                             for t in range(i + j + 1)}
        return E

    for axis, x in enumerate("xyz"):
        E = direct(2, 2, vals[f"bA{x}"], vals[f"bB{x}"], vals["bh"])
        for a in range(3):
            for b in range(3):
                for t, v in gen_hl.e1d("b", a, b, axis).items():
                    got = 1.0 if v is None else vals[v]  # None: the factor 1 of E^{00}_0
                    assert abs(got - E[(a, b)][t]) <= 1e-12 * max(1.0, abs(E[(a, b)][t])), (a, b, t)
