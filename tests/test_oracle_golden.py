"""Pin the CPU oracle against the reference's own outputs (CPU only).

The fixtures in tests/golden/ were produced by running the reference's
shelled.py (tests/golden/make_golden.py); oracle/_ref is the reference's
kernel source compiled as host code (oracle/build_ref.py)."""
import ctypes
import math

import numpy as np
import pytest
import scipy.special

from dft_b200 import geometry


def _shells(oracle_mod, atoms, centers):
    basis = oracle_mod.load_basis(_basis_path())
    return oracle_mod.build_shells(basis, [str(a) for a in atoms], centers)


def _basis_path():
    from dft_b200 import basis

    return basis.STO3G_PATH


def test_boys_against_scipy(oracle_mod):
    # F_m(T) = 1F1(m + 1/2; m + 3/2; -T) / (2m + 1).  The reference's
    # alternating 40-term series (shelled.py:174-182) cancels ~2 digits just
    # below T = 6, so its own accuracy there is ~1e-13.
    for T in [0.0, 1e-15, 1e-6, 0.3, 2.0, 5.99, 6.0, 6.5, 17.0, 40.0, 120.0]:
        F = oracle_mod.boys(6, T)
        for m in range(6):
            ref = scipy.special.hyp1f1(m + 0.5, m + 1.5, -T) / (2 * m + 1)
            assert abs(F[m] - ref) <= 3e-13 * max(1.0, abs(ref)), (T, m)


def test_h2o_one_electron(oracle_mod, golden_h2o):
    atoms, centers = [str(a) for a in golden_h2o["atoms"]], golden_h2o["centers"]
    sh = _shells(oracle_mod, atoms, centers)
    S, T, V = oracle_mod.one_electron(sh, atoms, centers)
    np.testing.assert_allclose(S, golden_h2o["overlaps"], atol=1e-13, rtol=0)
    np.testing.assert_allclose(T, golden_h2o["T_matrix"], atol=1e-12, rtol=0)
    np.testing.assert_allclose(V, golden_h2o["V_matrix"], atol=1e-12, rtol=0)


def test_h2o_eris_processed_order(oracle_mod, golden_h2o):
    atoms, centers = [str(a) for a in golden_h2o["atoms"]], golden_h2o["centers"]
    sh = _shells(oracle_mod, atoms, centers)
    q = oracle_mod.quartet_list(len(sh))
    assert (q == golden_h2o["eri_quads"]).all()
    vals, off = oracle_mod.eri_quartets(sh, q)
    order = oracle_mod.process_order(sh, q)
    assert (q[order] == golden_h2o["processed_eri_quads"]).all()
    pv = np.concatenate([vals[off[i]:off[i + 1]] for i in order])
    assert pv.shape == golden_h2o["processed_eri_values"].shape == (544,)
    np.testing.assert_allclose(pv, golden_h2o["processed_eri_values"], atol=1e-13, rtol=0)


def test_h2o_energy_reference_loop(oracle_mod, golden_h2o):
    atoms, centers = [str(a) for a in golden_h2o["atoms"]], golden_h2o["centers"]
    sh = _shells(oracle_mod, atoms, centers)
    S, T, V = oracle_mod.one_electron(sh, atoms, centers)
    q = oracle_mod.quartet_list(len(sh))
    vals, off = oracle_mod.eri_quartets(sh, q)
    na, nb = oracle_mod.electron_counts(atoms)
    jk = lambda P, Pa, Pb: oracle_mod.fill_matrices(sh, q, vals, off, P, Pa, Pb)
    r = oracle_mod.scf_uhf(T + V, S, jk, na, nb, geometry.nuclear_repulsion(atoms, centers), etol=1e-12, ptol=1e-9)
    assert r["iterations"] == golden_h2o["iterations"]
    assert abs(r["energy"] - golden_h2o["energy"]) < 1e-10
    assert abs(r["energy"] - (-74.96302777726069)) < 1e-10
    np.testing.assert_allclose(r["J"], golden_h2o["J_matrix"], atol=1e-12)
    np.testing.assert_allclose(r["K_a"], golden_h2o["K_a"], atol=1e-12)
    # reference thresholds give the reference's own energy too
    r2 = oracle_mod.scf_uhf(T + V, S, jk, na, nb, geometry.nuclear_repulsion(atoms, centers))
    assert abs(r2["energy"] - golden_h2o["energy_refthr"]) < 1e-10


def test_h2o_dense_tensor_matches_digestion(oracle_mod, golden_h2o):
    atoms, centers = [str(a) for a in golden_h2o["atoms"]], golden_h2o["centers"]
    sh = _shells(oracle_mod, atoms, centers)
    eri = oracle_mod.full_eri_tensor(sh)
    # 8-fold symmetry and Schwarz inequality (main.py:978-987 checks)
    for perm in [(1, 0, 2, 3), (0, 1, 3, 2), (2, 3, 0, 1)]:
        np.testing.assert_allclose(eri, eri.transpose(perm), atol=1e-14)
    N = eri.shape[0]
    diag = np.einsum("ijij->ij", eri)
    assert (diag >= 0).all()
    assert (eri ** 2 <= diag[:, :, None, None] * diag[None, None, :, :] + 1e-14).all()
    Pa, Pb = golden_h2o["P_a"], golden_h2o["P_b"]
    J = np.einsum("ijkl,kl->ij", eri, Pa + Pb)
    K = np.einsum("ikjl,kl->ij", eri, Pa)
    np.testing.assert_allclose(J, golden_h2o["J_matrix"], atol=1e-12)
    np.testing.assert_allclose(K, golden_h2o["K_a"], atol=1e-12)


def test_c10h22_one_electron_and_eri_sample(oracle_mod, golden_c10h22):
    g = golden_c10h22
    atoms, centers = [str(a) for a in g["atoms"]], g["centers"]
    sh = _shells(oracle_mod, atoms, centers)
    S, T, V = oracle_mod.one_electron(sh, atoms, centers)
    np.testing.assert_allclose(S, g["overlaps"], atol=1e-13, rtol=0)
    np.testing.assert_allclose(T, g["T_matrix"], atol=1e-12, rtol=0)
    np.testing.assert_allclose(V, g["V_matrix"], atol=1e-11, rtol=0)
    q = g["sample_quads"]
    vals, off = oracle_mod.eri_quartets(sh, q)
    np.testing.assert_array_equal(off, g["sample_offsets"])
    np.testing.assert_allclose(vals, g["sample_values"], atol=1e-13, rtol=0)
    assert g["n_quartets"] == len(oracle_mod.quartet_list(len(sh)))


def test_c10h22_energy_at_golden_density(oracle_mod, golden_c10h22):
    """E = 1/2 sum(P H + P_a F_a + P_b F_b) from oracle J/K at the reference's
    converged density reproduces the reference's energy."""
    g = golden_c10h22
    atoms, centers = [str(a) for a in g["atoms"]], g["centers"]
    sh = _shells(oracle_mod, atoms, centers)
    q = oracle_mod.quartet_list(len(sh))
    Pa = g["P_a"]
    J, Ka, _ = oracle_mod.direct_jk(sh, q, 2 * Pa, Pa, Pa)
    np.testing.assert_allclose(J, g["J_matrix"], atol=1e-11)
    np.testing.assert_allclose(Ka, g["K_a"], atol=1e-11)
    H = g["T_matrix"] + g["V_matrix"]
    F = H + J - Ka
    E = 0.5 * np.sum(2 * Pa * H + 2 * Pa * F) + g["E_NN"]
    assert abs(E - g["energy"]) < 1e-9


def test_h2o64_sample(oracle_mod, golden_h2o64):
    g = golden_h2o64
    atoms, centers = [str(a) for a in g["atoms"]], g["centers"]
    ref_atoms, ref_centers = geometry.water_cluster((4, 4, 4))
    np.testing.assert_array_equal(centers, ref_centers)
    sh = _shells(oracle_mod, atoms, centers)
    q = g["sample_quads"]
    vals, off = oracle_mod.eri_quartets(sh, q)
    np.testing.assert_allclose(vals, g["sample_values"], atol=1e-13, rtol=0)


# ----------------------------------------------------------- vs oracle/_ref
def _ref_or_skip(oracle_mod):
    lib = oracle_mod.ref_lib()
    if lib is None:
        pytest.skip("oracle/_ref not built (needs the reference tree)")
    return lib


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


def test_pair_and_eri_prims_match_reference_kernels(oracle_mod):
    ref = _ref_or_skip(oracle_mod)
    lib = oracle_mod.lib()
    rng = np.random.default_rng(5)
    for trial in range(20):
        la, lb = rng.integers(0, 3, size=2)
        pa = np.array(oracle_mod.combinations(int(la)), dtype=np.int32)
        pb = np.array(oracle_mod.combinations(int(lb)), dtype=np.int32)
        ea = np.repeat(rng.uniform(0.1, 30, size=2), 1)
        eb = rng.uniform(0.1, 30, size=2)
        exp_a = np.tile(ea, len(pa)); pow_a = np.repeat(pa, ea.size, axis=0).reshape(-1, 3).copy()
        exp_b = np.tile(eb, len(pb)); pow_b = np.repeat(pb, eb.size, axis=0).reshape(-1, 3).copy()
        ca, cb = rng.normal(size=3), rng.normal(size=3) * 1.5
        Z = np.array([1, 8, 6], dtype=np.int32)
        xyz = rng.normal(size=(3, 3)) * 2
        na, nb = exp_a.size, exp_b.size
        K = na * nb
        outs = []
        for fn in ("ref", "orc"):
            V, Ex, Ey, Ez = np.zeros(K), np.zeros(7 * K), np.zeros(7 * K), np.zeros(7 * K)
            p, P = np.zeros(K), np.zeros(3 * K)
            nx, ny, nz = (np.zeros(K, dtype=np.int32) for _ in range(3))
            args = [_p(exp_a), _p(exp_b), _p(ca), _p(cb), _p(pow_a), _p(pow_b), _p(Z), _p(xyz)]
            if fn == "ref":
                ref.ref_run_nuclear_kernel(ctypes.c_longlong(K), *args, ctypes.c_int(3), ctypes.c_int(na),
                                           ctypes.c_int(nb), _p(V), _p(Ex), _p(Ey), _p(Ez), _p(p), _p(P),
                                           _p(nx), _p(ny), _p(nz))
            else:
                lib.orc_pair_prims(ctypes.c_int(na), _p(exp_a), _p(pow_a), _p(ca), ctypes.c_int(nb), _p(exp_b),
                                   _p(pow_b), _p(cb), ctypes.c_int(3), _p(Z), _p(xyz), _p(V), _p(Ex), _p(Ey),
                                   _p(Ez), _p(p), _p(P), _p(nx), _p(ny), _p(nz))
            outs.append((V, Ex, Ey, Ez, p, P, nx, ny, nz))
        for a, b in zip(*outs):
            np.testing.assert_allclose(a, b, atol=1e-13, rtol=1e-13)
        # primitive ERIs of this pair with itself
        V, Ex, Ey, Ez, p, P, nx, ny, nz = outs[0]
        o_ref, o_orc = np.zeros(K * K), np.zeros(K * K)
        pair = [_p(p), _p(P), _p(Ex), _p(Ey), _p(Ez), _p(nx), _p(ny), _p(nz)]
        ref.ref_run_eri_kernel(ctypes.c_longlong(K * K), ctypes.c_int(K), *pair, ctypes.c_int(K), *pair, _p(o_ref))
        lib.orc_eri_prims(ctypes.c_int(K), *pair, ctypes.c_int(K), *pair, _p(o_orc))
        np.testing.assert_allclose(o_orc, o_ref, atol=1e-13, rtol=1e-12)


# ------------------------------------------------------- d shells, contractions
def _gc_path():
    import os

    from conftest import GOLDEN

    return os.path.join(GOLDEN, "dz_gc_test.json")


def test_br2_eris_and_energy(oracle_mod):
    """Br2 / STO-3G (3d shells on both atoms): every processed ERI, the
    spherical transform and the reference loop's energy in its spherical basis."""
    from conftest import load_golden

    g = load_golden("br2.npz")
    atoms, centers = [str(a) for a in g["atoms"]], g["centers"]
    sh = _shells(oracle_mod, atoms, centers)
    q = oracle_mod.quartet_list(len(sh))
    assert (q == g["eri_quads"]).all()
    vals, off = oracle_mod.eri_quartets(sh, q)
    order = oracle_mod.process_order(sh, q)
    assert (q[order] == g["processed_eri_quads"]).all()
    pv = np.concatenate([vals[off[i]:off[i + 1]] for i in order])
    np.testing.assert_allclose(pv, g["processed_eri_values"], atol=1e-13, rtol=0)
    A = oracle_mod.spherical_transform(sh)
    np.testing.assert_allclose(A, g["A"], atol=1e-15, rtol=0)
    S, T, V = oracle_mod.one_electron(sh, atoms, centers)
    for M, key in ((S, "overlaps"), (T, "T_matrix"), (V, "V_matrix")):
        assert np.abs(A @ M @ A.T - g[key]).max() < 1e-12 * max(1.0, np.abs(g[key]).max()), key
    na, nb = oracle_mod.electron_counts(atoms)
    jk = lambda P, Pa, Pb: oracle_mod.fill_matrices(sh, q, vals, off, P, Pa, Pb)
    r = oracle_mod.scf_uhf(T + V, S, jk, na, nb, geometry.nuclear_repulsion(atoms, centers), etol=1e-11,
                           ptol=1e-8, A=A)
    assert abs(r["energy"] - g["energy"]) < 1e-8


@pytest.mark.parametrize("case", ["gc", "gcf"])
def test_general_contraction_energy(oracle_mod, case):
    """H2O with the generally contracted, d-polarised test basis (gcf: with an
    f shell on O and a d shell on H as well): the oracle's contraction-matrix
    integrals reproduce the reference's spherical S/T/V and its SCF energy."""
    import os

    from conftest import GOLDEN, load_golden

    g = load_golden("h2o_gc.npz" if case == "gc" else "h2o_gcf.npz")
    path = _gc_path() if case == "gc" else os.path.join(GOLDEN, "dzf_gc_test.json")
    atoms, centers = [str(a) for a in g["atoms"]], g["centers"]
    sh = oracle_mod.build_shells(oracle_mod.load_basis(path), atoms, centers)
    A = oracle_mod.spherical_transform(sh)
    np.testing.assert_allclose(A, g["A"], atol=1e-15, rtol=0)
    S, T, V = oracle_mod.one_electron(sh, atoms, centers)
    for M, key in ((S, "overlaps"), (T, "T_matrix"), (V, "V_matrix")):
        assert np.abs(A @ M @ A.T - g[key]).max() < 1e-12 * max(1.0, np.abs(g[key]).max()), key
    q = oracle_mod.quartet_list(len(sh))
    na, nb = oracle_mod.electron_counts(atoms)
    jk = lambda P, Pa, Pb: oracle_mod.direct_jk(sh, q, P, Pa, Pb)
    r = oracle_mod.scf_uhf(T + V, S, jk, na, nb, geometry.nuclear_repulsion(atoms, centers), etol=1e-11,
                           ptol=1e-8, A=A)
    assert abs(r["energy"] - g["energy"]) < 1e-8


def test_segments_and_spherical_transform_host():
    """Host side of the d path: segments cover every AO row of a generally
    contracted shell once, and basis.spherical_transform is the reference's A."""
    import json

    from conftest import load_golden
    from dft_b200 import basis

    g = load_golden("h2o_gc.npz")
    with open(_gc_path()) as fh:
        data = json.load(fh)
    sh = basis.build_shells(data, [str(a) for a in g["atoms"]], g["centers"])
    segs = basis.segments(sh)
    rows = np.concatenate([np.arange(s["ao_start"], s["ao_start"] + s["n_ao"]) for s in segs])
    assert np.array_equal(np.sort(rows), np.arange(sh[-1]["ao_stop"]))
    assert len(segs) > len(sh)
    np.testing.assert_allclose(basis.spherical_transform(sh), g["A"], atol=1e-15, rtol=0)
    b = load_golden("br2.npz")
    shb = basis.build_shells(basis.load_basis(), [str(a) for a in b["atoms"]], b["centers"])
    np.testing.assert_allclose(basis.spherical_transform(shb), b["A"], atol=1e-15, rtol=0)
    import os

    from conftest import GOLDEN

    f = load_golden("h2o_gcf.npz")
    with open(os.path.join(GOLDEN, "dzf_gc_test.json")) as fh:
        shf = basis.build_shells(json.load(fh), [str(a) for a in f["atoms"]], f["centers"])
    assert max(s["angular_momentum"] for s in shf) == 3
    np.testing.assert_allclose(basis.spherical_transform(shf), f["A"], atol=1e-15, rtol=0)
