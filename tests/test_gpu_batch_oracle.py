"""Batches of molecules against the CPU oracle (needs a GPU).

A small uneven batch -- H2O, the water dimer, CH4, an s-only H2 and a water
trimer that is switched off -- goes through one BatchEngine.  Each molecule's
packed S/T/V and J/K blocks are compared with the oracle's own per-molecule
restatement of the reference (one_electron, and direct_jk over the full
unique-quartet list, shelled.py:770-877), and the batched SCF energies with
the oracle's UHF loop (shelled.py:1164-1293) on the same molecules.  This
pins the molecule table, the per-row ket bases and the packed matrix offsets
against an independent implementation, not only against the single-molecule
engine in the same library.
"""
import numpy as np
import pytest
import torch

from dft_b200 import basis, geometry
from dft_b200.batch import BatchEngine, scf_rhf_batch

pytestmark = pytest.mark.gpu

# FP64 J/K of small molecules: elements are sums of a few thousand terms
TOL_JK = 1e-11
TOL_1E = 1e-12
TOL_E = 1e-8


def _methane():
    d = 2.05  # bohr, C-H
    s = d / np.sqrt(3.0)
    c = np.array([[0, 0, 0], [s, s, s], [s, -s, -s], [-s, s, -s], [-s, -s, s]], dtype=np.float64)
    return ["6", "1", "1", "1", "1"], c


def _h2():
    return ["1", "1"], np.array([[0.0, 0.0, -0.7], [0.0, 0.0, 0.7]])


def _molecules():
    return [geometry.water(), geometry.water_cluster((1, 1, 2), seed=3), _methane(), _h2(),
            geometry.water_cluster((1, 1, 3), seed=4)]


INACTIVE = 4


def _oracle_shells(oracle, atoms, centers):
    return oracle.build_shells(oracle.load_basis(basis.STO3G_PATH), atoms, centers)


def test_batch_one_electron_and_jk_match_oracle(oracle_mod):
    mols = _molecules()
    eng = BatchEngine(mols, tau_schwarz=0.0)
    S, T, V = eng.one_electron()
    rng = np.random.default_rng(21)
    Dh = []
    for n in eng.mol_nao:
        A = rng.normal(size=(int(n), int(n))) * 0.2
        Dh.append(A + A.T)
    Dp = torch.cat([torch.as_tensor(d, device="cuda").reshape(-1) for d in Dh])
    eng.mol_active[INACTIVE] = 0
    try:
        J, K, _ = eng.jk(Dp, 0.5 * Dp, tau=0.0)
        torch.cuda.synchronize()
    finally:
        eng.mol_active.fill_(1)
    for m, (atoms, c) in enumerate(mols):
        osh = _oracle_shells(oracle_mod, atoms, c)
        S0, T0, V0 = oracle_mod.one_electron(osh, atoms, c)
        for got, want in ((S, S0), (T, T0), (V, V0)):
            assert np.abs(eng.block(got, m).cpu().numpy() - want).max() < TOL_1E, m
        Jm, Km = eng.block(J, m).cpu().numpy(), eng.block(K, m).cpu().numpy()
        if m == INACTIVE:
            assert not Jm.any() and not Km.any()
            continue
        q = oracle_mod.quartet_list(len(osh))
        J0, K0, _ = oracle_mod.direct_jk(osh, q, Dh[m], 0.5 * Dh[m], 0.5 * Dh[m])
        assert np.abs(Jm - J0).max() < TOL_JK, (m, np.abs(Jm - J0).max())
        assert np.abs(Km - K0).max() < TOL_JK, (m, np.abs(Km - K0).max())


def test_batch_scf_energies_match_oracle(oracle_mod):
    mols = _molecules()[:4]
    eng = BatchEngine(mols)
    res = scf_rhf_batch(eng, etol=1e-11, dtol=1e-9)
    assert res.converged.all()
    for m, (atoms, c) in enumerate(mols):
        osh = _oracle_shells(oracle_mod, atoms, c)
        S0, T0, V0 = oracle_mod.one_electron(osh, atoms, c)
        q = oracle_mod.quartet_list(len(osh))
        na, nb = oracle_mod.electron_counts(atoms)
        jk = lambda P, Pa, Pb, osh=osh, q=q: oracle_mod.direct_jk(osh, q, P, Pa, Pb)  # noqa: E731
        r = oracle_mod.scf_uhf(T0 + V0, S0, jk, na, nb, oracle_mod.nuclear_repulsion(atoms, c),
                               etol=1e-11, ptol=1e-8)
        assert abs(res.energy[m] - r["energy"]) < TOL_E, (m, res.energy[m], r["energy"])
