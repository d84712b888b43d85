"""Batches of molecules through one shell set (needs a GPU): packed J/K,
one-electron matrices, per-molecule convergence masks, batched SCF and
batched gradients against the single-molecule path."""
import numpy as np
import pytest
import torch

from dft_b200 import basis, geometry
from dft_b200.batch import BatchEngine, rhf_gradient_batch, scf_rhf_batch
from dft_b200.engine import IntegralEngine
from dft_b200.scf import scf_rhf

pytestmark = pytest.mark.gpu


def _molecules():
    mols = [geometry.water(), geometry.alkane(2)]
    mols += geometry.water_cluster_batch(5, 4, seed=11)
    return mols


def _rand_density(n, rng):
    A = rng.normal(size=(n, n)) * 0.3
    return torch.as_tensor(A + A.T, device="cuda")


def test_batch_one_electron_and_jk_match_single():
    mols = _molecules()
    eng = BatchEngine(mols, tau_schwarz=0.0)
    S, T, V = eng.one_electron()
    rng = np.random.default_rng(1)
    Ds = [_rand_density(int(n), rng) for n in eng.mol_nao]
    Dp = torch.cat([d.reshape(-1) for d in Ds])
    J, K, _ = eng.jk(Dp, 0.5 * Dp, tau=0.0)
    for m, (atoms, c) in enumerate(mols):
        single = IntegralEngine(basis.build_shells(basis.load_basis(), atoms, c), tau_schwarz=0.0)
        S1, T1, V1 = single.one_electron(atoms, c)
        for A, B in ((S, S1), (T, T1), (V, V1)):
            assert torch.allclose(eng.block(A, m), B, atol=1e-13, rtol=0)
        J1, K1, _ = single.jk(Ds[m], 0.5 * Ds[m], tau=0.0)
        assert (eng.block(J, m) - J1).abs().max() < 1e-12
        assert (eng.block(K, m) - K1).abs().max() < 1e-12


def test_batch_inactive_molecules_are_skipped():
    mols = _molecules()
    eng = BatchEngine(mols)
    rng = np.random.default_rng(2)
    Dp = torch.cat([_rand_density(int(n), rng).reshape(-1) for n in eng.mol_nao])
    J_all, K_all, _ = eng.jk(Dp, 0.5 * Dp)
    eng.mol_active[1] = 0
    eng.mol_active[4] = 0
    J, K, _ = eng.jk(Dp, 0.5 * Dp)
    eng.mol_active.fill_(1)
    for m in range(eng.n_mol):
        if m in (1, 4):
            assert eng.block(J, m).abs().max() == 0 and eng.block(K, m).abs().max() == 0
        else:
            assert torch.equal(eng.block(J, m), eng.block(J_all, m)) or \
                (eng.block(J, m) - eng.block(J_all, m)).abs().max() < 1e-13


def test_batch_scf_matches_single_solves():
    mols = geometry.water_cluster_batch(12, 6, seed=5) + [geometry.alkane(3)]
    eng = BatchEngine(mols)
    res = scf_rhf_batch(eng)
    assert res.converged.all()
    for m, (atoms, c) in enumerate(mols):
        sh = basis.build_shells(basis.load_basis(), atoms, c)
        single = IntegralEngine(sh)
        S, T, V = single.one_electron(atoms, c)
        r = scf_rhf(single, T + V, S, basis.n_electrons(atoms) // 2, geometry.nuclear_repulsion(atoms, c))
        assert r.converged
        assert abs(res.energy[m] - r.energy) < 1e-8, (m, res.energy[m], r.energy)
        assert abs(int(res.iterations[m]) - r.iterations) <= 3


def test_batch_gradient_matches_single():
    from dft_b200.gradient import energy_and_gradient

    mols = geometry.water_cluster_batch(6, 3, seed=9)
    eng = BatchEngine(mols)
    res = scf_rhf_batch(eng, etol=1e-11, dtol=1e-9)
    assert res.converged.all()
    grads = rhf_gradient_batch(eng, res)
    for m, (atoms, c) in enumerate(mols):
        E, g = energy_and_gradient(atoms, c, etol=1e-11, dtol=1e-9)
        assert abs(E - res.energy[m]) < 1e-8
        assert np.abs(grads[m] - g).max() < 1e-7, np.abs(grads[m] - g).max()


def test_persistent_launch_matches_class_launches():
    """DFTK_JK_PERSIST (one selection launch, one persistent launch per
    precision pulling tiles of every class) gives the class-by-class build's
    J/K: a packed batch (FP64) and one molecule (FP64 and mixed)."""
    mols = _molecules()
    eng = BatchEngine(mols, tau_schwarz=1e-12)
    rng = np.random.default_rng(5)
    Dp = torch.as_tensor(0.05 * rng.normal(size=eng.mat_elems), device=eng.device)
    blocks = [eng.block(Dp, m) for m in range(eng.n_mol)]
    for m, b in enumerate(blocks):  # symmetric per-molecule blocks
        b.copy_(0.5 * (b + b.T))
    J0, K0, _ = eng.jk(2 * Dp, Dp, tau=1e-14)
    J1, K1, _ = eng.jk(2 * Dp, Dp, tau=1e-14, persist=True)
    assert torch.abs(J1 - J0).max().item() < 1e-12 and torch.abs(K1 - K0).max().item() < 1e-12
    atoms, centers = geometry.water_cluster((2, 2, 2))
    e1 = IntegralEngine(basis.build_shells(basis.load_basis(), atoms, centers))
    N = e1.n_ao
    M = rng.normal(size=(N, N))
    D = torch.as_tensor(0.05 * (M + M.T), device=e1.device)
    for mixed in (False, True):
        a = e1.jk(2 * D, D, mixed=mixed, tau=1e-12, tau_fp32=1e-4)
        b = e1.jk(2 * D, D, mixed=mixed, tau=1e-12, tau_fp32=1e-4, persist=True)
        for x, y in zip(a[:2], b[:2]):
            assert torch.abs(x - y).max().item() < 1e-11
