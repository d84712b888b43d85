"""Edge cases (needs a GPU): molecules with s shells only (every p class
empty), a single atom, a batch mixing them, everything screened out, and the
argument checks of the C-ABI."""
import numpy as np
import pytest
import torch

from dft_b200 import _lib, basis, geometry
from dft_b200.batch import BatchEngine, scf_rhf_batch
from dft_b200.engine import IntegralEngine
from dft_b200.scf import scf_rhf

pytestmark = pytest.mark.gpu

H2 = (["1", "1"], np.array([[0.0, 0.0, 0.0], [0.0, 0.0, 1.4]]))
HE = (["2"], np.zeros((1, 3)))
LIH = (["3", "1"], np.array([[0.0, 0.0, 0.0], [0.0, 0.0, 3.015]]))


def _oracle_jk(oracle_mod, atoms, c, P):
    osh = oracle_mod.build_shells(oracle_mod.load_basis(basis.STO3G_PATH), atoms, c)
    q = oracle_mod.quartet_list(len(osh))
    return oracle_mod.direct_jk(osh, q, P, P / 2, P / 2), osh


@pytest.mark.parametrize("mol", [H2, HE, LIH])
def test_small_molecules_jk_energy_gradient(oracle_mod, mol):
    atoms, c = mol
    eng = IntegralEngine(basis.build_shells(basis.load_basis(), atoms, c), tau_schwarz=0.0)
    if atoms == ["1", "1"] or atoms == ["2"]:
        assert sum(eng.quartet_totals()[1:]) == 0  # s shells only: every p class empty
    rng = np.random.default_rng(1)
    A = rng.normal(size=(eng.n_ao, eng.n_ao))
    P = 0.2 * (A + A.T)
    J, K, _ = eng.jk(torch.as_tensor(P, device="cuda"), tau=0.0)
    (J0, K0, _), osh = _oracle_jk(oracle_mod, atoms, c, P)
    assert np.abs(J.cpu().numpy() - J0).max() < 1e-12
    assert np.abs(K.cpu().numpy() - K0).max() < 1e-12
    S, T, V = eng.one_electron(atoms, c)
    n_el = basis.n_electrons(atoms)
    r = scf_rhf(eng, T + V, S, n_el // 2, geometry.nuclear_repulsion(atoms, c) if len(atoms) > 1 else 0.0,
                etol=1e-12, dtol=1e-10)
    assert r.converged
    E_o, g_o = oracle_mod.scf_energy_gradient(basis.STO3G_PATH, atoms, c, with_gradient=len(atoms) > 1)
    assert abs(r.energy - E_o) < 1e-8
    if len(atoms) > 1:
        Cc = r.C_a[:, : n_el // 2]
        D = 2 * Cc @ Cc.T
        W = 2 * (Cc * r.eps_a[: n_el // 2]) @ Cc.T
        Dh = (0.5 * D).contiguous()
        g = eng.gradient(atoms, c, D, Dh, Dh, W, tau=0.0) + geometry.nuclear_repulsion_gradient(atoms, c)
        assert np.abs(g - g_o).max() < 1e-7  # the two SCFs converge to 1e-10 in density


def test_everything_screened_out():
    atoms, c = geometry.water()
    eng = IntegralEngine(basis.build_shells(basis.load_basis(), atoms, c))
    D = torch.eye(eng.n_ao, dtype=torch.float64, device="cuda")
    J, K, _ = eng.jk(D, tau=1e30)
    assert J.abs().max() == 0 and K.abs().max() == 0
    J, K, _ = eng.jk(torch.zeros_like(D), tau=0.0)
    assert J.abs().max() == 0 and K.abs().max() == 0


def test_batch_of_tiny_molecules_matches_single_solves():
    mols = [H2, HE, LIH, geometry.water(), H2]
    eng = BatchEngine(mols)
    res = scf_rhf_batch(eng)
    assert res.converged.all()
    for m, (atoms, c) in enumerate(mols):
        e1 = IntegralEngine(basis.build_shells(basis.load_basis(), atoms, c))
        S, T, V = e1.one_electron(atoms, c)
        enn = geometry.nuclear_repulsion(atoms, c) if len(atoms) > 1 else 0.0
        r = scf_rhf(e1, T + V, S, basis.n_electrons(atoms) // 2, enn)
        assert abs(res.energy[m] - r.energy) < 1e-8


def test_cabi_rejects_bad_inputs():
    atoms, c = geometry.water()
    eng = IntegralEngine(basis.build_shells(basis.load_basis(), atoms, c))
    D = torch.eye(eng.n_ao, dtype=torch.float64, device="cuda")
    with pytest.raises(_lib.DftkError):
        eng.jk(D, tau=-1.0)  # negative threshold
    with pytest.raises(_lib.DftkError):
        eng.jk(D, mixed=True, tau=1e-6, tau_fp32=1e-8)  # FP32 threshold below the FP64 one
    with pytest.raises(_lib.DftkError):
        eng.jk(torch.eye(3, dtype=torch.float64, device="cuda"))  # wrong shape
    with pytest.raises(_lib.DftkError):
        BatchEngine([])
