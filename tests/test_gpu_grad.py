"""Analytic nuclear gradients vs central finite differences (needs a GPU).

Bar: 1e-6 Eh/bohr against central differences of the energy at a 1e-4 bohr
step."""
import numpy as np
import pytest
import torch

from dft_b200 import geometry
from dft_b200.gradient import energy_and_gradient, rhf_energy

pytestmark = pytest.mark.gpu

SCF = dict(etol=1e-12, dtol=1e-10)
GRAD_TOL = 1e-6


def _fd(atoms, centers, h=1e-4, idx=None, scf=SCF):
    g = np.zeros_like(centers)
    for a in range(centers.shape[0]):
        for x in range(3):
            if idx is not None and (a, x) not in idx:
                continue
            cp, cm = centers.copy(), centers.copy()
            cp[a, x] += h
            cm[a, x] -= h
            ep, _ = energy_and_gradient(atoms, cp, **scf)
            em, _ = energy_and_gradient(atoms, cm, **scf)
            g[a, x] = (ep - em) / (2 * h)
    return g


def test_h2o_gradient_vs_fd():
    atoms, centers = geometry.water()
    centers = centers + np.array([[0.02, -0.03, 0.01], [0.0, 0.05, -0.02], [-0.04, 0.0, 0.03]])
    E, g = energy_and_gradient(atoms, centers, **SCF)
    fd = _fd(atoms, centers)
    assert np.abs(g - fd).max() < GRAD_TOL, (g, fd)
    # translational invariance of the total gradient
    assert np.abs(g.sum(axis=0)).max() < 1e-9


def test_water_dimer_gradient_vs_fd_subset():
    scf = dict(etol=1e-11, dtol=1e-9)
    atoms, centers = geometry.water_cluster((1, 1, 2), seed=3)
    E, g = energy_and_gradient(atoms, centers, **scf)
    idx = {(0, 0), (1, 2), (3, 1), (5, 0)}
    fd = _fd(atoms, centers, idx=idx, scf=scf)
    for a, x in idx:
        assert abs(g[a, x] - fd[a, x]) < GRAD_TOL, (a, x, g[a, x], fd[a, x])
    assert np.abs(g.sum(axis=0)).max() < 1e-9


def test_autograd_function():
    atoms, centers = geometry.water()
    coords = torch.tensor(centers, dtype=torch.float64, requires_grad=True)
    E = rhf_energy(coords, atoms, **SCF)
    E.backward()
    _, g = energy_and_gradient(atoms, centers, **SCF)
    np.testing.assert_allclose(coords.grad.numpy(), g, atol=1e-10)
    assert abs(E.item() - (-74.96302777726069)) < 1e-8


def _gpu_scf(atoms, centers, mixed=False, **kw):
    from dft_b200 import basis
    from dft_b200.engine import IntegralEngine
    from dft_b200.scf import scf_rhf

    sh = basis.build_shells(basis.load_basis(), atoms, centers)
    eng = IntegralEngine(sh, tau_schwarz=kw.pop("tau_schwarz", 1e-12))
    S, T, V = eng.one_electron(atoms, centers)
    n_occ = basis.n_electrons(atoms, 0) // 2
    res = scf_rhf(eng, T + V, S, n_occ, geometry.nuclear_repulsion(atoms, centers), mixed=mixed, **kw)
    assert res.converged
    C = res.C_a[:, :n_occ]
    D = 2.0 * (C @ C.T)
    W = 2.0 * ((C * res.eps_a[:n_occ]) @ C.T)
    return eng, res, D, W


@pytest.mark.parametrize("cluster", [None, (1, 1, 2), (1, 1, 3)])
def test_gradient_vs_oracle_same_density(oracle_mod, cluster):
    """GPU gradient against the oracle's explicit-derivative gradient at the
    same converged density: only the derivative integrals differ."""
    from dft_b200 import basis

    if cluster is None:
        atoms, centers = geometry.water()
    else:
        atoms, centers = geometry.water_cluster(cluster, seed=7)
    eng, res, D, W = _gpu_scf(atoms, centers, tau_schwarz=0.0, **SCF)
    Dh = (0.5 * D).contiguous()
    g = eng.gradient(atoms, centers, D, Dh, Dh, W, tau=0.0) + geometry.nuclear_repulsion_gradient(atoms, centers)
    osh = oracle_mod.build_shells(oracle_mod.load_basis(basis.STO3G_PATH), atoms, centers)
    Dn, Wn = D.cpu().numpy(), W.cpu().numpy()
    go = oracle_mod.gradient(osh, atoms, centers, Dn, Dn / 2, Dn / 2, Wn)
    assert np.abs(g - go).max() < 1e-10, np.abs(g - go).max()


def test_water16_gradient_fd_subset():
    """(H2O)_16 (2x2x4 lattice): analytic gradient against central differences
    on a few coordinates, and translational invariance."""
    scf = dict(etol=1e-11, dtol=1e-9)
    atoms, centers = geometry.water_cluster((2, 2, 4))
    E, g = energy_and_gradient(atoms, centers, **scf)
    assert np.abs(g.sum(axis=0)).max() < 1e-8
    idx = {(0, 0), (17, 1), (46, 2)}
    fd = _fd(atoms, centers, idx=idx, scf=scf)
    for a, x in idx:
        assert abs(g[a, x] - fd[a, x]) < GRAD_TOL, (a, x, g[a, x], fd[a, x])


def test_c10h22_gradient_fd_subset():
    scf = dict(etol=1e-11, dtol=1e-9)
    atoms, centers = geometry.alkane(10)
    E, g = energy_and_gradient(atoms, centers, **scf)
    assert np.abs(g.sum(axis=0)).max() < 1e-8
    idx = {(0, 0), (4, 1), (12, 2), (30, 0)}
    fd = _fd(atoms, centers, idx=idx, scf=scf)
    for a, x in idx:
        assert abs(g[a, x] - fd[a, x]) < GRAD_TOL, (a, x, g[a, x], fd[a, x])


def test_mixed_scf_gradient_matches_fp64():
    """Gradient at the density of the mixed FP32/FP64 incremental SCF against
    the plain FP64 one, (H2O)_16."""
    atoms, centers = geometry.water_cluster((2, 2, 4))
    _, g64 = energy_and_gradient(atoms, centers, mixed=False)
    _, gmx = energy_and_gradient(atoms, centers, mixed=True)
    assert np.abs(g64 - gmx).max() < GRAD_TOL


def _rand_sym(n, rng, scale):
    A = rng.normal(size=(n, n)) * scale
    return A + A.T


def test_uhf_scan_and_mixed_paths_vs_oracle(oracle_mod):
    """dftk_grad with D_a != D_b (the UHF Gamma), the direct-scan path and
    the mixed path, all at one set of random densities, against the oracle."""
    from dft_b200 import basis
    from dft_b200.engine import IntegralEngine

    atoms, centers = geometry.water_cluster((1, 1, 2), seed=8)
    eng = IntegralEngine(basis.build_shells(basis.load_basis(), atoms, centers), tau_schwarz=0.0)
    rng = np.random.default_rng(12)
    N = eng.n_ao
    Da, Db, W = _rand_sym(N, rng, 0.1), _rand_sym(N, rng, 0.1), _rand_sym(N, rng, 0.05)
    D = Da + Db
    t = lambda M: torch.as_tensor(M, device="cuda")
    gnn = geometry.nuclear_repulsion_gradient(atoms, centers)
    g_list = eng.gradient(atoms, centers, t(D), t(Da), t(Db), t(W), tau=0.0) + gnn
    g_scan = eng.gradient(atoms, centers, t(D), t(Da), t(Db), t(W), tau=0.0, scan=True) + gnn
    g_mix = eng.gradient(atoms, centers, t(D), t(Da), t(Db), t(W), tau=0.0, tau_fp32=1e-6) + gnn
    osh = oracle_mod.build_shells(oracle_mod.load_basis(basis.STO3G_PATH), atoms, centers)
    go = oracle_mod.gradient(osh, atoms, centers, D, Da, Db, W)
    assert np.abs(g_list - go).max() < 1e-10
    assert np.abs(g_scan - go).max() < 1e-10
    assert np.abs(g_mix - go).max() < 1e-7
