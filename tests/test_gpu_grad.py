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
