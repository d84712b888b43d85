"""Pin the oracle's analytic gradient (CPU only).

The reference has no gradients, so the oracle gradient (explicit derivative
integrals on all four centres, oracle/oracle.c orc_gradient) is pinned
against central finite differences of the oracle's own SCF energy, which is
itself pinned to the reference's energies by test_oracle_golden.py."""
import numpy as np

from dft_b200 import basis, geometry

H = 1e-4


def test_h2o_oracle_gradient_vs_fd(oracle_mod):
    atoms, c = geometry.water()
    c = c + np.array([[0.02, -0.03, 0.01], [0.0, 0.05, -0.02], [-0.04, 0.0, 0.03]])
    E, g = oracle_mod.scf_energy_gradient(basis.STO3G_PATH, atoms, c)
    fd = np.zeros_like(c)
    for a in range(3):
        for x in range(3):
            cp, cm = c.copy(), c.copy()
            cp[a, x] += H
            cm[a, x] -= H
            ep = oracle_mod.scf_energy_gradient(basis.STO3G_PATH, atoms, cp, with_gradient=False)[0]
            em = oracle_mod.scf_energy_gradient(basis.STO3G_PATH, atoms, cm, with_gradient=False)[0]
            fd[a, x] = (ep - em) / (2 * H)
    assert np.abs(g - fd).max() < 1e-7, np.abs(g - fd).max()


def test_water_dimer_oracle_gradient_invariances(oracle_mod):
    """Every centre's derivative is formed explicitly, so translational
    (sum_A g_A = 0) and rotational (sum_A R_A x g_A = 0) invariance are
    independent checks of the derivative integrals."""
    atoms, c = geometry.water_cluster((1, 1, 2), seed=3)
    E, g = oracle_mod.scf_energy_gradient(basis.STO3G_PATH, atoms, c)
    assert np.abs(g.sum(axis=0)).max() < 1e-10
    torque = np.cross(c, g).sum(axis=0)
    assert np.abs(torque).max() < 1e-8
    # one coordinate against central differences
    a, x = 4, 1
    cp, cm = c.copy(), c.copy()
    cp[a, x] += H
    cm[a, x] -= H
    ep = oracle_mod.scf_energy_gradient(basis.STO3G_PATH, atoms, cp, with_gradient=False)[0]
    em = oracle_mod.scf_energy_gradient(basis.STO3G_PATH, atoms, cm, with_gradient=False)[0]
    assert abs((ep - em) / (2 * H) - g[a, x]) < 1e-7


def test_nuclear_repulsion_gradient_matches_product(oracle_mod):
    atoms, c = geometry.alkane(10)
    np.testing.assert_allclose(geometry.nuclear_repulsion_gradient(atoms, c),
                               oracle_mod.nuclear_repulsion_gradient(atoms, c), atol=1e-12)
    assert abs(geometry.nuclear_repulsion(atoms, c) - oracle_mod.nuclear_repulsion(atoms, c)) < 1e-9
