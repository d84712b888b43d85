"""SCF energies through the CUDA J/K build (needs a GPU)."""
import numpy as np
import pytest
import torch

from dft_b200 import basis, geometry, shelled
from dft_b200.engine import IntegralEngine
from dft_b200.scf import scf_reference, scf_rhf

pytestmark = pytest.mark.gpu


def _setup(atoms, centers, tau_schwarz=1e-12):
    sh = basis.build_shells(basis.load_basis(), atoms, centers)
    eng = IntegralEngine(sh, tau_schwarz=tau_schwarz)
    S, T, V = eng.one_electron(atoms, centers)
    return eng, S, T + V, geometry.nuclear_repulsion(atoms, centers)


def test_h2o_reference_loop_energy(golden_h2o):
    g = golden_h2o
    atoms, centers = [str(a) for a in g["atoms"]], g["centers"]
    eng, S, H, enn = _setup(atoms, centers, tau_schwarz=0.0)
    r = scf_reference(eng, H, S, 5, 5, enn, etol=1e-12, ptol=1e-9)
    assert abs(r.energy - g["energy"]) < 1e-8
    assert abs(r.iterations - int(g["iterations"])) <= 2
    r2 = scf_reference(eng, H, S, 5, 5, enn)
    assert abs(r2.energy - g["energy_refthr"]) < 1e-8


def test_h2o_scf_entry_point(golden_h2o):
    g = golden_h2o
    r = shelled.scf([str(a) for a in g["atoms"]], g["centers"], method="rhf")
    assert r.converged and abs(r.energy - g["energy"]) < 1e-8


def test_c10h22_rhf_energy(golden_c10h22):
    g = golden_c10h22
    atoms, centers = [str(a) for a in g["atoms"]], g["centers"]
    eng, S, H, enn = _setup(atoms, centers)
    r = scf_rhf(eng, H, S, 41, enn)
    assert r.converged
    assert abs(r.energy - g["energy"]) < 1e-8


def test_mixed_precision_energy_water16():
    atoms, centers = geometry.water_cluster((2, 2, 4))
    eng, S, H, enn = _setup(atoms, centers)
    r64 = scf_rhf(eng, H, S, 5 * 16, enn, mixed=False)
    rmx = scf_rhf(eng, H, S, 5 * 16, enn, mixed=True, count_quartets=True)
    assert r64.converged and rmx.converged
    assert abs(rmx.energy - r64.energy) < 1e-6
    # the energy of the last mixed incremental build itself, before the final FP64 rebuild
    assert abs(rmx.energy_last_build - r64.energy) < 1e-6
    assert sum(rmx.counts[6:12]) > 0


def test_mixed_precision_energy_water64():
    """Config-size check of the mixed form: (H2O)_64, budget-derived tau_fp32,
    against the FP64 incremental SCF: the final energy and the energy of the
    last mixed incremental build within 1 uEh, with most quartets in FP32."""
    from dft_b200.scf import fp32_threshold

    atoms, centers = geometry.water_cluster((4, 4, 4))
    eng, S, H, enn = _setup(atoms, centers)
    tau32 = fp32_threshold(sum(eng.quartet_totals()))
    assert 1e-6 <= tau32 <= 1e-4
    r64 = scf_rhf(eng, H, S, 5 * 64, enn, mixed=False)
    rmx = scf_rhf(eng, H, S, 5 * 64, enn, mixed=True, count_quartets=True)
    assert r64.converged and rmx.converged
    assert abs(rmx.energy - r64.energy) < 1e-6
    assert abs(rmx.energy_last_build - r64.energy) < 1e-6
    # the incremental builds put over 1e8 quartets (about one full build's worth) through FP32
    assert sum(rmx.counts[6:12]) > 1e8
