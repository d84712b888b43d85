"""Orbital densities on a grid on the GPU against the reference's evaluation
script (H2O fixture) and the oracle (larger molecules, open shells, chunking)."""
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN, load_golden

pytestmark = pytest.mark.gpu


def _close(a, b):
    np.testing.assert_allclose(a, b, rtol=1e-6, atol=1e-12 * float(np.abs(b).max()))


def _ckpt():
    from dft_b200 import grid

    return grid.load_eval_checkpoint(os.path.join(GOLDEN, "h2o_eval_checkpoint.npz"))


def test_grid_h2o_matches_reference_script():
    from dft_b200 import grid

    g = load_golden("grid_h2o.npz")
    og = grid.OrbitalGrid(_ckpt())
    total, phase = og.evaluate(g["grid"], chunk_size=500)  # the fixture's chunking: 8 chunks, the last partial
    _close(total, g["total_density"])
    _close(phase, g["phase_density"])
    # one chunk: the GEMM may sum in another order, so equal to rounding
    t2, p2 = og.evaluate(g["grid"], chunk_size=10 ** 6)
    _close(t2, total)
    _close(p2, phase)


def test_grid_d_shells_general_contractions_match_reference_script():
    """The reference's evaluation script on the checkpoint its SCF wrote for
    H2O with the generally contracted, d-polarised test basis: d shells,
    contraction matrices and the spherical transform A in the checkpoint."""
    from dft_b200 import grid

    g = load_golden("grid_h2o_gc.npz")
    ck = grid.load_eval_checkpoint(os.path.join(GOLDEN, "h2o_gc_eval_checkpoint.npz"))
    assert max(s["angular_momentum"] for s in ck["shells"]) == 2
    assert ck["A"].shape[0] < ck["A"].shape[1]
    total, phase = grid.OrbitalGrid(ck).evaluate(g["grid"], chunk_size=500)
    _close(total, g["total_density"])
    _close(phase, g["phase_density"])


def test_grid_open_shell_c10h22_against_oracle(oracle_mod):
    """A 72-AO molecule with distinct alpha/beta coefficients and N_a != N_b."""
    from dft_b200 import basis, geometry, grid

    atoms, centers = geometry.alkane(10)
    shells = basis.build_shells(basis.load_basis(), atoms, centers)
    n = int(shells[-1]["ao_stop"])
    rng = np.random.default_rng(11)
    Ca = np.linalg.qr(rng.standard_normal((n, n)))[0]
    Cb = np.linalg.qr(rng.standard_normal((n, n)))[0]
    ck = {"centers": np.asarray(centers), "N_a": np.float64(41), "N_b": np.float64(40), "C_a": Ca, "C_b": Cb,
          "total_ao": np.int64(n), "shells": shells, "A": np.eye(n)}
    pts = rng.uniform(-3, 3, size=(20011, 3)).astype(np.float32) + np.asarray(centers).mean(axis=0).astype(np.float32)
    total, phase = grid.OrbitalGrid(ck).evaluate(pts, chunk_size=4096)
    t_ref, p_ref = oracle_mod.grid_densities(ck, pts)
    _close(total, t_ref)
    _close(phase, p_ref)
    assert not phase[41:].any()


def test_grid_device_chunk_and_empty():
    from dft_b200 import grid

    og = grid.OrbitalGrid(_ckpt())
    t, p = og.evaluate(np.zeros((0, 3), dtype=np.float32))
    assert t.shape == (5, 0) and p.shape == (5, 0)
    pts = torch.tensor([[0.0, 0.0, 0.2217]], dtype=torch.float32, device="cuda")  # the oxygen nucleus
    tot = torch.full((5, 1), -1.0, dtype=torch.float32, device="cuda")
    ph = torch.zeros((5, 1), dtype=torch.float32, device="cuda")
    og.chunk(pts, tot, ph)
    assert (tot >= 0).all() and torch.isfinite(ph).all()


def test_grid_doublet_without_beta_electrons(oracle_mod):
    """One alpha and no beta electron (an H atom's doublet): total = psi_a^2
    in row 0, phase row 0 only."""
    from dft_b200 import basis, grid

    atoms, centers = ["1"], np.zeros((1, 3))
    shells = basis.build_shells(basis.load_basis(), atoms, centers)
    ck = {"centers": centers, "N_a": np.float64(1), "N_b": np.float64(0), "C_a": np.ones((1, 1)),
          "C_b": np.ones((1, 1)), "total_ao": np.int64(1), "shells": shells, "A": np.eye(1)}
    pts = np.random.default_rng(5).uniform(-3, 3, size=(999, 3)).astype(np.float32)
    total, phase = grid.OrbitalGrid(ck).evaluate(pts, chunk_size=256)
    t_ref, p_ref = oracle_mod.grid_densities(ck, pts)
    _close(total, t_ref)
    _close(phase, p_ref)
    np.testing.assert_allclose(total[0], phase[0].astype(np.float64) ** 2, rtol=1e-6)
