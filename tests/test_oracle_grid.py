"""Orbital densities on a grid (CPU): the oracle restatement against the
reference's evaluation script run on the reference's own H2O checkpoint
(tests/golden/make_golden.py grid), the grid construction, the checkpoint
format, and the C-ABI argument checks (no GPU needed)."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, load_golden


def _ckpt():
    from dft_b200 import grid

    path = os.path.join(GOLDEN, "h2o_eval_checkpoint.npz")
    if not os.path.exists(path):
        pytest.skip("h2o_eval_checkpoint.npz not generated")
    return grid.load_eval_checkpoint(path)


def _close(a, b):
    # near-zero orbital values cancel; compare against each array's scale
    np.testing.assert_allclose(a, b, rtol=1e-6, atol=1e-12 * float(np.abs(b).max()))


def test_oracle_grid_matches_reference_script(oracle_mod):
    g = load_golden("grid_h2o.npz")
    total, phase = oracle_mod.grid_densities(_ckpt(), g["grid"])
    _close(total, g["total_density"])
    _close(phase, g["phase_density"])
    # closed shell: every row is 2 psi_a^2 of the phase row
    np.testing.assert_allclose(total, 2.0 * phase.astype(np.float64) ** 2, rtol=1e-6,
                               atol=1e-12 * float(total.max()))


def test_oracle_grid_d_shells_matches_reference_script(oracle_mod):
    """The evaluation script's densities for the checkpoint with d shells,
    general contractions and a spherical transform A."""
    from dft_b200 import grid

    g = load_golden("grid_h2o_gc.npz")
    ck = grid.load_eval_checkpoint(os.path.join(GOLDEN, "h2o_gc_eval_checkpoint.npz"))
    total, phase = oracle_mod.grid_densities(ck, g["grid"])
    _close(total, g["total_density"])
    _close(phase, g["phase_density"])


def test_reference_grid_reproduces_script_grid():
    from dft_b200 import grid

    g = load_golden("grid_h2o.npz")
    ck = _ckpt()
    # the fixture's grid: spacing 0.15, x widened by 1 bohr each way
    pts, shape = grid.reference_grid(ck["centers"], spacing=0.15, pad_lo=(1.0, -0.75, 1.0), pad_hi=(1.0, -0.75, 1.0))
    assert pts.dtype == np.float32 and pts.shape == (int(np.prod(shape)), 3)
    np.testing.assert_array_equal(pts, g["grid"])
    # the script's own x bounds on a molecule flat in x give no points
    with pytest.raises(ValueError):
        grid.reference_grid(ck["centers"], spacing=0.15)


def test_checkpoint_round_trip(tmp_path):
    from dft_b200 import grid

    ck = _ckpt()
    path = str(tmp_path / "ck.npz")
    grid.save_eval_checkpoint(path, ck["centers"], ck["N_a"], ck["N_b"], ck["C_a"], ck["C_b"], ck["total_ao"],
                              ck["shells"], ck["A"])
    back = grid.load_eval_checkpoint(path)
    for k in ("centers", "N_a", "N_b", "C_a", "C_b", "total_ao", "A"):
        np.testing.assert_array_equal(back[k], ck[k])
    assert len(back["shells"]) == len(ck["shells"])
    for a, b in zip(back["shells"], ck["shells"]):
        assert a["ao_start"] == b["ao_start"] and a["angular_momentum"] == b["angular_momentum"]
        np.testing.assert_array_equal(a["exponents"], b["exponents"])
    np.savez(str(tmp_path / "bad.npz"), centers=ck["centers"])
    with pytest.raises(KeyError):
        grid.load_eval_checkpoint(str(tmp_path / "bad.npz"))


def test_oracle_grid_open_shell_rows(oracle_mod):
    """N_a != N_b: rows past N_b hold alpha only, phase rows past N_a stay zero."""
    ck = dict(_ckpt())
    rng = np.random.default_rng(3)
    ck["C_b"] = ck["C_a"] + 0.01 * rng.standard_normal(ck["C_a"].shape)
    ck["N_a"], ck["N_b"] = np.float64(5), np.float64(4)
    pts = rng.uniform(-2, 2, size=(257, 3)).astype(np.float32)
    total, phase = oracle_mod.grid_densities(ck, pts)
    assert total.shape == (5, 257)
    ao = oracle_mod.grid_ao(ck["shells"], pts)
    pa = ck["C_a"].astype(np.float32)[:, :5].T.astype(np.float64) @ ao
    np.testing.assert_allclose(total[4], (pa[4] ** 2).astype(np.float32), rtol=1e-6)
    assert not phase[5:].any()


def test_grid_cabi_argument_errors_without_gpu():
    from dft_b200 import _lib

    lib = _lib.load()
    assert lib.dftk_grid_ao(None, 10, None, None, 10, None) == _lib.ERR_ARG
    # ld shorter than the point count, n_a beyond n_mo
    assert lib.dftk_grid_density(3, 1, 1, 100, None, None, 50, None, None, 100, None) == _lib.ERR_ARG
    assert lib.dftk_grid_density(3, 4, 1, 100, None, None, 100, None, None, 100, None) == _lib.ERR_ARG
