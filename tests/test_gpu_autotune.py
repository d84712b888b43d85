"""Autotuned launch shapes (needs a GPU): the tuner picks a shape per class
and the J/K build gives the same matrices with it."""
import pytest
import torch

from dft_b200 import autotune, basis, geometry
from dft_b200.engine import IntegralEngine

pytestmark = pytest.mark.gpu


def test_tuned_shapes_keep_results():
    atoms, c = geometry.water_cluster((2, 2, 2), seed=4)
    eng = IntegralEngine(basis.build_shells(basis.load_basis(), atoms, c))
    g = torch.Generator(device="cpu").manual_seed(3)
    A = torch.randn(eng.n_ao, eng.n_ao, dtype=torch.float64, generator=g).cuda() * 0.2
    D = A + A.T
    before = autotune.get_shapes(autotune.FAMILY_JK)
    J0, K0, _ = eng.jk(D)
    try:
        res = autotune.tune_jk(eng, D, repeats=1)
        assert len(res["shapes"]) == 6
        assert autotune.get_shapes(autotune.FAMILY_JK) == [tuple(s) for s in res["shapes"]]
        assert sum(res["tuned_ms"]) <= sum(res["default_ms"]) * 1.0001
        J1, K1, _ = eng.jk(D)
        assert (J1 - J0).abs().max() < 1e-12 and (K1 - K0).abs().max() < 1e-12
    finally:
        autotune.set_shapes(autotune.FAMILY_JK, before)
