"""Sharded queues on one GPU (needs a GPU): the ranks' partial J/K, built one
after another, sum to the full build."""
import numpy as np
import pytest
import torch

from dft_b200 import basis, geometry
from dft_b200.engine import IntegralEngine

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("world", [2, 3])
def test_shard_partials_sum_to_full(world):
    atoms, c = geometry.water_cluster((2, 2, 2), seed=6)
    eng = IntegralEngine(basis.build_shells(basis.load_basis(), atoms, c))
    g = torch.Generator(device="cpu").manual_seed(2)
    A = torch.randn(eng.n_ao, eng.n_ao, dtype=torch.float64, generator=g).cuda() * 0.2
    D = A + A.T
    J, K, _ = eng.jk(D)
    Js, Ks = torch.zeros_like(J), torch.zeros_like(K)
    totals = np.zeros(6, dtype=np.int64)
    for r in range(world):
        q = eng.shard_queue(r, world)
        totals += np.array([q.total[c] for c in range(6)])
        Jr, Kr, _ = eng.jk(D, queue=q)
        Js += Jr
        Ks += Kr
    assert list(totals) == eng.quartet_totals()
    assert (Js - J).abs().max() < 1e-12 and (Ks - K).abs().max() < 1e-12
