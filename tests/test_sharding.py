"""Sharded Fock build, host side (CPU, gloo, world size 2): the row split
gives every candidate quartet to exactly one rank, and the oracle's J/K over
each rank's quartets, summed by an all-reduce, equals the full J/K."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from dft_b200 import basis, geometry
from dft_b200.engine import QCLASS_PAIRS, candidate_offsets, shard_row_offsets


def test_shard_offsets_partition_every_candidate():
    rng = np.random.default_rng(0)
    for world in (1, 2, 3, 7):
        cnt = rng.integers(0, 50, size=300)
        cnt[rng.integers(0, 300, size=40)] = 0
        off = np.concatenate([[0], np.cumsum(cnt)])
        owner = np.full(off[-1], -1)
        sizes = []
        for r in range(world):
            o = shard_row_offsets(off, r, world)
            mine = np.diff(o)
            assert np.all((mine == 0) | (mine == cnt))
            rows = np.nonzero(mine)[0]
            for row in rows:
                seg = slice(off[row], off[row + 1])
                assert np.all(owner[seg] == -1)
                owner[seg] = r
            sizes.append(int(o[-1]))
        assert np.all(owner >= 0)
        assert sum(sizes) == off[-1]
        assert max(sizes) <= off[-1] / world + cnt.max() + 1  # balanced up to one row


def _quartets(oracle_mod, shells, offsets_fn):
    """Unique candidate quartets (reference shell indices) of every class,
    from Schwarz factors of the oracle's diagonal integrals, restricted by
    offsets_fn(class, row_off)."""
    l = np.array([s["angular_momentum"] for s in shells])
    ii, jj = np.tril_indices(len(shells))
    diag = np.stack([ii, jj, ii, jj], axis=1).astype(np.int32)
    vals, off = oracle_mod.eri_quartets(shells, diag)
    q = np.array([np.sqrt(np.abs(vals[off[t]:off[t + 1]]).max()) for t in range(len(ii))])
    pc = l[ii] + l[jj]
    order = [np.nonzero(pc == c)[0][np.argsort(-q[pc == c], kind="stable")] for c in range(3)]
    quads = []
    for c, (X, Y) in enumerate(QCLASS_PAIRS):
        qx, qy = q[order[X]], q[order[Y]]
        ro = offsets_fn(c, candidate_offsets(qx, qy, X == Y, 1e-12))
        for r in range(qx.size):
            for k in range(ro[r + 1] - ro[r]):
                px, py = order[X][r], order[Y][k]
                quads.append((ii[px], jj[px], ii[py], jj[py]))
    return np.array(quads, dtype=np.int32).reshape(-1, 4)


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import oracle as orc

        atoms, c = geometry.water_cluster((1, 1, 2), seed=2)
        shells = orc.build_shells(orc.load_basis(basis.STO3G_PATH), atoms, c)
        N = shells[-1]["ao_stop"]
        rng = np.random.default_rng(4)
        A = rng.normal(size=(N, N))
        P = (A + A.T) * 0.2
        quads = _quartets(orc, shells, lambda cls, off: shard_row_offsets(off, rank, world))
        J, Ka, _ = orc.direct_jk(shells, quads, P, P / 2, P / 2)
        buf = torch.as_tensor(np.stack([J, Ka]))
        dist.all_reduce(buf)
        full = _quartets(orc, shells, lambda cls, off: off)
        Jf, Kf, _ = orc.direct_jk(shells, full, P, P / 2, P / 2)
        out[rank] = float(max(np.abs(buf[0].numpy() - Jf).max(), np.abs(buf[1].numpy() - Kf).max()))
        out[world + rank] = len(quads)
        out[2 * world + rank] = len(full)
    finally:
        dist.destroy_process_group()


def test_sharded_jk_gloo_two_ranks(oracle_mod):
    world = 2
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    out = mp.get_context("spawn").Manager().list([0.0] * (3 * world))
    mp.start_processes(_worker, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
    assert max(out[:world]) < 1e-12
    assert sum(out[world:2 * world]) == out[2 * world]  # every quartet exactly once
    assert min(out[world:2 * world]) > 0
