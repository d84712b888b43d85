"""One system's Fock build split over the ranks of a process group.

Every rank holds the whole system (shells, pairs, densities: a few MB) and
builds its share of each quartet class's candidate space: contiguous bra-row
ranges holding equal numbers of candidates (``engine.shard_row_offsets``),
so the class kernels, the selection pass and the screening are unchanged.
The partial Y and Z accumulators are symmetrised locally (J = Y + Y^T is
linear), and one all-reduce of the stacked J and K (3 N^2 FP64, 4.8 MB for
N = 448) over NCCL sums them.  The batch path shards by molecule instead and
needs no exchange.
"""
from __future__ import annotations

from typing import Optional

import torch


class ShardedFock:
    def __init__(self, engine, group=None):
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.engine = engine
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.queue = engine.shard_queue(self.rank, self.world)

    def jk(self, D: torch.Tensor, D_a: Optional[torch.Tensor] = None, D_b: Optional[torch.Tensor] = None,
           uhf: bool = False, **kw):
        """J, K_a (, K_b) of the whole system: this rank's partial build,
        then one all-reduce (sum) over the group."""
        J, Ka, Kb = self.engine.jk(D, D_a, D_b, uhf=uhf, queue=self.queue, **kw)
        parts = [J, Ka] + ([Kb] if uhf else [])
        buf = torch.stack(parts)
        self.dist.all_reduce(buf, group=self.group)
        J, Ka = buf[0], buf[1]
        return J, Ka, (buf[2] if uhf else Ka)
