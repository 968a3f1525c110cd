"""Multi-GPU data parallelism over independent molecules (one process per GPU).

Molecules are independent, so a batch is sharded across ranks with no
collective on the data path: each rank prepares and executes its shard on its
own GPU, and the per-molecule results are gathered once on the host at the
end (``torch.distributed.all_gather_object``).  Shards are balanced greedily
(longest processing time first) on a cost model of the dominant work, the
exchange build 2 X N^2 o + X o N (N + 1) per SCF iteration.

The reference has no multi-GPU path (its fleet runs buckets sequentially on
one device, ``src/scf/fleet.cpp:325-332``); this module is the B200-native
equivalent of spreading that fleet over the GPUs of one node.
"""

from __future__ import annotations

import heapq
from typing import Callable, Sequence

import torch
import torch.distributed as dist

from . import basis as bas
from .calculator import BatchItemResult, BatchResult


def molecule_cost(atoms, orbital_basis, auxiliary_basis, spherical: bool = True) -> float:
    z = [bas.atomic_number(a[0]) for a in atoms]
    n = bas.count_functions(bas.expand_shells(z, orbital_basis), spherical)
    x = bas.count_functions(bas.expand_shells(z, auxiliary_basis), spherical)
    o = max(1, sum(z) // 2)
    return 2.0 * x * n * n * o + x * o * n * (n + 1)


def shard(costs: Sequence[float], world: int) -> list[list[int]]:
    """Greedy longest-first assignment of item indices to ``world`` shards."""
    if world < 1:
        raise ValueError("world size must be positive")
    heap = [(0.0, r) for r in range(world)]
    out: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda k: -costs[k]):
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    for part in out:
        part.sort()
    return out


def max_over_ranks(value: float, device: torch.device | None = None) -> float:
    """Maximum of a host scalar over all ranks (identity without a process group)."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class DistributedBatch:
    """A ragged batch sharded over the ranks of the default process group.

    ``make_local(systems, charges, multiplicities)`` builds the rank-local
    prepared batch (normally ``calculator.prepare_batch``); ``execute`` runs
    the local shard and returns the full, input-ordered :class:`BatchResult`
    on every rank.
    """

    def __init__(self, systems: Sequence, costs: Sequence[float],
                 make_local: Callable, *, charges=None, multiplicities=None):
        self.world = dist.get_world_size() if dist.is_initialized() else 1
        self.rank = dist.get_rank() if dist.is_initialized() else 0
        n = len(systems)
        if len(costs) != n:
            raise ValueError("one cost per system is required")
        charges = [0] * n if charges is None else list(charges)
        mults = [1] * n if multiplicities is None else list(multiplicities)
        self.n = n
        self.shards = shard(costs, self.world)
        self.local_indices = self.shards[self.rank]
        self.local = None
        if self.local_indices:
            self.local = make_local([systems[i] for i in self.local_indices],
                                    [charges[i] for i in self.local_indices],
                                    [mults[i] for i in self.local_indices])

    def execute(self, coordinates=None, **kwargs) -> BatchResult:
        local_items = []
        if self.local is not None:
            coords = None if coordinates is None else [coordinates[i] for i in self.local_indices]
            res = self.local.execute(coords, **kwargs)
            for k, it in zip(self.local_indices, res.items):
                local_items.append((k, it))
        if self.world > 1:
            gathered: list = [None] * self.world
            dist.all_gather_object(gathered, local_items)
        else:
            gathered = [local_items]
        items: list = [None] * self.n
        for part in gathered:
            for k, it in part:
                items[k] = _reindex(it, k)
        return BatchResult(tuple(items))

    def close(self) -> None:
        if self.local is not None:
            self.local.close()


def _reindex(item: BatchItemResult, index: int) -> BatchItemResult:
    from dataclasses import replace

    return replace(item, index=index)
