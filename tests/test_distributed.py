"""Multi-process (gloo, world size 2, CPU) tests of the data-parallel host logic."""

import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from vibeqc_b200 import geometry
from vibeqc_b200.calculator import BatchItemResult, BatchResult
from vibeqc_b200.distributed import DistributedBatch, max_over_ranks, molecule_cost, shard


def test_shard_balances_and_covers():
    costs = [float(c) for c in np.random.default_rng(0).integers(1, 1000, size=257)]
    parts = shard(costs, 4)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(257))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(costs)


def test_cost_model_grows_with_size():
    small = molecule_cost(geometry.water_cluster(2, 0), "def2-svp", "cc-pvdz-jkfit")
    big = molecule_cost(geometry.water_cluster(8, 0), "def2-svp", "cc-pvdz-jkfit")
    assert big > 50 * small


class _FakeLocal:
    """Stands in for a GPU prepared batch: energy = -sum of atomic numbers."""

    def __init__(self, systems, charges, mults):
        self.systems = systems

    def execute(self, coords=None, **kw):
        items = []
        for i, s in enumerate(self.systems):
            e = -float(len(s))
            items.append(BatchItemResult(i, 0, "success", e, np.full((len(s), 3), e), True, 1, 0.0,
                                         0.0, "cuda", 0))
        return BatchResult(tuple(items))

    def close(self):
        pass


def _worker(rank, world, port, sizes, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        systems = [geometry.water_cluster(n, n) for n in sizes]
        costs = [molecule_cost(s, "def2-svp", "cc-pvdz-jkfit") for s in systems]
        db = DistributedBatch(systems, costs, _FakeLocal)
        res = db.execute()
        slowest = max_over_ranks(1.0 + rank)
        out[rank] = ([it.energy for it in res.items], [it.index for it in res.items], slowest,
                     len(db.local_indices))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_rank_gather_is_input_ordered():
    sizes = [2, 5, 3, 7, 2, 4, 6]
    manager = mp.get_context("spawn").Manager()
    out = manager.dict()
    mp.start_processes(_worker, args=(2, _free_port(), sizes, out), nprocs=2, join=True,
                       start_method="spawn")
    expected = [-3.0 * n for n in sizes]
    for rank in (0, 1):
        energies, indices, slowest, nlocal = out[rank]
        assert energies == expected
        assert indices == list(range(len(sizes)))
        assert slowest == 2.0
    assert out[0][3] + out[1][3] == len(sizes) and out[0][3] > 0 and out[1][3] > 0
