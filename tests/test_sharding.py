"""Host logic of ensembles spread over ranks (ns2d.sharding): the cost-balanced
partition, and the gathering of per-member diagnostics over two gloo ranks on
the CPU, with a stand-in for the local GPU ensemble."""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

from ns2d import abi
from ns2d import sharding

BENCH_SIZES = [128] * 32 + [256] * 24 + [512] * 8


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_partition_covers_each_member_once(world):
    parts = sharding.partition(BENCH_SIZES, world)
    flat = sorted(m for p in parts for m in p)
    assert flat == list(range(len(BENCH_SIZES)))
    assert sharding.partition(BENCH_SIZES, world) == parts  # deterministic


@pytest.mark.parametrize("world", [2, 4, 8])
def test_partition_balances_cost(world):
    # the benchmark ensemble splits within 20 % of even up to 8 GPUs
    assert sharding.imbalance(BENCH_SIZES, world) <= 1.2


class FakeEnsemble:
    """CPU stand-in: member measurables are a known function of its size and
    of a value set through set_w_hat."""

    def __init__(self, params, sizes):
        self.sizes = sizes
        self.vals = [0.0] * len(sizes)
        self.steps = 0

    def set_w_hat(self, i, w):
        self.vals[i] = float(np.abs(w).max())

    def step_n(self, n, dt):
        self.steps += n

    def measurables(self, i):
        m = abi.Measures()
        m.energy = self.sizes[i] + self.vals[i]
        m.enstrophy = float(self.steps)
        return m


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        sizes = [64, 128, 64, 256, 128, 64]
        e = sharding.ShardedEnsemble(abi.default_params(), sizes, make=FakeEnsemble)
        for m in range(len(sizes)):
            e.set_w_hat(m, np.full((2, 2), float(m)))
        e.step_n(5, 1e-3)
        q.put((rank, e.owned, e.measurables()))
    finally:
        dist.destroy_process_group()


def test_two_rank_gather_of_measurables():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    res.sort()
    sizes = [64, 128, 64, 256, 128, 64]
    owned = [r[1] for r in res]
    assert sorted(owned[0] + owned[1]) == list(range(len(sizes)))
    want = np.zeros((len(sizes), 13))
    for m, n in enumerate(sizes):
        want[m, 0] = n + m
        want[m, 1] = 5.0
    for _, _, table in res:
        assert np.array_equal(table, want)
