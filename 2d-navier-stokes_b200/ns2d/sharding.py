"""Ensembles spread over the GPUs of a job (one process per GPU).

Members are independent trajectories, so they shard with no exchange while
stepping: each rank owns a subset and advances it as one local Ensemble.  The
subsets balance the cost of a step, which grows as N^2 log N per member
(longest-processing-time assignment).  Diagnostics are the only collective:
the per-member measurables (FP64) are summed over ranks at save points with
torch.distributed (NCCL on GPUs, gloo on CPU), so every rank sees the whole
table.  The reference runs such sweeps as separate processes
(run_solver.py:270-292).
"""
import math

import numpy as np

from . import abi


def member_cost(n):
    """Relative cost of one step of an n^2 member (FFT work, n^2 log2 n^2)."""
    return float(n * n) * math.log2(float(n * n))


def partition(sizes, world):
    """Member indices per rank: largest members first, each to the rank with
    the least cost so far (ties to the lower rank).  Deterministic, so every
    rank computes the same assignment without communication."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(sizes)), key=lambda m: (-member_cost(sizes[m]), m))
    load = [0.0] * world
    out = [[] for _ in range(world)]
    for m in order:
        r = min(range(world), key=lambda q: (load[q], q))
        out[r].append(m)
        load[r] += member_cost(sizes[m])
    for r in range(world):
        out[r].sort()
    return out


def imbalance(sizes, world):
    """max rank cost / mean rank cost of `partition`."""
    parts = partition(sizes, world)
    loads = [sum(member_cost(sizes[m]) for m in p) for p in parts]
    mean = sum(loads) / world
    return max(loads) / mean if mean else 1.0


class ShardedEnsemble:
    """The members of `sizes` owned by this rank, as one local ensemble.

    Global member indices are kept at the interface: set_w_hat / get_w_hat on a
    member another rank owns are no-ops / return None.  `make` builds the local
    ensemble (default: ns2d.Ensemble on this process's GPU)."""

    def __init__(self, params, sizes, group=None, make=None):
        import torch.distributed as dist
        self.dist = dist if dist.is_available() and dist.is_initialized() else None
        self.group = group
        self.rank = self.dist.get_rank(group) if self.dist else 0
        self.world = self.dist.get_world_size(group) if self.dist else 1
        self.sizes = [int(s) for s in sizes]
        self.owned = partition(self.sizes, self.world)[self.rank]
        self.local_index = {m: i for i, m in enumerate(self.owned)}
        if make is None:
            from .ensemble import Ensemble
            make = Ensemble
        self.local = make(params, [self.sizes[m] for m in self.owned]) if self.owned else None

    def owns(self, m):
        return m in self.local_index

    def set_w_hat(self, m, w):
        if self.owns(m):
            self.local.set_w_hat(self.local_index[m], w)

    def get_w_hat(self, m):
        return self.local.get_w_hat(self.local_index[m]) if self.owns(m) else None

    def step_n(self, nsteps, dt):
        if self.local is not None:
            self.local.step_n(nsteps, dt)

    def measurables(self, device=None):
        """[n_members, 13] FP64 table of ComputeSystemMeasurables scalars,
        identical on every rank (a sum over ranks of the owned rows)."""
        import torch
        table = np.zeros((len(self.sizes), len(abi.Measures._fields_)))
        for m, i in self.local_index.items():
            table[m] = self.local.measurables(i).as_list()
        if self.dist is None:
            return table
        t = torch.from_numpy(table)
        if device is not None:
            t = t.to(device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM, group=self.group)
        return t.cpu().numpy()

    def close(self):
        if self.local is not None and hasattr(self.local, "close"):
            self.local.close()
            self.local = None
