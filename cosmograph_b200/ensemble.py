"""Ensembles of independent periodic boxes: specification, initial data and
partitioning across ranks.

The reference evolves one box per process; an ensemble of boxes of uneven
sizes and seeds is what a user runs many of.  Here a whole ensemble lives in
one context per GPU (boxes of the same order, matter and precision share one
launch per substep).  Across GPUs the boxes are independent, so ranks take
disjoint shares with no data-path communication: partition() balances the
shares by grid points (largest box first onto the least-loaded rank) and only
per-box results are gathered at the end.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from . import ics


@dataclasses.dataclass(frozen=True)
class BoxSpec:
    box_id: int
    n: int            # points per axis
    seed: int
    rms_delta: float  # rms density contrast of the Gaussian random field

    @property
    def points(self) -> int:
        return self.n ** 3


def standard_ensemble(base_seed: int = 1000, per_size: int = 16, sizes=(32, 64, 96),
                      rms_range=(1.0e-5, 1.0e-3)) -> list[BoxSpec]:
    """per_size boxes of each size; seed = base_seed + box id; rms delta drawn
    log-uniformly in rms_range from a generator seeded with base_seed."""
    rng = np.random.Generator(np.random.MT19937(base_seed))
    specs = []
    for n in sizes:
        for _ in range(per_size):
            bid = len(specs)
            rms = float(np.exp(rng.uniform(np.log(rms_range[0]), np.log(rms_range[1]))))
            specs.append(BoxSpec(bid, n, base_seed + bid, rms))
    return specs


def initial_states(specs, order: int = 4, gpu: bool = False):
    """Seeded Gaussian-random-field dust initial data for each box (random
    field on the host; the construction on the GPU when gpu=True, the same
    data to rounding)."""
    if gpu:
        return [ics.grf_dust_gpu(s.n, seed=s.seed, rms_delta=s.rms_delta, order=order, host_delta=True)
                for s in specs]
    return [ics.grf_dust(s.n, seed=s.seed, rms_delta=s.rms_delta, order=order) for s in specs]


def partition(costs, world: int) -> list[list[int]]:
    """Indices of `costs` split into `world` shares of near-equal total cost:
    largest first onto the least-loaded share (ties to the lower rank); each
    share in ascending index order.  Deterministic, so every rank computes the
    same split without communication."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0] * world
    shares: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        shares[r].append(i)
        load[r] += costs[i]
    return [sorted(s) for s in shares]


def local_share(specs, rank: int, world: int):
    """The specs this rank evolves."""
    return [specs[i] for i in partition([s.points for s in specs], world)[rank]]


def gather(results: dict, world: int) -> dict:
    """Merge per-rank {box_id: result} dictionaries (all ranks receive the
    union); a plain copy when world == 1."""
    if world == 1:
        return dict(results)
    import torch.distributed as dist

    parts = [None] * world
    dist.all_gather_object(parts, results)
    merged = {}
    for p in parts:
        overlap = merged.keys() & p.keys()
        if overlap:
            raise RuntimeError(f"boxes evolved on two ranks: {sorted(overlap)}")
        merged.update(p)
    return merged
