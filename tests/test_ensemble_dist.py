"""Ensemble partitioning across ranks and the gather of per-box results.

The multi-GPU form of the path is a set of independent boxes split across
ranks with no data-path communication.  These CPU tests run the rank logic
with the gloo backend (world size 2): each rank evolves its share of a small
ensemble with the CPU restatement (test infrastructure) and the gathered
results must equal a single-process run box for box.
"""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from cosmograph_b200 import ensemble

SMALL = [ensemble.BoxSpec(i, n, 500 + i, rms) for i, (n, rms) in
         enumerate([(8, 1e-4), (12, 3e-5), (8, 1e-3), (10, 2e-4), (12, 1e-5)])]


def test_standard_ensemble_spec():
    specs = ensemble.standard_ensemble()
    assert len(specs) == 48
    assert [s.n for s in specs] == [32] * 16 + [64] * 16 + [96] * 16
    assert [s.seed for s in specs] == list(range(1000, 1048))
    assert all(1e-5 <= s.rms_delta <= 1e-3 for s in specs)
    assert specs == ensemble.standard_ensemble()  # deterministic


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_partition_complete_disjoint_balanced(world):
    specs = ensemble.standard_ensemble()
    costs = [s.points for s in specs]
    shares = ensemble.partition(costs, world)
    flat = sorted(i for s in shares for i in s)
    assert flat == list(range(len(specs)))
    loads = [sum(costs[i] for i in s) for s in shares]
    assert max(loads) <= 1.25 * min(loads)
    assert ensemble.partition(costs, world) == shares


def evolve_checksums(specs):
    import oracle

    out = {}
    for s, st in zip(specs, ensemble.initial_states(specs, order=4)):
        ev = oracle.evolve(st, 1, order=4, threads=1)
        out[s.box_id] = (float(np.abs(ev.fields).sum()), float(ev.fields[6].sum()))
    return out


def _rank(rank, world, port, outdir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = ensemble.local_share(SMALL, rank, world)
        merged = ensemble.gather(evolve_checksums(mine), world)
        with open(os.path.join(outdir, f"rank{rank}.txt"), "w") as fh:
            fh.write(repr(sorted(merged.items())) + "\n" + repr([s.box_id for s in mine]))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_match_one_process(tmp_path):
    world = 2
    mp.spawn(_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    want = sorted(evolve_checksums(SMALL).items())
    shares = []
    for r in range(world):
        merged, mine = (tmp_path / f"rank{r}.txt").read_text().splitlines()
        assert eval(merged) == want
        shares.append(eval(mine))
    assert sorted(shares[0] + shares[1]) == [s.box_id for s in SMALL] and not set(shares[0]) & set(shares[1])
