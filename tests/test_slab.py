"""x-slab decomposition (cosmograph_b200.slab): the slab layout and the ghost
exchange, on the CPU.  The exchange between ranks runs with the gloo backend
(world sizes 2 and 3), each rank holding one slab whose ghost planes start
poisoned; afterwards they must equal the periodic neighbours' planes."""
import ctypes
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from cosmograph_b200 import _lib, ics, slab, state as S
from cosmograph_b200.build import build

NX, G = 24, 4


def global_arrays(seed=0):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((5, NX, 6, 8)), rng.standard_normal((7, NX, 6, 8))


def slab_of(a, nslabs, s, g=G):
    x0, nloc = slab.slab_bounds(a.shape[1], nslabs, s)
    return a[:, np.arange(x0 - g, x0 + nloc + g) % a.shape[1]].copy()


def test_split_and_assemble_round_trip():
    st = ics.perturbed((24, 6, 8), S.DUST, seed=4, amp=1e-2)
    for nslabs in (1, 2, 3, 6):
        parts = slab.split(st, nslabs, G)
        assert all(p.shape == (24 // nslabs + 2 * G, 6, 8) for p in parts)
        back = slab.assemble(parts, G)
        assert np.array_equal(back.fields, st.fields)
        # ghosts are the periodic neighbours' planes
        assert np.array_equal(parts[0].fields[:, :G], st.fields[:, -G:])
        assert np.array_equal(parts[-1].fields[:, -G:], st.fields[:, :G])


def test_ghost_width_and_bounds():
    assert [slab.ghost_width(o) for o in (2, 4, 6, 8)] == [4, 4, 4, 4]
    assert slab.ghost_width(8, ko=True) == 8 and slab.ghost_width(2, ko=True) == 4
    assert slab.slab_bounds(32, 4, 3) == (24, 8)
    with pytest.raises(ValueError):
        slab.slab_bounds(30, 4, 0)
    with pytest.raises(ValueError):
        slab.slab_bounds(24, 4, 0)  # 6 planes: not a multiple of 4


def test_fill_ghosts_local():
    a, f = global_arrays(1)
    for nslabs in (1, 2, 3):
        want = [[torch.from_numpy(slab_of(x, nslabs, s)) for x in (a, f)] for s in range(nslabs)]
        got = [[w.clone() for w in ws] for ws in want]
        for ws in got:
            for w in ws:
                w[:, :G] = float("nan")
                w[:, -G:] = float("nan")
        slab.fill_ghosts(got, G)
        for gs, ws in zip(got, want):
            for g_, w in zip(gs, ws):
                assert torch.equal(g_, w)


def _rank(rank, world, port, outdir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        a, f = global_arrays(2)
        mine = [torch.from_numpy(slab_of(x, world, rank)) for x in (a, f)]
        want = [m.clone() for m in mine]
        for m in mine:
            m[:, :G] = float("nan")
            m[:, -G:] = float("nan")
        halo = slab.DistHalo(G)
        halo.exchange_arrays(mine)
        halo.exchange_arrays(mine)  # a second round on refreshed data changes nothing
        ok = all(torch.equal(m, w) for m, w in zip(mine, want))
        with open(os.path.join(outdir, f"rank{rank}.txt"), "w") as fh:
            fh.write("ok" if ok else "mismatch")
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [1, 2, 3])
def test_gloo_ranks_exchange_ghost_planes(tmp_path, world):
    mp.spawn(_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    for r in range(world):
        assert (tmp_path / f"rank{r}.txt").read_text() == "ok", r


@pytest.mark.parametrize("changes,msg", [
    ({"x_ghost": 3}, "multiple of 4"),
    ({"x_ghost": 8}, "interior planes"),
    ({"x_ghost": 4, "nx": 18}, "interior planes"),
    ({"x_ghost": 4, "nx": 24, "precision": 2, "lapse": 5}, "without K_avg"),
    ({"x_ghost": 4, "nx": 24, "ko_coeff": 0.1}, "Kreiss-Oliger"),
])
def test_create_rejects_bad_slabs(changes, msg):
    build()
    L = _lib.load()
    d = _lib.BoxDesc()
    L.cg_box_desc_default(ctypes.byref(d), 16)
    for k, v in changes.items():
        setattr(d, k, v)
    h = ctypes.c_void_p()
    rc = L.cg_create(ctypes.byref(d), 1, ctypes.byref(h))
    assert rc == -1 and not h.value
    assert msg in L.cg_last_error(None).decode()
