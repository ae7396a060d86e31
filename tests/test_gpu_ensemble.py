"""Ensembles of boxes advanced by one launch per substep (launch groups).

A group's launch must give every box exactly what its own launch gives: the
bricks are independent, so the launch order, the persistent grid the
autotuner picks and the CUDA-graph replay change nothing, bit for bit.
"""
import numpy as np
import pytest

from cosmograph_b200 import ics, state as S
from cosmograph_b200.evolution import BoxConfig, Evolution, evolve

pytestmark = pytest.mark.gpu


def ensemble(shapes, matter=S.DUST, seed0=40):
    return [ics.perturbed(sh, matter, seed=seed0 + q, amp=1e-3) for q, sh in enumerate(shapes)]


def run(states, cfg, steps, **opts):
    with Evolution(states, [cfg] * len(states)) as ev:
        for k, v in opts.items():
            ev.set_option(k, v)
        ev.step(steps)
        ev.synchronize()
        groups = ev.groups()
        return [ev.download(b).fields for b in range(len(states))], groups


# uneven sizes, including boxes that are not whole numbers of bricks
SHAPES = [(16, 16, 16), (24, 20, 18), (16, 16, 32), (20, 16, 16), (12, 14, 16)]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("grid", [0, 7, 64])
def test_group_launch_equals_per_box_launches(precision, grid):
    """One CTA per brick (grid 0) and persistent grids smaller than the work
    list, the last CTA getting one brick fewer (7) or a box boundary inside a
    CTA's stride (64)."""
    states = ensemble(SHAPES)
    cfg = BoxConfig(order=4, lapse="Harmonic", precision=precision)
    per_box, g0 = run(states, cfg, 3, batch=0)
    grouped, g1 = run(states, cfg, 3, autotune=0, group_grid=grid)
    assert g0 == [] and len(g1) == 1 and g1[0]["boxes"] == len(states) and g1[0]["grid"] == grid
    for a, b in zip(per_box, grouped):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_autotuned_group_equals_per_box_launches(precision):
    states = ensemble(SHAPES, seed0=45)
    cfg = BoxConfig(order=8, lapse="Harmonic", precision=precision)
    per_box, _ = run(states, cfg, 2, batch=0)
    tuned, g = run(states, cfg, 2)
    assert g[0]["tuned"] and g[0]["grid"] >= -1
    for a, b in zip(per_box, tuned):
        assert np.array_equal(a, b)


def test_graph_replay_and_launch_shapes_change_nothing():
    states = ensemble(SHAPES[:4], seed0=50)
    cfg = BoxConfig(order=8, lapse="Harmonic", precision="fp64")
    ref, _ = run(states, cfg, 2, batch=0)
    untuned, gu = run(states, cfg, 2, autotune=0)
    assert gu[0]["grid"] == 0 and not gu[0]["tuned"]
    graphed, _ = run(states, cfg, 2, graph=1)
    for a, b, c in zip(ref, untuned, graphed):
        assert np.array_equal(a, b) and np.array_equal(a, c)
    # repeated graph calls (the executable graph is updated in place)
    with Evolution(states, [cfg] * len(states)) as ev:
        ev.set_option("graph", 1)
        ev.step(1)
        ev.step(1)
        ev.synchronize()
        for q in range(len(states)):
            assert np.array_equal(ev.download(q).fields, ref[q])


def test_substeps_and_mixed_matter_groups():
    dust = ensemble([(16, 16, 16), (16, 16, 32)], seed0=60)
    vac = ensemble([(16, 16, 16), (32, 16, 16)], matter=S.VACUUM, seed0=70)
    states = dust + vac
    cfg = BoxConfig(order=4, lapse="Harmonic")
    with Evolution(states, [cfg] * 4) as ev:
        groups = ev.groups()
        assert sorted(g["boxes"] for g in groups) == [2, 2]
        ev.step_init()
        for n in (1, 2, 3, 4):
            ev.rk_stage(n)
        ev.synchronize()
        got = [ev.download(q).fields for q in range(4)]
    ref, _ = run(states, cfg, 1, batch=0)
    for a, b in zip(got, ref):
        assert np.array_equal(a, b)


def test_every_box_is_stepped_with_mixed_options():
    """Boxes with Kreiss-Oliger dissipation keep their own launches; the others
    of the same kind still form a group; every box advances."""
    shapes = [(16, 16, 16), (16, 16, 32), (20, 16, 16)]
    states = ensemble(shapes, seed0=80)
    cfgs = [BoxConfig(order=8, ko_coeff=0.2), BoxConfig(order=8), BoxConfig(order=8)]
    with Evolution(states, cfgs) as ev:
        assert [g["boxes"] for g in ev.groups()] == [2]
        ev.step(2)
        ev.synchronize()
        got = [ev.download(q) for q in range(3)]
    for q, (st, cfg) in enumerate(zip(states, cfgs)):
        ref = evolve(st, 2, cfg)
        assert got[q].step == 2 and np.array_equal(got[q].fields, ref.fields), q
