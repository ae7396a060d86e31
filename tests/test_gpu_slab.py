"""A box cut into x-slabs (x_ghost > 0), all slabs in one context on one GPU
with the ghost planes refreshed by device copies before every substep, must
evolve exactly as the undivided box: the assembled interiors equal the
single-box run bit for bit (FP64; every point sees the same taps and the same
arithmetic).  The exchange between GPUs uses the same planes
(tests/test_slab.py checks it on CPU ranks)."""
import numpy as np
import pytest

from cosmograph_b200 import ics, slab, state as S
from cosmograph_b200.evolution import BoxConfig, Evolution, evolve

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("matter,order,nslabs,precision", [
    (S.DUST, 4, 2, "fp64"), (S.DUST, 8, 4, "fp64"), (S.SCALAR, 6, 2, "fp64"),
    (S.VACUUM, 2, 3, "fp64_fma"), (S.DUST, 8, 2, "fp64_fma"),
])
def test_slabs_evolve_like_the_whole_box(matter, order, nslabs, precision):
    shape = (8 * nslabs, 20, 48)  # nz = 48: interior z bricks take the TMA path
    st = ics.perturbed(shape, matter, seed=31 + order, amp=1e-3)
    cfg = BoxConfig(order=order, precision=precision)
    g = slab.ghost_width(order)
    with slab.SlabEvolution(slab.split(st, nslabs, g), cfg, g) as se:
        se.step(3)
        se.ev.synchronize()
        got = slab.assemble(se.download(), g)
    want = evolve(st, 3, cfg)
    assert np.array_equal(got.fields, want.fields)
    assert got.frw_phi == want.frw_phi and got.frw_K == want.frw_K


def test_slabs_with_kreiss_oliger():
    st = ics.perturbed((32, 12, 16), S.DUST, seed=5, amp=1e-3)
    cfg = BoxConfig(order=8, ko_coeff=0.05)
    g = slab.ghost_width(8, ko=True)
    with slab.SlabEvolution(slab.split(st, 2, g), cfg, g) as se:
        se.step(2)
        got = slab.assemble(se.download(), g)
    assert np.array_equal(got.fields, evolve(st, 2, cfg).fields)


def test_slab_constraints_cover_the_interior():
    """Constraint statistics of one slab after a ghost refresh equal those of
    the same planes inside the whole box: the means of the slab interiors
    average to the box's mean."""
    st = ics.perturbed((16, 16, 16), S.DUST, seed=8, amp=1e-3)
    cfg = BoxConfig(order=4)
    g = slab.ghost_width(4)
    with slab.SlabEvolution(slab.split(st, 2, g), cfg, g) as se:
        se.step(1)
        se.refresh()
        parts = [se.ev.constraints(b)["H"] for b in range(2)]
    with Evolution(st, cfg) as ev:
        ev.step(1)
        whole = ev.constraints(0)["H"]
    mean = 0.5 * (parts[0][0] + parts[1][0])
    assert abs(mean - whole[0]) <= 1e-12 * max(abs(whole[0]), 1e-300) + 1e-18
    assert max(parts[0][2], parts[1][2]) == pytest.approx(whole[2], rel=1e-13)


def test_cg_step_refuses_slabs():
    st = ics.perturbed((16, 8, 8), S.DUST, seed=2, amp=1e-3)
    with Evolution(slab.split(st, 1, 4)[0], BoxConfig(order=4, x_ghost=4)) as ev:
        with pytest.raises(RuntimeError, match="x-slab"):
            ev.step(1)


@pytest.mark.parametrize("matter,order", [(S.DUST, 4), (S.DUST, 8), (S.SCALAR, 6)])
def test_mixed_slabs_follow_the_whole_box(matter, order):
    """FP32-mixed slabs with the whole box's background (the slabs' sums
    added up): the assembled fields agree with the undivided mixed run to
    FP32 roundoff of the perturbation, and with FP64 as the mixed form does."""
    shape = (32, 16, 24)
    st = ics.perturbed(shape, matter, seed=41, amp=1e-3)
    cfg = BoxConfig(order=order, precision="mixed")
    g = slab.ghost_width(order)
    with slab.SlabEvolution(slab.split(st, 2, g), cfg, g) as se:
        se.step(4)
        got = slab.assemble(se.download(), g)
    whole = evolve(st, 4, cfg)
    ref = evolve(st, 4, BoxConfig(order=order, precision="fp64"))
    for f in range(ref.fields.shape[0]):
        spread = np.abs(ref.fields[f] - ref.fields[f].mean()).max()
        if spread == 0.0:
            continue
        assert np.abs(got.fields[f] - whole.fields[f]).max() <= 1e-6 * spread, ref.names[f]
        assert np.abs(got.fields[f] - ref.fields[f]).max() <= 1e-4 * spread, ref.names[f]


def test_mixed_slab_constraints_are_refused():
    st = ics.perturbed((16, 8, 8), S.DUST, seed=2, amp=1e-3)
    with slab.SlabEvolution(slab.split(st, 1, 4), BoxConfig(order=4, precision="mixed"), 4) as se:
        se.step(1)
        with pytest.raises(RuntimeError, match="x-slab"):
            se.ev.constraints(0)


@pytest.mark.parametrize("lapse", ["OnePlusLog", "ConformalFLRW"])
def test_slabs_with_a_kavg_lapse(lapse):
    """Lapses that use the grid average of K: every slab takes the whole box's
    K_avg (the slabs' sums added up) before each substep.  The sums run in a
    different order than the undivided box's, so the agreement is to
    roundoff, not bit for bit."""
    st = ics.perturbed((24, 16, 32), S.DUST, seed=12, amp=1e-3)
    cfg = BoxConfig(order=4, lapse=lapse)
    g = slab.ghost_width(4)
    with slab.SlabEvolution(slab.split(st, 3, g), cfg, g) as se:
        se.step(3)
        got = slab.assemble(se.download(), g)
    want = evolve(st, 3, cfg)
    for f in range(want.fields.shape[0]):
        scale = max(np.abs(want.fields[f]).max(), 1e-300)
        assert np.abs(got.fields[f] - want.fields[f]).max() <= 1e-12 * scale, want.names[f]


def test_kavg_slab_refuses_a_substep_without_kavg():
    st = ics.perturbed((16, 8, 8), S.DUST, seed=2, amp=1e-3)
    part = slab.split(st, 1, 4)[0]
    with Evolution(part, BoxConfig(order=4, lapse="OnePlusLog", x_ghost=4)) as ev:
        ev.step_init()
        with pytest.raises(RuntimeError, match="cg_set_kavg"):
            ev.rk_stage(1)
