"""Halo tiles copied by the tensor memory accelerator (TMA) against tiles
copied by the CTA's threads (CG_OPT_TMA = 0).

Bricks away from the periodic wrap take their tiles from a 4-D tensor map of
the substep input; the others, and every brick with the option off, copy by
thread loads with the wrap applied.  The tiles hold the same values, so the
fields must come out identical, for every precision, stencil order and matter
model, on one box and in a launch group (whose kernel reads the maps from its
device table).  The boxes are non-cubic; the last one has no maps (an nz of
18 FP32 or 17 FP64 values is no multiple of 16 bytes).
"""
import numpy as np
import pytest

from cosmograph_b200 import ics, state as S
from cosmograph_b200.evolution import BoxConfig, Evolution

pytestmark = pytest.mark.gpu


def run(states, cfg, tma, steps=3):
    with Evolution(states[0], cfg) as ev:
        ev.set_option("tma", tma)
        ev.step(steps)
        ev.synchronize()
        one = ev.download(0).fields
    with Evolution(states, [cfg] * len(states)) as ev:
        ev.set_option("tma", tma)
        ev.set_option("autotune", 0)
        ev.step(steps)
        ev.synchronize()
        assert ev.groups()[0]["boxes"] == len(states)
        group = [ev.download(q).fields for q in range(len(states))]
    return one, group


@pytest.mark.parametrize("precision", ["fp64", "fp64_fma", "mixed"])
@pytest.mark.parametrize("matter", [S.DUST, S.SCALAR, S.VACUUM])
@pytest.mark.parametrize("order", [2, 4, 6, 8])
def test_tma_tile_copies_match_thread_copies(precision, matter, order):
    # FP64 bricks are 16 points long in z: interior bricks need nz >= 36
    if precision == "mixed":
        shapes = [(24, 20, 32), (20, 28, 16), (12, 16, 18)]
    else:
        shapes = [(24, 20, 48), (20, 28, 40), (12, 16, 17)]
    states = [ics.perturbed(sh, matter, seed=5 + q, amp=1e-3) for q, sh in enumerate(shapes)]
    cfg = BoxConfig(order=order, precision=precision)
    one_t, group_t = run(states, cfg, 1)
    one_c, group_c = run(states, cfg, 0)
    assert np.array_equal(one_t, one_c)
    for q in range(len(states)):
        assert np.array_equal(group_t[q], group_c[q]), q
    assert np.array_equal(one_t, group_t[0])


def test_option_changes_between_steps_only():
    st = ics.perturbed((16, 16, 16), S.DUST, seed=3, amp=1e-3)
    with Evolution(st, BoxConfig(order=4)) as ev:
        ev.step_init()
        ev.rk_stage(1)
        with pytest.raises(RuntimeError, match="between steps"):
            ev.set_option("tma", 0)
