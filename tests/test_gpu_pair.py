"""The FP64 substep with two threads per grid point (CG_OPT_PAIR = 1, the
default) against one thread per point (CG_OPT_PAIR = 0).

Both evaluate every value by the same expression in the same operand order;
only the thread that computes it changes.  The parity build must therefore
agree bit for bit, for every stencil order and matter model, with
Kreiss-Oliger dissipation, on bricks copied by TMA and by threads (boxes that
are not whole numbers of bricks, and one with no tensor maps), one box at a
time and in a launch group.  The FMA build may contract differently in the
two kernels: it is held to 1e-12 of each field's scale.
"""
import numpy as np
import pytest

from cosmograph_b200 import ics, state as S
from cosmograph_b200.evolution import BoxConfig, Evolution

pytestmark = pytest.mark.gpu


def evolve_opts(states, cfg, steps, **opts):
    if not isinstance(states, list):
        states = [states]
    with Evolution(states, [cfg] * len(states)) as ev:
        for k, v in opts.items():
            ev.set_option(k, v)
        ev.step(steps)
        ev.synchronize()
        return [ev.download(q).fields for q in range(len(states))]


SHAPES = [(24, 20, 48), (20, 18, 22), (12, 16, 17)]


@pytest.mark.parametrize("matter", [S.DUST, S.SCALAR, S.VACUUM])
@pytest.mark.parametrize("order", [2, 4, 6, 8])
def test_pair_equals_single_bit_for_bit(matter, order):
    for q, sh in enumerate(SHAPES):
        st = ics.perturbed(sh, matter, seed=60 + q, amp=2e-2)
        cfg = BoxConfig(order=order)
        a = evolve_opts(st, cfg, 3, pair=1)[0]
        b = evolve_opts(st, cfg, 3, pair=0)[0]
        assert np.array_equal(a, b), (sh, int((a != b).sum()))
        c = evolve_opts(st, cfg, 3, pair=1, tma=0)[0]
        assert np.array_equal(a, c), sh


@pytest.mark.parametrize("matter,order", [(S.DUST, 8), (S.VACUUM, 2), (S.SCALAR, 8)])
def test_pair_with_kreiss_oliger(matter, order):
    st = ics.perturbed((20, 18, 40), matter, seed=71, amp=2e-2)
    cfg = BoxConfig(order=order, ko_coeff=0.3)
    a = evolve_opts(st, cfg, 3, pair=1)[0]
    b = evolve_opts(st, cfg, 3, pair=0)[0]
    assert np.array_equal(a, b)


@pytest.mark.parametrize("matter", [S.DUST, S.SCALAR])
def test_pair_group_launch_equals_single_per_box(matter):
    states = [ics.perturbed(sh, matter, seed=80 + q, amp=1e-3)
              for q, sh in enumerate([(16, 16, 16), (24, 20, 18), (16, 16, 48), (12, 14, 16)])]
    cfg = BoxConfig(order=4)
    single = evolve_opts(states, cfg, 3, pair=0, batch=0)
    for grid in (0, 7):
        grouped = evolve_opts(states, cfg, 3, pair=1, autotune=0, group_grid=grid)
        for a, b in zip(single, grouped):
            assert np.array_equal(a, b), grid


def test_pair_fma_build_close_to_single():
    st = ics.perturbed((24, 20, 48), S.DUST, seed=91, amp=2e-2)
    cfg = BoxConfig(order=8, precision="fp64_fma")
    a = evolve_opts(st, cfg, 3, pair=1)[0]
    b = evolve_opts(st, cfg, 3, pair=0)[0]
    scale = np.maximum(np.abs(b).max(axis=(1, 2, 3)), 1e-3)
    assert (np.abs(a - b).max(axis=(1, 2, 3)) / scale).max() < 1e-12


def test_pair_option_changes_between_steps_only():
    st = ics.perturbed((16, 16, 16), S.DUST, seed=3, amp=1e-3)
    with Evolution(st, BoxConfig(order=4)) as ev:
        ev.step_init()
        ev.rk_stage(1)
        with pytest.raises(RuntimeError, match="between steps"):
            ev.set_option("pair", 0)
