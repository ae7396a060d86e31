"""The bounded wait of the TMA tile copies (CG_STATUS_TILE_TIMEOUT).

With CG_OPT_TMA_WAIT set to one clock cycle, every tile copy outlasts the
first wait, so each substep must flag the timeout and cg_synchronize must
fail.  The waits then go on (bounded) until the late copies land, before a
buffer is reused or a CTA leaves: the fields come out exactly as without the
option, and the context and the device stay usable.  Nothing here makes a
GPU fault or hang: every copy completes; only the reporting path runs.
"""
import numpy as np
import pytest

from cosmograph_b200 import _lib, ics
from cosmograph_b200.evolution import BoxConfig, Evolution, evolve

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_late_tile_copies_are_reported_and_waited_for(precision):
    st = ics.grf_dust(64, seed=3, rms_delta=1e-4, order=4)
    cfg = BoxConfig(order=4, precision=precision)
    ref = evolve(st, 2, cfg)
    with Evolution(st, cfg) as ev:
        ev.set_option("tma_wait", 1)
        ev.step(2)
        assert ev.status() & _lib.STATUS_TILE_TIMEOUT
        with pytest.raises(RuntimeError, match="TMA tile copy"):
            ev.synchronize()
        got = ev.download(0)
    assert np.array_equal(got.fields, ref.fields)
    again = evolve(st, 2, cfg)  # a new context on the same device
    assert np.array_equal(again.fields, ref.fields)


def test_tma_wait_option_is_checked():
    st = ics.grf_dust(16, seed=3, rms_delta=1e-4, order=4)
    with Evolution(st, BoxConfig(order=4)) as ev:
        with pytest.raises(RuntimeError, match="cycle count"):
            ev.set_option("tma_wait", -5)
        ev.set_option("tma_wait", 0)  # the default
        ev.step(1)
        ev.synchronize()
        assert ev.status() == 0
