"""Host <-> device state copies through the C ABI: the overlapped exchange
(cg_exchange_state_async) must equal a download followed by an upload on the
same context (the FRW background and the step count behave the same way)."""
import ctypes

import numpy as np
import pytest
import torch

from cosmograph_b200 import ics, state as S
from cosmograph_b200.evolution import BoxConfig, Evolution

pytestmark = pytest.mark.gpu

DP = ctypes.POINTER(ctypes.c_double)


def pinned(a: np.ndarray) -> torch.Tensor:
    return torch.from_numpy(np.ascontiguousarray(a).reshape(-1)).pin_memory()


def ptr(t: torch.Tensor):
    return ctypes.cast(t.data_ptr(), DP)


def stream_states(states, cfg, exchange: bool, prefetch: bool = False):
    """One step per state, each state uploaded in turn; returns each step's result."""
    ins = [pinned(s.fields) for s in states]
    outs = [torch.zeros_like(ins[0]).pin_memory() for _ in states]
    with Evolution(states[0], cfg) as ev:
        n = ins[0].numel()
        ev._check(ev.L.cg_upload_state_async(ev.ctx, 0, ptr(ins[0]), n))
        ev.step(1)
        for q in range(1, len(states)):
            if prefetch:
                ev._check(ev.L.cg_prefetch_state_async(ev.ctx, 0, ptr(ins[q]), n))
            if exchange:
                ev._check(ev.L.cg_exchange_state_async(ev.ctx, 0, ptr(outs[q - 1]), ptr(ins[q]), n))
            else:
                ev._check(ev.L.cg_download_state_async(ev.ctx, 0, ptr(outs[q - 1]), n))
                ev._check(ev.L.cg_upload_state_async(ev.ctx, 0, ptr(ins[q]), n))
            ev.step(1)
        ev._check(ev.L.cg_download_state_async(ev.ctx, 0, ptr(outs[-1]), n))
        ev.synchronize()
        steps = ev.download(0).step
    return [o.numpy().copy() for o in outs], steps


@pytest.mark.parametrize("prefetch", [False, True])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_exchange_equals_download_then_upload(precision, prefetch):
    """Plain exchange (field-by-field overlap) and staged exchange (prefetched
    input, download from a device copy while the next step runs)."""
    cfg = BoxConfig(order=8, precision=precision)
    states = [ics.perturbed((16, 20, 32), S.DUST, seed=q, amp=1e-3) for q in range(4)]
    got, steps_x = stream_states(states, cfg, exchange=True, prefetch=prefetch)
    want, steps_s = stream_states(states, cfg, exchange=False)
    for q in range(len(states)):
        assert np.array_equal(got[q], want[q]), q
        assert not np.array_equal(got[q], pinned(states[q].fields).numpy())  # a step was taken
    assert steps_x == steps_s


def test_exchange_rejects_bad_arguments():
    st = ics.perturbed((8, 8, 8), S.DUST, seed=1, amp=1e-3)
    h = pinned(st.fields)
    with Evolution(st, BoxConfig(order=2)) as ev:
        assert ev.L.cg_exchange_state_async(ev.ctx, 0, ptr(h), ptr(h), h.numel() - 1) == -1
        assert b"count" in ev.L.cg_last_error(ev.ctx)
        assert ev.L.cg_exchange_state_async(ev.ctx, 0, None, ptr(h), h.numel()) == -1
        assert ev.L.cg_exchange_state_async(ev.ctx, 3, ptr(h), ptr(h), h.numel()) == -1


def test_prefetch_then_plain_copies_keep_order():
    """A staged exchange followed by a plain download into the same host
    buffer: the plain download lands last."""
    cfg = BoxConfig(order=4)
    a = ics.perturbed((16, 16, 16), S.DUST, seed=1, amp=1e-3)
    b = ics.perturbed((16, 16, 16), S.DUST, seed=2, amp=1e-3)
    h_b = pinned(b.fields)
    h_out = torch.zeros_like(h_b).pin_memory()
    with Evolution(a, cfg) as ev:
        n = h_b.numel()
        ev.step(1)
        ev._check(ev.L.cg_prefetch_state_async(ev.ctx, 0, ptr(h_b), n))
        ev._check(ev.L.cg_exchange_state_async(ev.ctx, 0, ptr(h_out), ptr(h_b), n))
        ev._check(ev.L.cg_download_state_async(ev.ctx, 0, ptr(h_out), n))
        ev.synchronize()
    assert np.array_equal(h_out.numpy(), h_b.numpy())
    with Evolution(a, cfg) as ev:
        assert ev.L.cg_prefetch_state_async(ev.ctx, 0, ptr(h_b), n + 1) == -1
        assert ev.L.cg_prefetch_state_async(ev.ctx, 0, None, n) == -1
