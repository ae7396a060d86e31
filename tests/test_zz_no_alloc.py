"""cg_conformal_average_noalloc: the allocation-free grid average, through the
C ABI, against the allocating cg_conformal_average on the same device data.

It serves callers that cannot let a library call cudaMalloc (their own memory
pool, a fixed memory budget, or no implicit device synchronisation); its
scratch is a fixed array inside the library.  This file is collected last so
that a failure here never hides the other GPU tests.
"""
import ctypes

import numpy as np
import pytest

from cosmograph_b200 import _lib, ics, state as S
from cosmograph_b200.evolution import BoxConfig, Evolution

pytestmark = pytest.mark.gpu


def test_noalloc_matches_allocating_entry_point_twice():
    import torch

    L = _lib.load()
    stream = torch.cuda.Stream()
    with Evolution(ics.perturbed((6, 6, 6), S.VACUUM), BoxConfig(order=2)) as ev:
        ev.set_stream(stream.cuda_stream)
        for call, n in enumerate((3_000_000, 4097)):
            rng = np.random.default_rng(100 + call)
            field = torch.tensor(rng.normal(-3.0, 0.2, n), device="cuda")
            phi = torch.tensor(rng.normal(0.0, 0.05, n), device="cuda")
            d_out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
            with torch.cuda.stream(stream):
                rc = L.cg_conformal_average_noalloc(field.data_ptr(), phi.data_ptr(), n, 0.02,
                                                    d_out.data_ptr(), stream.cuda_stream)
            assert rc == 0, L.cg_last_error(None)
            stream.synchronize()
            ref = ctypes.c_double()
            ev._check(L.cg_conformal_average(ev.ctx, field.data_ptr(), phi.data_ptr(), n, 0.02,
                                             ctypes.byref(ref)))
            got = float(d_out.cpu().item())
            assert abs(got - ref.value) <= 1e-13 * abs(ref.value), (call, got, ref.value)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    L = _lib.load()
    too_many = (1 << 30) + 1
    rc = L.cg_conformal_average_noalloc(ctypes.c_void_p(16), ctypes.c_void_p(16), too_many, 0.0,
                                        ctypes.c_void_p(16), None)
    assert rc == -1
    assert b"CG_NOALLOC" not in L.cg_last_error(None)
    assert b"n must be in 1.." in L.cg_last_error(None)
