"""cg_conformal_average: the reference's conformal_average (utils/math.h:1403-1415)
on device arrays, through the C ABI, against numpy in FP64."""
import ctypes

import numpy as np
import pytest

from cosmograph_b200 import _lib, ics, state as S
from cosmograph_b200.evolution import BoxConfig, Evolution

pytestmark = pytest.mark.gpu


def reference_average(field, phi, phi_frw):
    e = np.exp(6.0 * (phi + phi_frw))
    n = field.size
    vol = e.sum() / n
    return (e * field).sum() / n / vol


@pytest.mark.parametrize("n", [1, 255, 256, 257, 100_000, 3_000_000])
def test_conformal_average_matches_numpy(n):
    import torch

    rng = np.random.default_rng(n)
    field = rng.normal(-3.0, 0.1, n)
    phi = rng.normal(0.0, 0.05, n)
    dfield = torch.tensor(field, device="cuda")
    dphi = torch.tensor(phi, device="cuda")
    with Evolution(ics.perturbed((6, 6, 6), S.VACUUM), BoxConfig(order=2)) as ev:
        out = ctypes.c_double()
        ev._check(ev.L.cg_conformal_average(ev.ctx, dfield.data_ptr(), dphi.data_ptr(), n, 0.01,
                                            ctypes.byref(out)))
    ref = reference_average(field, phi, 0.01)
    assert abs(out.value - ref) <= 1e-13 * abs(ref)


def test_conformal_average_rejects_bad_arguments():
    with Evolution(ics.perturbed((6, 6, 6), S.VACUUM), BoxConfig(order=2)) as ev:
        out = ctypes.c_double()
        rc = ev.L.cg_conformal_average(ev.ctx, None, None, 10, 0.0, ctypes.byref(out))
        assert rc == -1 and b"null" in ev.L.cg_last_error(ev.ctx)
