"""GRF dust initial data built on the GPU (cg_ic_grf_dust) against the host
construction (cosmograph_b200.ics.grf_dust, the steps of the reference's
dust_ic_set_random).

Given the host's density contrast, every field must agree with the host
result to rounding (cuFFT against numpy's FFT, multiplications by 1/dx
against divisions).  With the GPU's own random field: deterministic per seed,
the requested rms contrast, and constraint violations as small as the host
data's.
"""
import numpy as np
import pytest

from cosmograph_b200 import ics, state as S
from cosmograph_b200.evolution import BoxConfig, Evolution

pytestmark = pytest.mark.gpu


def host_delta(shape, seed, rms, ns=0.96):
    kc = min(shape) / 4.0
    return ics.gaussian_random_field(shape, seed, lambda k: k ** ns * np.exp(-(k / kc) ** 2), rms)


@pytest.mark.parametrize("shape,order", [((32, 32, 32), 4), ((24, 20, 16), 8), ((16, 16, 16), 2)])
def test_gpu_construction_matches_host_given_delta(shape, order):
    ref = ics.grf_dust(shape, seed=5, rms_delta=1e-4, order=order)
    got = ics.grf_dust_gpu(shape, seed=5, rms_delta=1e-4, order=order, delta=host_delta(shape, 5, 1e-4))
    assert got.lam == ref.lam and got.dx == ref.dx and got.dt == ref.dt
    for f, name in enumerate(ref.names):
        r, g = ref.fields[f], got.fields[f]
        scale = np.abs(r).max()
        if scale == 0.0:
            assert np.abs(g).max() == 0.0, name
        else:
            assert np.abs(g - r).max() <= 1e-10 * scale, (name, np.abs(g - r).max() / scale)


def test_gpu_random_field():
    a = ics.grf_dust_gpu(32, seed=7, rms_delta=1e-4, order=4)
    b = ics.grf_dust_gpu(32, seed=7, rms_delta=1e-4, order=4)
    c = ics.grf_dust_gpu(32, seed=8, rms_delta=1e-4, order=4)
    assert np.array_equal(a.fields, b.fields)
    assert not np.array_equal(a.fields, c.fields)
    # density contrast of the constructed data: rms close to the request
    rho = a.field("D") * np.exp(-6.0 * a.field("DIFFphi"))
    contrast = (rho - rho.mean()) / rho.mean()
    assert 0.7e-4 < contrast.std() < 1.3e-4
    # constraint violation as small as for the host construction
    host = ics.grf_dust(32, seed=7, rms_delta=1e-4, order=4)
    h = {}
    for name, st in (("gpu", a), ("host", host)):
        with Evolution(st, BoxConfig(order=4)) as ev:
            h[name] = ev.constraints(0)["H"]
    assert h["gpu"][6] < 10 * h["host"][6] and h["gpu"][6] < 1e-3


def test_gpu_ics_reject_non_dust_and_negative_density():
    st = ics.perturbed((16, 16, 16), S.VACUUM, amp=0.0)
    with Evolution(st, BoxConfig(order=4)) as ev:
        with pytest.raises(RuntimeError, match="dust"):
            ev.ic_grf_dust(0)
    with pytest.raises(RuntimeError, match="negative density"):
        ics.grf_dust_gpu(16, seed=3, rms_delta=3.0, order=4)


@pytest.mark.parametrize("shape,order", [((32, 32, 32), 8), ((24, 20, 16), 4)])
def test_gpu_scalar_construction_matches_host_given_the_fluctuation(shape, order):
    """cg_ic_grf_scalar with the host's fluctuation against ics.grf_scalar:
    phi, psi_i and DIFFK to rounding, every other field zero."""
    ref = ics.grf_scalar(shape, seed=6, phi0=1e-2, rms=1e-5, mass=1.0, order=order)
    got = ics.grf_scalar_gpu(shape, seed=6, phi0=1e-2, rms=1e-5, mass=1.0, order=order, host_field=True)
    assert got.dx == ref.dx and got.dt == ref.dt
    for f, name in enumerate(ref.names):
        r, g = ref.fields[f], got.fields[f]
        scale = np.abs(r).max()
        if scale == 0.0:
            assert np.abs(g).max() == 0.0, name
        else:
            assert np.abs(g - r).max() <= 1e-12 * scale, (name, np.abs(g - r).max() / scale)


def test_gpu_scalar_random_field():
    a = ics.grf_scalar_gpu(32, seed=7, phi0=1e-2, rms=1e-5, order=8)
    b = ics.grf_scalar_gpu(32, seed=7, phi0=1e-2, rms=1e-5, order=8)
    c = ics.grf_scalar_gpu(32, seed=8, phi0=1e-2, rms=1e-5, order=8)
    assert np.array_equal(a.fields, b.fields)
    assert not np.array_equal(a.fields, c.fields)
    phi = a.field("phi")
    assert abs(phi.mean() - 1e-2) < 1e-14 and abs(phi.std() - 1e-5) < 1e-12
    # a k^-3 spectrum cut at N/4: no power above the cutoff
    spec = np.abs(np.fft.rfftn(phi - phi.mean())) ** 2
    px, py, pz = np.meshgrid(np.fft.fftfreq(32) * 32, np.fft.fftfreq(32) * 32, np.arange(17), indexing="ij")
    k = np.sqrt(px ** 2 + py ** 2 + pz ** 2)
    assert spec[k > 8.0].max() < 1e-20 * spec[k <= 8.0].max()
    with pytest.raises(RuntimeError, match="scalar"):
        with Evolution(ics.perturbed((16, 16, 16), S.DUST, amp=0.0), BoxConfig(order=4)) as ev:
            ev.ic_grf_scalar(0)
