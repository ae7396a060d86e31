"""The shift (the reference's compile-time USE_BSSN_SHIFT with
USE_GAMMA_DRIVER: beta^i, the Gamma-driver's B^i and expN evolved, every
field advected with upwinded stencils) against the reference's own sources
built with both switches and correctly rounded exp/expm1/log1p
(oracle/_ref/*_strict_cr_shift).  Every call goes through the C ABI.

Tolerances: bit for bit where the right-hand side takes no logarithm and no
grid average; 1e-12 norm-wise per field for the damped-wave gauges (the
C library's log and CUDA's may differ in the last bit) and for the 1+log
lapse (K_avg is summed in a different order than the reference's OpenMP
reduction).  The golden fixtures of tests/golden/*_shift* (the reference's
strict build) are checked by test_gpu_parity.test_golden_evolve.
"""
import numpy as np
import pytest

import oracle
from oracle import build_ref
from cosmograph_b200 import ics, state as S
from cosmograph_b200.evolution import BoxConfig, evolve
from helpers import field_errors, worst

pytestmark = pytest.mark.gpu

SHIFT_CASES = [
    # matter, shape, order, shift gauge, lapse, gauge parameters, KO coefficient, bit for bit
    (S.DUST, (16, 12, 20), 4, "GammaDriver", "Harmonic", {"gd_eta": 0.5}, 0.0, True),
    (S.DUST, (16, 12, 20), 4, "AwAShiftedWave", "AwAShiftedWave", {"gauge_wave_dir": 2}, 0.0, True),
    (S.SCALAR, (12, 16, 12), 2, "AijDriverShift", "OnePlusLog", {}, 0.2, False),
    (S.VACUUM, (16, 16, 16), 8, "DampedWave", "DampedWave", {"dw_mu_l": 0.2, "dw_mu_s": 0.3, "dw_p": 0.5}, 0.1,
     False),
    (S.SCALAR, (12, 12, 16), 6, "Static", "Harmonic", {}, 0.0, True),
]


@pytest.mark.parametrize("matter,shape,order,shift,lapse,extra,ko,exact", SHIFT_CASES,
                         ids=[f"{c[3]}-o{c[2]}" for c in SHIFT_CASES])
def test_shift_against_the_reference_build(matter, shape, order, shift, lapse, extra, ko, exact):
    binp = build_ref.binary_path(*shape, order, "strict_cr_shift")
    if not binp.exists():
        pytest.skip(f"{binp.name} was not built")
    st = ics.perturbed(shape, matter, seed=31 + order, amp=2e-2, shift=True)
    kw = dict(lapse=lapse, shift=shift, ko_coeff=ko, **extra)
    ref, _ = oracle.run_reference(binp, "evolve", st, steps=4, **kw)
    got = evolve(st, 4, BoxConfig(order=order, **kw))
    diff = int((got.fields != ref.fields).sum())
    errs = field_errors(got.fields, ref.fields, st.names, floor=1e-18)
    print("shift", shift, "lapse", lapse, "order", order, "worst", worst(errs), "differing values:", diff)
    if exact:
        assert diff == 0, worst(errs)
    assert worst(errs)[1] <= 1e-12, worst(errs)
    # the shift matters: without its fields the same data end elsewhere
    nbase = S.num_fields(matter)
    plain = S.BoxState(fields=st.fields[:nbase].copy(), matter=matter, dx=st.dx, dt=st.dt, lam=st.lam)
    other = evolve(plain, 4, BoxConfig(order=order, lapse=lapse, ko_coeff=ko, **{
        k: v for k, v in extra.items() if k in ("dw_mu_l", "dw_p")}))
    assert np.abs(other.fields - got.fields[:nbase]).max() > 1e-6


def test_zero_shift_leaves_the_other_fields_unchanged():
    """beta^i = 0 under the static shift gauge: every shift term is an exact
    zero, so the BSSN and matter fields come out bit for bit as without the
    shift fields, beta stays zero and expN follows -alpha K / 3."""
    st = ics.perturbed((16, 16, 20), S.DUST, seed=5, amp=2e-2, shift=True)
    nbase = S.num_fields(S.DUST)
    st.fields[nbase:nbase + 3] = 0.0
    got = evolve(st, 3, BoxConfig(order=4, shift="Static"))
    plain = S.BoxState(fields=st.fields[:nbase].copy(), matter=S.DUST, dx=st.dx, dt=st.dt, lam=st.lam)
    ref = evolve(plain, 3, BoxConfig(order=4))
    assert np.array_equal(got.fields[:nbase], ref.fields)
    assert not np.any(got.fields[nbase:nbase + 3])
    assert not np.array_equal(got.field("expN"), st.field("expN"))
