"""The CPU restatement (oracle/cg_oracle.c) against the reference's own outputs.

The golden fixtures were produced by the reference's BSSN/Dust/Scalar/Lambda
sources compiled unmodified (tests/golden/make_golden.py); these tests pin the
restatement to them before it is trusted as the checker of the CUDA path.
"""
import math

import numpy as np
import pytest

import oracle
from helpers import field_errors, golden_index, load_golden, worst

# the shift fixtures pin the CUDA path on the reference build directly (the
# restatement has no shift)
EVOLVE_CASES = [k for k, v in golden_index().items() if v["mode"] == "evolve" and "shift" not in v["config"]]


@pytest.mark.parametrize("name", EVOLVE_CASES)
def test_restatement_matches_reference_evolve(name):
    inp, out, _, meta = load_golden(name)
    got = oracle.evolve(inp, meta["steps"], meta["order"], threads=2, **meta["config"])
    errs = field_errors(got.fields, out.fields, inp.names)
    # bit-identical except where the reference reduces over the grid in an
    # OpenMP-order-dependent way (K_avg for the OnePlusLog lapse)
    tol = 1e-13 if meta["config"]["lapse"] in ("OnePlusLog", "ConformalFLRW", "Anharmonic") else 0.0
    assert worst(errs)[1] <= tol, worst(errs)


SHIFT_CASES = [k for k, v in golden_index().items() if v["mode"] == "evolve" and "shift" in v["config"]]


@pytest.mark.parametrize("name", SHIFT_CASES)
def test_shift_fixtures_reproduce_on_the_reference_build(name):
    """The shift fixtures (the CUDA path's parity cases for USE_BSSN_SHIFT with
    USE_GAMMA_DRIVER) come back bit for bit from a fresh run of the
    reference's own shift build; runs only where the reference checkout is."""
    from oracle import build_ref

    if not build_ref.reference_available():
        pytest.skip("reference checkout not present")
    inp, out, _, meta = load_golden(name)
    binp = build_ref.build(*meta["shape"], meta["order"], "strict_shift")
    got, _ = oracle.run_reference(binp, "evolve", inp, steps=meta["steps"], threads=1, **meta["config"])
    assert got.shift and np.array_equal(got.fields, out.fields)


def test_restatement_matches_reference_rhs():
    inp, out, _, meta = load_golden("dust_o4_rhs")
    got = oracle.rhs(inp, meta["order"], **meta["config"])
    assert np.array_equal(got, out.fields)


@pytest.mark.parametrize("name", ["dust_o8_constraints", "scalar_o6_constraints"])
def test_restatement_matches_reference_constraints(name):
    inp, _, ref, meta = load_golden(name)
    got = oracle.constraints(inp, meta["order"], **meta["config"])
    for c in "HMGAS":
        # A and S vanish after the normalisation up to roundoff: floor 1e-3
        floor = 1e-3 if c in "AS" else 1e-300
        rel = np.abs(got[c] - ref[c]) / np.maximum(np.abs(ref[c]), floor)
        assert rel.max() < 1e-12, (c, got[c], ref[c])


@pytest.mark.parametrize("name", ["dust_o8_constraints", "scalar_o6_constraints"])
def test_restatement_matches_reference_field_statistics(name):
    """io_bssn_dump_statistics (IO/io.cc:8-14, 386-403): volume-weighted mean
    and stdev of DIFFphi, DIFFK, DIFFr, ricci and the volume average, against
    the reference's own functions (STATS row of the fixture)."""
    inp, _, ref, meta = load_golden(name)
    got = oracle.field_statistics(inp, meta["order"], **meta["config"])
    rel = np.abs(got - ref["STATS"]) / np.abs(ref["STATS"])
    assert rel.max() < 1e-12, (got, ref["STATS"])


def test_frw_known_answer():
    """tests/reference_frw.cc:1-52: four fluids, H0 = 2.89440502, dt = 0.01;
    the Friedmann residual K^2 - 24 pi rho stays below dt^2."""
    H0 = 2.89440502
    fluids = [(0.25, 0.0), (0.25, 1.0 / 3.0), (0.25, -1.0), (0.25, -0.5)]
    st = oracle.frw_evolve(0.0, -3.0 * H0, fluids, 0.01, 100)
    K, rho = st[1], st[2:].sum()
    resid = K * K - 24.0 * math.pi * rho
    assert abs(resid) < 0.01 ** 2
    assert st[0] > 0.0  # phi grows as the box expands


def test_rk4_known_answer_uniform_vacuum():
    """tests/rk4.cc idea on the register update: a uniform vacuum box reduces to
    ODEs (dK/dt = alpha K^2/3, dalpha/dt = -alpha K, dphi/dt = -alpha K/6 for
    the harmonic lapse); the restatement must equal a scalar RK4 of them."""
    from cosmograph_b200 import ics, state as S
    st = ics.perturbed((6, 6, 6), S.VACUUM, amp=0.0)
    st.fields[S.BSSN_FIELDS.index("DIFFK")] = -0.3
    st.dt = 0.05
    steps = 40
    got = oracle.evolve(st, steps, 4, lapse="Harmonic")
    y = np.array([0.0, -0.3, 0.0])  # phi, K, DIFFalpha

    def f(y):
        al = y[2] + 1.0
        return np.array([-1.0 / 6.0 * (al * y[1]), al * (1.0 / 3.0 * y[1] * (y[1] + 2.0 * 0.0) + 0.0), -1.0 * al * y[1]])

    dt = st.dt
    for _ in range(steps):
        k1 = f(y); k2 = f(y + dt * k1 / 2.0); k3 = f(y + dt * k2 / 2.0); k4 = f(y + dt * k3)
        y = dt * k1 / 6.0 + dt * k2 / 3.0 + dt * k3 / 3.0 + (dt * k4 / 6.0 + y)
    for f_, v in zip(("DIFFphi", "DIFFK", "DIFFalpha"), y):
        arr = got.field(f_)
        assert np.ptp(arr) == 0.0
        # stencils of a uniform field leave ulp-level residues (e.g. 1/12 - 2/3
        # + 2/3 - 1/12 of a constant), so the grid is an ODE only to ~1e-15/step
        assert abs(arr.flat[0] - v) <= 1e-13 * max(1.0, abs(v)), (f_, arr.flat[0], v)


def test_restatement_conserves_dust_mass():
    """sum D over the periodic grid is conserved by the flux-divergence form
    (the property the GPU full-size test checks at 256^3)."""
    from cosmograph_b200 import ics, state as S

    st = ics.perturbed((12, 10, 8), S.DUST, seed=6, amp=2e-2)
    d = st.names.index("D")
    out = oracle.evolve(st, 3, 4, lapse="Harmonic")
    assert not np.array_equal(out.fields[d], st.fields[d])
    assert abs(out.fields[d].sum() - st.fields[d].sum()) / st.fields[d].sum() < 1e-14
