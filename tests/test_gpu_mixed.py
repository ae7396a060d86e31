"""The FP32-mixed substep kernel against the FP64 GPU path.

Two measures of accuracy:

* against the run's perturbation amplitude (the bound the design targets,
  1e-6): the amplitude is the rms of the perturbation the initial data are
  built from -- the density contrast delta of the dust runs (rms 1e-4), the
  scalar-field fluctuation delta phi of the scalar runs (rms 1e-5).  The
  mixed run's error in that quantity (max over the box of
  |D_mixed - D_fp64| / mean(D), or |phi_mixed - phi_fp64|) must stay below
  1e-6 of it, and its Hamiltonian and momentum constraint norms within 2x
  of the FP64 run's;
* per field, against the field's own spread about its mean,
  max|mixed - fp64| / max|fp64 - mean(fp64)| (fields whose perturbation
  vanishes identically are skipped).  This is the stricter measure for the
  metric components, whose spread is small: their FP32 right-hand sides
  carry a rounding error of a few 2^-24 per substep, which accumulates as a
  random walk (about 2^-24 sqrt(substeps) relative); the bounds below are
  that estimate with a margin (measured: 2.8e-7 after 13 steps at 256^3,
  1.4e-6 after 100 and 1.6e-5 after 500 steps at 128^3).
"""
import numpy as np
import pytest

from cosmograph_b200 import ics, state as S
from cosmograph_b200.evolution import BoxConfig, Evolution, evolve

pytestmark = pytest.mark.gpu


def perturbation_errors(got, ref, names):
    out = {}
    for f, n in enumerate(names):
        spread = float(np.abs(ref[f] - ref[f].mean()).max())
        if spread == 0.0:
            continue
        out[n] = float(np.abs(got[f] - ref[f]).max()) / spread
    return out


def test_uniform_box_follows_the_background():
    st = ics.perturbed((16, 16, 16), S.DUST, amp=0.0)
    a = evolve(st, 20, BoxConfig(order=8, precision="mixed"))
    b = evolve(st, 20, BoxConfig(order=8, precision="fp64"))
    for f in range(a.fields.shape[0]):
        assert np.ptp(a.fields[f]) == 0.0
    # the background is integrated on the host, the FP64 path on the grid:
    # agreement to roundoff on the scale max(1, |field|)
    scale = np.maximum(np.abs(b.fields).max(axis=(1, 2, 3)), 1.0)
    assert (np.abs(a.fields - b.fields).max(axis=(1, 2, 3)) / scale).max() < 1e-13


@pytest.mark.parametrize("order,steps", [(4, 60), (8, 40)])
def test_grf_dust_against_fp64(order, steps):
    st = ics.grf_dust(32, seed=11, rms_delta=1e-4, order=order)
    a = evolve(st, steps, BoxConfig(order=order, precision="mixed"))
    b = evolve(st, steps, BoxConfig(order=order, precision="fp64"))
    errs = perturbation_errors(a.fields, b.fields, st.names)
    worst = max(errs, key=errs.get)
    D = b.field("D")
    delta_err = float(np.abs(a.field("D") - D).max() / D.mean())
    print("mixed vs fp64, worst field", worst, errs[worst], "density-contrast error / amplitude", delta_err / 1e-4)
    assert delta_err <= 1e-6 * 1e-4  # 1e-6 of the density-contrast amplitude
    assert errs[worst] < 1e-5, errs


def test_hamiltonian_constraint_no_worse_than_twice_fp64():
    st = ics.grf_dust(32, seed=12, rms_delta=1e-4, order=4)
    res = {}
    for prec in ("fp64", "mixed"):
        with Evolution(st, BoxConfig(order=4, precision=prec)) as ev:
            ev.step(40)
            res[prec] = ev.constraints(0)
    h64, hmx = res["fp64"]["H"][7], res["mixed"]["H"][7]
    print("H L2: fp64", h64, "mixed", hmx)
    assert hmx <= 2.0 * h64


def test_vacuum_mixed_runs_and_rejects_unsupported():
    st = ics.perturbed((16, 16, 16), S.VACUUM, amp=1e-3)
    a = evolve(st, 5, BoxConfig(order=4, precision="mixed"))
    b = evolve(st, 5, BoxConfig(order=4, precision="fp64"))
    errs = perturbation_errors(a.fields, b.fields, st.names)
    print("vacuum mixed vs fp64, worst", max(errs.values()))
    assert max(errs.values()) < 1e-5
    with pytest.raises(RuntimeError, match="Z4c"):
        evolve(ics.perturbed((16, 16, 16), S.DUST, z4c=True), 1, BoxConfig(order=4, precision="mixed"))
    dust = ics.perturbed((16, 16, 16), S.DUST)
    dust.frw_K = -0.5
    with pytest.raises(RuntimeError, match="trivial FRW"):
        evolve(dust, 1, BoxConfig(order=4, precision="mixed"))


# every lapse gauge but the harmonic one (covered above), with its parameters
LAPSES = [
    ("Static", {}), ("ConformalFLRW", {}), ("ConformalSync", {}), ("Anharmonic", {}),
    ("OnePlusLog", {"gd_c": 0.7}), ("AwAGaugeWave", {}), ("AwAShiftedWave", {}),
    ("DampedWave", {"dw_mu_l": 0.3, "dw_p": 0.5}),
]


@pytest.mark.parametrize("lapse,extra", LAPSES, ids=[n for n, _ in LAPSES])
def test_lapse_gauges_against_fp64(lapse, extra):
    """GRF dust (rms delta 1e-4) with a lapse perturbation, 30 steps at
    order 4: the mixed form against the FP64 GPU run, density-contrast error
    below 1e-6 of the amplitude and every field within 1e-5 of its spread.
    The K_avg lapses take the conformal average of the perturbation from a
    reduction of the FP32 inputs each substep."""
    st = ics.grf_dust(32, seed=21, rms_delta=1e-4, order=4)
    f = st.names.index("DIFFalpha")
    # a smooth lapse perturbation of its own (grid-scale noise would grow
    # exponentially under the anharmonic lapse, dalpha/dt = +alpha^2 (K - K_avg))
    x = np.arange(32) / 32.0
    st.fields[f] += 1e-5 * (np.sin(2 * np.pi * x)[:, None, None] * np.cos(4 * np.pi * x)[None, :, None] +
                            np.sin(2 * np.pi * x + 1.0)[None, None, :])
    a = evolve(st, 30, BoxConfig(order=4, precision="mixed", lapse=lapse, **extra))
    b = evolve(st, 30, BoxConfig(order=4, precision="fp64", lapse=lapse, **extra))
    errs = perturbation_errors(a.fields, b.fields, st.names)
    worst = max(errs, key=errs.get)
    D = b.field("D")
    delta_err = float(np.abs(a.field("D") - D).max() / D.mean())
    print("mixed vs fp64", lapse, "worst field", worst, errs[worst], "delta error / amplitude", delta_err / 1e-4)
    assert delta_err <= 1e-6 * 1e-4
    assert errs[worst] < 1e-5, errs


@pytest.mark.parametrize("matter", [S.DUST, S.SCALAR])
def test_constraint_damping_against_fp64(matter):
    """a_adj_amp and k_damping_amp (the Hamiltonian-constraint terms of the
    gamma, A, phi and K equations, bssn.cc:748-820): the mixed form takes H in
    perturbation form about the background's own constraint, which the host
    adds to the background's phi and K.  Against the FP64 run: every field
    within 1e-5 of its spread, and the damping visibly at work."""
    # smooth perturbations of every field (amplitude 1e-4) about a background
    # that satisfies its own constraint: H is of the perturbations' order
    st = ics.perturbed((24, 20, 28), matter, seed=25, amp=1e-4)
    kw = {"potential": "quadratic", "pot_mass": 1.0} if matter == S.SCALAR else {}
    damp = dict(a_adj_amp=0.5, k_damping_amp=0.5, **kw)
    a = evolve(st, 30, BoxConfig(order=4, precision="mixed", **damp))
    b = evolve(st, 30, BoxConfig(order=4, precision="fp64", **damp))
    c = evolve(st, 30, BoxConfig(order=4, precision="fp64", **kw))
    errs = perturbation_errors(a.fields, b.fields, st.names)
    effect = perturbation_errors(c.fields, b.fields, st.names)
    worst = max(errs, key=errs.get)
    print("damping mixed vs fp64", matter, worst, errs[worst], "effect", max(effect.values()))
    assert errs[worst] < 1e-5, errs
    assert max(effect.values()) > 100 * errs[worst]


@pytest.mark.parametrize("order", [2, 8])
def test_kreiss_oliger_against_fp64(order):
    """Kreiss-Oliger dissipation (coefficient 0.3, orders 2 and 8) on a
    perturbed dust box with grid-scale noise, which the dissipation damps:
    mixed against FP64, every field within 1e-5 of its spread, and the
    dissipation visibly at work (the run without it differs by far more)."""
    st = ics.perturbed((24, 20, 28), S.DUST, seed=31, amp=1e-4)
    # grid-scale noise in Gamma^1, which the dissipation damps at any order
    st.fields[st.names.index("Gamma1")] += 1e-5 * np.random.default_rng(7).standard_normal(st.shape)
    cfg = dict(order=order, ko_coeff=0.3)
    a = evolve(st, 20, BoxConfig(precision="mixed", **cfg))
    b = evolve(st, 20, BoxConfig(precision="fp64", **cfg))
    c = evolve(st, 20, BoxConfig(precision="fp64", order=order))
    errs = perturbation_errors(a.fields, b.fields, st.names)
    effect = perturbation_errors(c.fields, b.fields, st.names)
    worst = max(errs, key=errs.get)
    print("KO mixed vs fp64", order, worst, errs[worst], "effect of the dissipation", max(effect.values()))
    assert errs[worst] < 1e-5, errs
    assert max(effect.values()) > 100 * errs[worst]


@pytest.mark.parametrize("order,potential", [(4, "const"), (8, "quadratic")])
def test_grf_scalar_against_fp64(order, potential):
    """BSSN + scalar field, phi_0 = 1e-2 with a k^-3 Gaussian random
    fluctuation of rms 1e-5: mixed vs FP64 fields and Hamiltonian constraint."""
    st = ics.grf_scalar(32, seed=14, phi0=1e-2, rms=1e-5, order=order)
    cfgs = {p: BoxConfig(order=order, precision=p, potential=potential, pot_mass=1.0) for p in ("fp64", "mixed")}
    res = {}
    for prec, cfg in cfgs.items():
        with Evolution(st, cfg) as ev:
            ev.step(30)
            res[prec] = (ev.download(0), ev.constraints(0))
    errs = perturbation_errors(res["mixed"][0].fields, res["fp64"][0].fields, st.names)
    worst = max(errs, key=errs.get)
    f = st.names.index("phi")
    phi_err = float(np.abs(res["mixed"][0].fields[f] - res["fp64"][0].fields[f]).max()) / 1e-5
    print("scalar mixed vs fp64", order, potential, worst, errs[worst], "phi error / fluctuation rms", phi_err,
          "H", res["mixed"][1]["H"][7], res["fp64"][1]["H"][7])
    assert phi_err < 1e-6  # 1e-6 of the fluctuation amplitude
    assert res["mixed"][1]["H"][7] <= 2.0 * res["fp64"][1]["H"][7]
    assert errs[worst] < 2e-5, errs


def test_a_register_of_a_mixed_box():
    st = ics.grf_dust(32, seed=13, rms_delta=1e-4, order=4)
    with Evolution(st, BoxConfig(order=4, precision="mixed")) as em, \
            Evolution(st, BoxConfig(order=4, precision="fp64")) as ef:
        for ev in (em, ef):
            ev.step(2)
            ev.step_init()
            ev.rk_stage(1)
        for f, name in enumerate(st.names):
            a = em.download_field(0, f, "a")
            b = ef.download_field(0, f, "a")
            spread = np.abs(b - b.mean()).max()
            if spread > 0:
                assert np.abs(a - b).max() <= 1e-5 * spread, name
        with pytest.raises(RuntimeError, match="read-only"):
            em.upload_field(0, 0, "a", np.zeros(st.shape))


def test_grf_dust_128_order8_500_steps():
    """128^3, 8th order, GRF dust at rms delta 1e-4, 500 RK4 steps: the mixed
    form against the FP64 GPU run.  Field errors relative to each field's
    spread (printed with the density-contrast amplitude) and the Hamiltonian
    and momentum constraint norms."""
    st = ics.grf_dust(128, seed=17, rms_delta=1e-4, order=8)
    res = {}
    for prec in ("fp64", "mixed"):
        with Evolution(st, BoxConfig(order=8, precision=prec)) as ev:
            ev.step(500)
            ev.synchronize()
            res[prec] = (ev.download(0), ev.constraints(0))
    ref, got = res["fp64"][0], res["mixed"][0]
    errs = perturbation_errors(got.fields, ref.fields, st.names)
    worst = max(errs, key=errs.get)
    D = ref.field("D")
    delta_err = float(np.abs(got.field("D") - D).max() / D.mean())
    h64, hmx = res["fp64"][1]["H"][7], res["mixed"][1]["H"][7]
    m64, mmx = res["fp64"][1]["M"][7], res["mixed"][1]["M"][7]
    print("128^3 o8 500 steps: worst field", worst, errs[worst], "density-contrast error", delta_err,
          "H L2", hmx, h64, "M L2", mmx, m64)
    assert delta_err <= 1e-6 * 1e-4  # 1e-6 of the density-contrast amplitude
    assert hmx <= 2.0 * h64 and mmx <= 2.0 * m64
    assert errs[worst] < 5e-5, errs  # FP32 rounding over 2000 substeps (module docstring)



def test_grf_scalar_256_order8_200_steps():
    """256^3, 8th order, BSSN + scalar field with V = m^2 phi^2 / 2 (m = 1),
    phi_0 = 1e-2 plus a k^-3 random fluctuation of rms 1e-5, 200 RK4 steps:
    the mixed form against the FP64 run.  The scalar field's error is stated
    against the fluctuation amplitude; every field against its spread; the
    Hamiltonian constraint norm no worse than twice FP64's."""
    st = ics.grf_scalar(256, seed=4, phi0=1e-2, rms=1e-5, order=8)
    res = {}
    for prec in ("fp64", "mixed"):
        cfg = BoxConfig(order=8, precision=prec, potential="quadratic", pot_mass=1.0)
        with Evolution(st, cfg) as ev:
            ev.step(200)
            ev.synchronize()
            res[prec] = (ev.download(0), ev.constraints(0))
    ref, got = res["fp64"][0], res["mixed"][0]
    errs = perturbation_errors(got.fields, ref.fields, st.names)
    worst = max(errs, key=errs.get)
    f = st.names.index("phi")
    phi_err = float(np.abs(got.fields[f] - ref.fields[f]).max()) / 1e-5
    h64, hmx = res["fp64"][1]["H"][7], res["mixed"][1]["H"][7]
    print("256^3 scalar o8 200 steps: worst field", worst, errs[worst], "phi error / fluctuation rms", phi_err,
          "H L2", hmx, h64)
    assert phi_err < 1e-6  # 1e-6 of the fluctuation amplitude
    assert hmx <= 2.0 * h64
    assert errs[worst] < 5e-5, errs  # FP32 rounding over 800 substeps (module docstring)
