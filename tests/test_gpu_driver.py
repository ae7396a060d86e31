"""The config-file driver (C++ facade over the C ABI) on the GPU.

A dust run of `steps = S` performs S + 1 RK4 steps (sims/sim.cc:103-122 loops
step = 0..num_steps).  Its final state must equal the Python front end's
evolution of the same initial data bit for bit (same kernels, same substep
sequence), and its constraint time series must hold the statistics of the
states at the output steps.
"""
import gzip
import subprocess

import numpy as np
import pytest

from cosmograph_b200 import build, ics, snapshots, state as S
from cosmograph_b200.evolution import BoxConfig, Evolution, evolve

pytestmark = pytest.mark.gpu


def run_driver(tmp_path, text):
    build.build()
    (tmp_path / "config.txt").write_text(text)
    r = subprocess.run([str(build.DRIVER), "config.txt"], capture_output=True, text=True, cwd=tmp_path,
                       timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return r


def rows(path):
    with gzip.open(path, "rt") as fh:
        return [[float(x) for x in line.split()] for line in fh.read().strip().splitlines()]


def test_dust_run_matches_python_front_end(tmp_path):
    st = ics.grf_dust(32, seed=21, rms_delta=1e-4, order=4)
    st.save(tmp_path / "ic.bin")
    run_driver(tmp_path, "\n".join([
        "simulation_type = dust", "steps = 9", "stencil_order = 4", "lapse = Harmonic",
        "ic_file = ic.bin", "output_file = final.bin", "output_dir = out", "dump_file = calculated",
        "IO_constraint_interval = 5", "IO_bssnstats_interval = 5", ""]))
    got = S.load(tmp_path / "final.bin")
    ref = evolve(st, 10, BoxConfig(order=4, lapse="Harmonic"))
    assert got.step == 10
    assert np.array_equal(got.fields, ref.fields)
    assert got.frw_phi == ref.frw_phi and got.frw_K == ref.frw_K

    h = rows(tmp_path / "out" / "H_violations.dat.gz")
    m = rows(tmp_path / "out" / "M_violations.dat.gz")
    fs = rows(tmp_path / "out" / "calculated.dat.gz")
    assert len(h) == 2 and len(m) == 2 and all(len(r) == 5 for r in h)
    assert len(fs) == 2 and all(len(r) == 9 for r in fs)
    with Evolution(st, BoxConfig(order=4, lapse="Harmonic")) as ev:
        for row_h, row_m, row_s, steps in zip(h, m, fs, (0, 5)):
            if steps:
                ev.step(steps)
            c = ev.constraints(0)
            want_h = [c["H"][4], c["H"][5], c["H"][6], c["H"][2], c["H"][7]]
            want_m = [c["M"][4], c["M"][5], c["M"][6], c["M"][2], c["M"][7]]
            np.testing.assert_allclose(row_h, want_h, rtol=1e-14, atol=0)
            np.testing.assert_allclose(row_m, want_m, rtol=1e-14, atol=0)
            np.testing.assert_allclose(row_s, ev.field_statistics(0), rtol=1e-14, atol=0)
    frw = rows(tmp_path / "out" / "calculated.frwdat.gz")
    assert len(frw) == 2 and frw[0][0] == st.frw_phi
    log = (tmp_path / "out" / "log.txt").read_text()
    assert "Max. (Normed) Hamiltonian constraint violation" in log


def test_scalar_and_vacuum_runs(tmp_path):
    for sim, st in (("scalar", ics.grf_scalar(16, seed=3, order=4)),
                    ("vacuum", ics.perturbed((16, 16, 16), S.VACUUM, amp=1e-3))):
        d = tmp_path / sim
        d.mkdir()
        st.save(d / "ic.bin")
        run_driver(d, "\n".join([
            f"simulation_type = {sim}", "steps = 2", "stencil_order = 4", "lapse = Harmonic",
            "ic_file = ic.bin", "output_file = final.bin", "output_dir = out", ""]))
        got = S.load(d / "final.bin")
        ref = evolve(st, 3, BoxConfig(order=4, lapse="Harmonic"))
        assert np.array_equal(got.fields, ref.fields), sim


def test_mixed_dust_run(tmp_path):
    st = ics.grf_dust(32, seed=22, rms_delta=1e-4, order=4)
    st.save(tmp_path / "ic.bin")
    run_driver(tmp_path, "\n".join([
        "simulation_type = dust", "steps = 9", "stencil_order = 4", "lapse = Harmonic", "precision = mixed",
        "ic_file = ic.bin", "output_file = final.bin", "output_dir = out", ""]))
    got = S.load(tmp_path / "final.bin")
    ref = evolve(st, 10, BoxConfig(order=4, lapse="Harmonic"))
    for f in range(ref.fields.shape[0]):
        spread = np.abs(ref.fields[f] - ref.fields[f].mean()).max()
        if spread > 0:
            assert np.abs(got.fields[f] - ref.fields[f]).max() <= 1e-5 * spread, ref.names[f]


def test_nan_stops_the_run_with_code_10(tmp_path):
    st = ics.perturbed((16, 16, 16), S.VACUUM, amp=1e-3)
    st.field("DIFFphi")[3, 4, 5] = np.nan
    st.save(tmp_path / "ic.bin")
    (tmp_path / "config.txt").write_text("\n".join([
        "simulation_type = vacuum", "steps = 3", "stencil_order = 4", "lapse = Harmonic",
        "ic_file = ic.bin", "output_dir = out", ""]))
    r = subprocess.run([str(build.DRIVER), "config.txt"], capture_output=True, text=True, cwd=tmp_path,
                       timeout=600)
    assert r.returncode == 10, r.stdout[-1000:] + r.stderr[-1000:]
    assert "NAN detected" in (tmp_path / "out" / "log.txt").read_text()


def test_dust_run_with_gpu_initial_data(tmp_path):
    """Without ic_file the dust driver builds GRF initial data on the GPU
    (the reference's DustSim::setICs path) and evolves them."""
    run_driver(tmp_path, "\n".join([
        "simulation_type = dust", "steps = 4", "N = 32", "stencil_order = 4", "lapse = Harmonic",
        "seed = 11", "rms_delta = 1e-4", "Omega_L = 1e-6", "output_file = final.bin", "output_dir = out",
        "IO_constraint_interval = 1", ""]))
    got = S.load(tmp_path / "final.bin")
    ic = ics.grf_dust_gpu(32, seed=11, rms_delta=1e-4, order=4)
    ic.dx, ic.dt = got.dx, got.dt  # H_LEN_FRAC default 0.5: dx = 0.5/32
    assert got.step == 5 and np.isfinite(got.fields).all()
    h = rows(tmp_path / "out" / "H_violations.dat.gz")
    assert len(h) == 5 and all(np.isfinite(r).all() for r in h)


def test_scalar_run_with_gpu_initial_data(tmp_path):
    """Without ic_file the scalar driver builds the GRF scalar data on the GPU
    (cg_ic_grf_scalar) and evolves them: the same as the Python front end's
    run of the same GPU initial data, bit for bit."""
    run_driver(tmp_path, "\n".join([
        "simulation_type = scalar", "steps = 2", "N = 24", "stencil_order = 4", "lapse = Harmonic",
        "H_LEN_FRAC = 1", "potential = quadratic", "scalar_mass = 1.0", "seed = 12", "scalar_phi0 = 0.01",
        "scalar_rms = 1e-5", "output_file = final.bin", "output_dir = out", ""]))
    got = S.load(tmp_path / "final.bin")
    ic = ics.grf_scalar_gpu(24, seed=12, phi0=0.01, rms=1e-5, mass=1.0, order=4)
    ic.dx, ic.dt = got.dx, got.dt
    ref = evolve(ic, 3, BoxConfig(order=4, lapse="Harmonic", potential="quadratic", pot_mass=1.0))
    assert got.step == 3
    assert np.array_equal(got.fields, ref.fields)


def test_field_snapshots(tmp_path):
    """IO_3D / IO_2D / IO_1D keys (the reference's io_bssn_fields_snapshot) for
    the _a register after stepInit at the output steps."""
    st = ics.grf_dust(16, seed=23, rms_delta=1e-4, order=4)
    st.save(tmp_path / "ic.bin")
    run_driver(tmp_path, "\n".join([
        "simulation_type = dust", "steps = 2", "stencil_order = 4", "lapse = Harmonic", "ic_file = ic.bin",
        "output_dir = out", "IO_3D_grid_interval = 2", "IO_3D_DIFFphi_a = 1", "IO_2D_grid_interval = 2",
        "IO_2D_D_a = 1", "IO_1D_grid_interval = 1", "IO_1D_DIFFK_a = 1", "IO_1D_DIFFK_a_axis = 3",
        "IO_1D_DIFFK_a_xoffset = 2", "IO_1D_DIFFK_a_yoffset = 5", ""]))
    out = tmp_path / "out"
    phi0 = np.frombuffer(gzip.open(out / "3D_DIFFphi_a0.3d_grid.f64.gz").read(), dtype="<f8").reshape(16, 16, 16)
    assert np.array_equal(phi0, st.field("DIFFphi"))
    D0 = np.frombuffer(gzip.open(out / "2D_D_a0.2d_grid.f64.gz").read(), dtype="<f8").reshape(16, 16)
    assert np.array_equal(D0, st.field("D")[0])
    with np.load(snapshots.convert(out / "3D_DIFFphi_a0.3d_grid.f64.gz", 16, 16, 16)) as z:
        assert np.array_equal(z["DS1"], phi0)
    assert (out / "3D_DIFFphi_a2.3d_grid.f64.gz").exists() and not (out / "3D_DIFFphi_a1.3d_grid.f64.gz").exists()
    strip = rows(out / "1D_DIFFK_a.strip.dat.gz")
    assert len(strip) == 3 and len(strip[0]) == 16
    np.testing.assert_allclose(strip[0], st.field("DIFFK")[2, 5, :], rtol=1e-14)
