"""The C++ facade and the config-file driver, host side (no GPU call).

The facade (cosmograph_b200/host) keeps the reference's component API
(components/bssn/bssn.h, components/dust_fluid/dust.h, utils/ConfigParser.h,
sims/sim.h); these tests build a small C++ program against it and run the
driver's error paths, which all end before the box is created.
"""
import os
import subprocess
from pathlib import Path

import pytest

from cosmograph_b200 import build

ROOT = Path(__file__).resolve().parent.parent


@pytest.fixture(scope="module")
def driver():
    build.build()
    return build.DRIVER


def run(driver, args, cwd):
    return subprocess.run([str(driver), *args], capture_output=True, text=True, cwd=cwd, timeout=60)


def test_facade_checks(tmp_path):
    build.build()
    exe = tmp_path / "facade_checks"
    cmd = ["g++", "-std=c++17", "-O1", f"-I{build.INCLUDE}", f"-I{build.HOST}",
           str(ROOT / "tests" / "cpp" / "facade_checks.cc"), str(build.HOST / "facade.cc"),
           f"-L{build.PKG}", "-lcosmograph_b200", "-lz", f"-Wl,-rpath,{build.PKG}", "-o", str(exe)]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    r = subprocess.run([str(exe), str(tmp_path)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "facade checks: ok" in r.stdout


def test_driver_usage(driver, tmp_path):
    r = run(driver, [], tmp_path)
    assert r.returncode == 1
    assert "exactly one config filename" in r.stdout


def test_driver_missing_config(driver, tmp_path):
    r = run(driver, [str(tmp_path / "nope.txt")], tmp_path)
    assert r.returncode == 1
    assert "error opening" in r.stderr


def test_driver_unknown_simulation_type(driver, tmp_path):
    (tmp_path / "c.txt").write_text("steps = 3\nsimulation_type = sheets\n")
    r = run(driver, ["c.txt"], tmp_path)
    assert r.returncode == 2
    assert "Invalid simulation type" in r.stderr


def test_driver_required_steps(driver, tmp_path):
    (tmp_path / "c.txt").write_text(f"simulation_type = dust\noutput_dir = {tmp_path / 'out'}\n")
    r = run(driver, ["c.txt"], tmp_path)
    assert r.returncode == 1
    assert "param `steps` is required" in r.stderr
    assert (tmp_path / "out" / "log.txt").exists()


def test_driver_output_dir_not_overwritten(driver, tmp_path):
    out = tmp_path / "out"
    (tmp_path / "c.txt").write_text(f"simulation_type = vacuum\nsteps = 2\noutput_dir = {out}\n")
    for _ in range(2):
        r = run(driver, ["c.txt"], tmp_path)
        assert r.returncode == 1
        assert "set ic_file" in r.stderr
    assert (out / "log.txt").exists() and (tmp_path / "out.1" / "log.txt").exists()
