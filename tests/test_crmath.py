"""The correctly rounded exp, expm1 and log1p of the FP64 parity build
(cosmograph_b200/csrc/cg_crmath.h).

CPU: the header compiled for the host against 113-bit quad-precision
evaluations rounded once (libquadmath), on random arguments over each
function's range, small and tiny magnitudes, and powers of two with their
neighbours (tests/cpp/crmath_check.cc): every result must be the correctly
rounded one.  GPU: the same header compiled for sm_100a must return the
host's bits on every argument.
"""
import ctypes
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
CSRC = ROOT / "cosmograph_b200" / "csrc"
CPP = Path(__file__).resolve().parent / "cpp"


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    if not shutil.which("g++"):
        pytest.skip("no host C++ compiler")
    exe = tmp_path_factory.mktemp("crm") / "crmath_check"
    subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", f"-I{CSRC}", str(CPP / "crmath_check.cc"),
                    "-lquadmath", "-o", str(exe)], check=True)
    return exe


@pytest.mark.parametrize("fn,lo,hi", [("exp", -745.2, 709.9), ("exp", -0.02, 0.02), ("expm1", -45.0, 709.9),
                                      ("expm1", -1e-3, 1e-3), ("log1p", -0.999, 1e6), ("log1p", -1e-3, 1e-3)])
def test_correctly_rounded_on_the_host(checker, fn, lo, hi):
    r = subprocess.run([str(checker), fn, "400000", "5", repr(lo), repr(hi)], capture_output=True, text=True)
    print(r.stdout.strip())
    assert r.returncode == 0, r.stdout + r.stderr
    assert "mismatches=0" in r.stdout


def _arguments(fn: str, n: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    if fn == "log1p":
        a = np.concatenate([rng.uniform(-0.999, 10.0, n // 3), rng.normal(0, 1e-4, n // 3),
                            rng.normal(0, 1e-13, n - 2 * (n // 3))])
    else:
        a = np.concatenate([rng.uniform(-745.0, 709.0, n // 3), rng.normal(0, 1e-2, n // 3),
                            rng.normal(0, 1e-4, n - 2 * (n // 3))])
    e = np.arange(1, 80, dtype=np.float64)
    return np.concatenate([a, 2.0 ** -e, -(2.0 ** -e), 3 * 2.0 ** -e])


@pytest.mark.gpu
@pytest.mark.parametrize("fn", ["exp", "expm1", "log1p"])
def test_device_matches_host_bit_for_bit(tmp_path, fn):
    lib = tmp_path / "libcrm_device.so"
    subprocess.run(["/usr/local/cuda/bin/nvcc", "-std=c++17", "-O3", "-gencode", "arch=compute_100a,code=sm_100a",
                    "--fmad=false", "-Xcompiler", "-fPIC,-ffp-contract=off", "-shared", f"-I{CSRC}",
                    str(CPP / "crmath_device.cu"), "-o", str(lib)], check=True)
    L = ctypes.CDLL(str(lib))
    dp = ctypes.POINTER(ctypes.c_double)
    L.crm_eval_device.argtypes = [ctypes.c_int, dp, dp, ctypes.c_size_t]
    L.crm_eval_host.argtypes = [ctypes.c_int, dp, dp, ctypes.c_size_t]
    k = ["exp", "expm1", "log1p"].index(fn)
    x = np.ascontiguousarray(_arguments(fn, 3_000_000, 9 + k))
    dev, host = np.empty_like(x), np.empty_like(x)
    assert L.crm_eval_device(k, x.ctypes.data_as(dp), dev.ctypes.data_as(dp), x.size) == 0
    L.crm_eval_host(k, x.ctypes.data_as(dp), host.ctypes.data_as(dp), x.size)
    same = (dev.view(np.int64) == host.view(np.int64)) | (np.isnan(dev) & np.isnan(host))
    assert same.all(), x[~same][:5]
