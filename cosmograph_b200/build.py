"""Build the CUDA library in-tree: cosmograph_b200/libcosmograph_b200.so, and
the config-file driver cosmograph_b200/cosmo_b200 (C++ facade, g++).

Every kernel is compiled for sm_100a only.  The substep kernels are compiled
twice from the same source: without FMA contraction (the FP64 parity build)
and with it.  Objects are cached under cosmograph_b200/_build/ and rebuilt
when a source or header is newer than the object.

Usage: python -m cosmograph_b200.build [--force] [--verbose]
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libcosmograph_b200.so"
INCLUDE = ROOT / "include"
HOST = PKG / "host"
DRIVER = PKG / "cosmo_b200"   # config-file driver (C++ facade over the C ABI)

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", *ARCH, f"-I{INCLUDE}", f"-I{CSRC}"]

# (object name, source, extra flags)
UNITS = [
    ("stage_exact.o", "cg_stage_inst.cu", ["--fmad=false", "-DCG_VARIANT_NS=exact", "-DCG_REFERENCE_ORDER=1"]),
    ("stage_fast.o", "cg_stage_inst.cu", ["--fmad=true", "-DCG_VARIANT_NS=fast"]),
    ("stage_exact_z4c.o", "cg_stage_inst.cu",
     ["--fmad=false", "-DCG_VARIANT_NS=exact", "-DCG_REFERENCE_ORDER=1", "-DCG_Z4C_UNIT=1"]),
    ("stage_fast_z4c.o", "cg_stage_inst.cu", ["--fmad=true", "-DCG_VARIANT_NS=fast", "-DCG_Z4C_UNIT=1"]),
    ("stage_exact_shift.o", "cg_stage_inst.cu",
     ["--fmad=false", "-DCG_VARIANT_NS=exact", "-DCG_REFERENCE_ORDER=1", "-DCG_SHIFT_UNIT=1"]),
    ("abi.o", "cg_abi.cu", []),
    ("noalloc.o", "cg_noalloc.cu", []),
    ("peak.o", "cg_peak.cu", []),
    ("mixed.o", "cg_mixed_inst.cu", []),
    ("ics.o", "cg_ics.cu", []),
    ("tma_host.o", "cg_tma_host.cu", []),
]


def _deps() -> list[Path]:
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + \
        sorted(INCLUDE.glob("*.h")) + [Path(__file__)]


def build(force: bool = False, verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    newest = max(p.stat().st_mtime for p in _deps())
    objs = []
    jobs = []
    for obj, src, flags in UNITS:
        o = BUILD / obj
        objs.append(o)
        if force or not o.exists() or o.stat().st_mtime < newest:
            cmd = [NVCC, *COMMON, *flags, "-c", str(CSRC / src), "-o", str(o)]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
            jobs.append(cmd)

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        if verbose:
            sys.stderr.write(r.stderr)

    if jobs:
        with ThreadPoolExecutor(max_workers=len(jobs)) as ex:
            list(ex.map(run, jobs))
    if force or jobs or not LIB.exists() or LIB.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        tmp = LIB.with_suffix(".so.tmp")
        run([NVCC, *ARCH, "-shared", "-Xcompiler", "-fPIC", *map(str, objs), "-lcufft", "-o", str(tmp)])
        os.replace(tmp, LIB)
    build_driver(force)
    return LIB


def build_driver(force: bool = False) -> Path:
    """g++ build of the C++ facade (BSSN, Dust, Scalar, Lambda, sims) and the
    config-file driver `cosmo_b200`, linked against the CUDA library."""
    srcs = sorted(HOST.glob("*.cc"))
    deps = srcs + sorted(HOST.glob("*.hpp")) + [INCLUDE / "cosmograph_b200.h", LIB, Path(__file__)]
    if not force and DRIVER.exists() and DRIVER.stat().st_mtime >= max(p.stat().st_mtime for p in deps):
        return DRIVER
    tmp = DRIVER.with_suffix(".tmp")
    cmd = [os.environ.get("CXX", "g++"), "-std=c++17", "-O2", "-Wall", "-Wextra", f"-I{INCLUDE}", f"-I{HOST}",
           *map(str, srcs), f"-L{PKG}", "-lcosmograph_b200", "-lz", "-Wl,-rpath,$ORIGIN", "-o", str(tmp)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"g++ failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, DRIVER)
    return DRIVER


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args(argv)
    print(build(force=a.force, verbose=a.verbose))
    return 0


if __name__ == "__main__":
    sys.exit(main())
