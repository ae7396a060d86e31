"""Build recipe for the reference-source oracle.  TEST INFRASTRUCTURE.

Compiles the reference's own hot-path sources, unmodified and where they lie
under the reference checkout, together with oracle/ref_driver.cc into one
binary per (grid size, stencil order, flavour).  The reference fixes the grid
size and stencil order at compile time (cosmo_macros.h:12-40), so every
(N, order) needs its own binary.  Outputs go to oracle/_ref/ only; they are
git-ignored but travel with the repository snapshot to the GPU machine, where
no reference checkout exists.

Flavours:
  strict : -O2 -ffp-contract=off          (parity oracle; no FMA contraction,
                                            no reassociation)
  strict_cr : strict, with the C library's exp, expm1 and log1p replaced by
           correctly rounded ones (cr_libm.c) at link time
  strict_z4c, strict_cr_z4c : the same with Z4c damping compiled in
           (-DUSE_Z4c_DAMPING=1, cosmo_macros.h:91-100)
  fast   : -O3 -ffast-math -march=x86-64-v3 (the reference's own optimisation
           flags, cmake/optimization.cmake:18, with a portable -march so the
           binary also runs on the GPU machine's host CPU; CPU-baseline timing)

Usage: python oracle/build_ref.py --grid 32 32 32 --order 4 --flavour strict
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
import tempfile
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
REF_ROOT = Path(os.environ.get("CG_REFERENCE_ROOT", "/root/reference"))
OUT_DIR = HERE / "_ref"

REF_SOURCES = [
    "components/bssn/bssn.cc",
    "components/bssn/BSSNGaugeHandler.cc",
    "components/dust_fluid/dust.cc",
    "components/scalar/scalar.cc",
    "components/static/static.cc",
    "components/Lambda/lambda.cc",
    "utils/ConfigParser.cc",
    "utils/Timer.cc",
]

FLAVOURS = {
    "strict": ["-O2", "-ffp-contract=off"],
    "strict_cr": ["-O2", "-ffp-contract=off"],
    "strict_z4c": ["-O2", "-ffp-contract=off", "-DUSE_Z4c_DAMPING=1"],
    "strict_cr_z4c": ["-O2", "-ffp-contract=off", "-DUSE_Z4c_DAMPING=1"],
    # the shift (beta^i, expN, upwinded advection) with the Gamma-driver's auxB^i
    "strict_shift": ["-O2", "-ffp-contract=off", "-DUSE_BSSN_SHIFT=1", "-DUSE_GAMMA_DRIVER=1"],
    "strict_cr_shift": ["-O2", "-ffp-contract=off", "-DUSE_BSSN_SHIFT=1", "-DUSE_GAMMA_DRIVER=1"],
    "fast": ["-O3", "-ffast-math", "-march=x86-64-v3"],
}
# strict_cr: the strict build linked with correctly rounded exp, expm1 and
# log1p (cr_libm.c, in place of the C library's) -- the reference as a
# correctly rounded C library runs it


def binary_name(nx: int, ny: int, nz: int, order: int, flavour: str) -> str:
    return f"cg_ref_{nx}x{ny}x{nz}_o{order}_{flavour}"


def binary_path(nx: int, ny: int, nz: int, order: int, flavour: str) -> Path:
    return OUT_DIR / binary_name(nx, ny, nz, order, flavour)


def reference_available() -> bool:
    return all((REF_ROOT / s).is_file() for s in REF_SOURCES)


def build(nx: int, ny: int, nz: int, order: int, flavour: str = "strict",
          force: bool = False) -> Path:
    """Compile one oracle binary; returns its path (skips if up to date)."""
    out = binary_path(nx, ny, nz, order, flavour)
    driver = HERE / "ref_driver.cc"
    newest = max(driver.stat().st_mtime, (HERE / "cr_libm.c").stat().st_mtime, (HERE / "cr_libm.h").stat().st_mtime)
    if out.exists() and not force and out.stat().st_mtime >= newest:
        return out
    if not reference_available():
        raise FileNotFoundError(f"reference sources not found under {REF_ROOT}")
    if order not in (2, 4, 6, 8):
        raise ValueError("stencil order must be 2, 4, 6 or 8")
    OUT_DIR.mkdir(parents=True, exist_ok=True)
    defs = [
        f"-DNX={nx}", f"-DNY={ny}", f"-DNZ={nz}", f"-DCOSMO_N={nx}",
        f"-DSTENCIL_ORDER={order}", "-DH_LEN_FRAC=1", "-DUSE_MULTIGRID=0",
        "-DUSE_COSMOTRACE=0",
    ]
    common = ["g++", "-std=c++11", "-fopenmp", "-w", *FLAVOURS[flavour], *defs,
              f"-I{HERE / 'stub'}", f"-I{HERE}", f"-I{REF_ROOT}"]
    with tempfile.TemporaryDirectory(prefix="cg_ref_build_") as tmp:
        srcs = [REF_ROOT / s for s in REF_SOURCES] + [driver]
        objs = [Path(tmp) / f"{i}.o" for i in range(len(srcs))]

        def cc(pair):
            src, obj = pair
            subprocess.run([*common, "-c", str(src), "-o", str(obj)], check=True)

        with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
            list(ex.map(cc, zip(srcs, objs)))
        libs = ["-lz"]
        if flavour.startswith("strict_cr"):
            crobj = Path(tmp) / "cr_libm.o"
            subprocess.run(["gcc", "-std=gnu11", "-O2", "-ffp-contract=off", f"-I{HERE}", "-c",
                            str(HERE / "cr_libm.c"), "-o", str(crobj)], check=True)
            objs.append(crobj)
            libs.append("-lquadmath")
        tmp_out = Path(tmp) / out.name
        subprocess.run([*common, *map(str, objs), *libs, "-o", str(tmp_out)], check=True)
        shutil.move(str(tmp_out), out)
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--grid", type=int, nargs=3, required=True, metavar=("NX", "NY", "NZ"))
    ap.add_argument("--order", type=int, required=True)
    ap.add_argument("--flavour", choices=sorted(FLAVOURS), default="strict")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args(argv)
    print(build(*a.grid, a.order, a.flavour, a.force))
    return 0


if __name__ == "__main__":
    sys.exit(main())
