"""Oracles for the BSSN(+dust/+scalar) RK4 evolution path.  TEST INFRASTRUCTURE.

Two CPU oracles live here; neither is part of the product:

* the C restatement (cg_oracle.c, run-time grid size and stencil order),
  loaded through ctypes from oracle/_build/libcg_oracle.so;
* the reference's own sources compiled per (N, order) by build_ref.py into
  oracle/_ref/, driven through ref_driver.cc on state files.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this package, as the checker or as the timed CPU baseline.
"""
from __future__ import annotations

import ctypes
import json
import os
import subprocess
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
BUILD_DIR = HERE / "_build"
LIB_PATH = BUILD_DIR / "libcg_oracle.so"
# the same restatement with correctly rounded exp, expm1, log1p (cr_libm.h)
LIB_CR_PATH = BUILD_DIR / "libcg_oracle_cr.so"

LAPSES = {
    "Static": 0, "Harmonic": 1, "ConformalFLRW": 2, "ConformalSync": 3,
    "Anharmonic": 4, "OnePlusLog": 5, "AwAGaugeWave": 6, "AwAShiftedWave": 7,
    "DampedWave": 8,
}
POTENTIALS = {"const": 0, "quadratic": 1}


class CgoParams(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("order", ctypes.c_int), ("matter", ctypes.c_int), ("lapse", ctypes.c_int),
        ("normalize_metric", ctypes.c_int), ("potential", ctypes.c_int),
        ("dx", ctypes.c_double), ("dt", ctypes.c_double), ("lam", ctypes.c_double),
        ("ko_coeff", ctypes.c_double), ("a_adj_amp", ctypes.c_double),
        ("k_damping_amp", ctypes.c_double), ("gd_c", ctypes.c_double),
        ("dw_mu_l", ctypes.c_double), ("dw_p", ctypes.c_double),
        ("pot_const", ctypes.c_double), ("pot_mass", ctypes.c_double),
        ("frw_phi", ctypes.c_double), ("frw_K", ctypes.c_double),
        ("nfluids", ctypes.c_int),
        ("fluid_rho", ctypes.c_double * 4), ("fluid_w", ctypes.c_double * 4),
        ("z4c", ctypes.c_int),
    ]


def build_lib(force: bool = False) -> Path:
    """Compile the C restatement (strict FP: no FMA contraction), with the C
    library's exp/expm1/log1p (libcg_oracle.so) and with correctly rounded
    ones (libcg_oracle_cr.so)."""
    src = HERE / "cg_oracle.c"
    hdr = HERE / "cg_oracle.h"
    newest = max(src.stat().st_mtime, hdr.stat().st_mtime, (HERE / "cr_libm.h").stat().st_mtime)
    BUILD_DIR.mkdir(exist_ok=True)
    for path, extra in ((LIB_PATH, []), (LIB_CR_PATH, ["-include", str(HERE / "cr_libm.h")])):
        if path.exists() and not force and path.stat().st_mtime >= newest:
            continue
        tmp = path.with_suffix(".so.tmp")
        subprocess.run(["gcc", "-std=gnu11", "-O2", "-ffp-contract=off", "-fopenmp", "-fPIC", *extra,
                        "-shared", "-o", str(tmp), str(src), "-lquadmath", "-lm"], check=True)
        os.replace(tmp, path)
    return LIB_PATH


_libs = {}


def lib(cr: bool = False) -> ctypes.CDLL:
    """The restatement; cr=True: with correctly rounded exp, expm1, log1p."""
    if cr not in _libs:
        build_lib()  # no-op when the libraries are newer than their sources
        L = ctypes.CDLL(str(LIB_CR_PATH if cr else LIB_PATH))
        dp = ctypes.POINTER(ctypes.c_double)
        L.cgo_evolve.argtypes = [ctypes.POINTER(CgoParams), dp, ctypes.c_int, dp]
        L.cgo_rhs.argtypes = [ctypes.POINTER(CgoParams), dp, dp]
        L.cgo_constraints.argtypes = [ctypes.POINTER(CgoParams), dp, dp, dp, dp, dp, dp]
        L.cgo_field_statistics.argtypes = [ctypes.POINTER(CgoParams), dp, dp]
        L.cgo_frw_evolve.argtypes = [dp, dp, ctypes.c_int, ctypes.c_double, ctypes.c_int]
        L.cgo_frw_evolve.restype = None
        L.cgo_set_threads.argtypes = [ctypes.c_int]
        L.cgo_set_threads.restype = None
        _libs[cr] = L
    return _libs[cr]


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def make_params(state, order: int, lapse: str = "Harmonic", normalize_metric: int = 1,
                potential: str = "const", pot_const: float = 3.0e-4, pot_mass: float = 1.0,
                ko_coeff: float = 0.0, a_adj_amp: float = 0.0, k_damping_amp: float = 0.0,
                gd_c: float = 1.0, dw_mu_l: float = 0.0, dw_p: float = 0.0) -> CgoParams:
    if getattr(state, "shift", False):
        raise ValueError("the restatement has no shift: shift runs are checked against the reference build (oracle/_ref)")
    nx, ny, nz = state.shape
    p = CgoParams()
    p.nx, p.ny, p.nz = nx, ny, nz
    p.order, p.matter, p.lapse = order, state.matter, LAPSES[lapse]
    p.normalize_metric, p.potential = normalize_metric, POTENTIALS[potential]
    p.dx, p.dt, p.lam = state.dx, state.dt, state.lam
    p.ko_coeff, p.a_adj_amp, p.k_damping_amp = ko_coeff, a_adj_amp, k_damping_amp
    p.gd_c, p.dw_mu_l, p.dw_p = gd_c, dw_mu_l, dw_p
    p.pot_const, p.pot_mass = pot_const, pot_mass
    p.frw_phi, p.frw_K = state.frw_phi, state.frw_K
    p.nfluids = len(state.fluids)
    for i, (rho, w) in enumerate(state.fluids):
        p.fluid_rho[i], p.fluid_w[i] = rho, w
    p.z4c = 1 if getattr(state, "z4c", False) else 0
    return p


def evolve(state, steps: int, order: int, threads: int = 0, cr: bool = False, **kw):
    """Run the C restatement for `steps` RK4 steps; returns a new state.
    cr=True: with correctly rounded exp, expm1 and log1p."""
    L = lib(cr)
    if threads:
        L.cgo_set_threads(threads)
    p = make_params(state, order, **kw)
    out = state.copy()
    f = np.ascontiguousarray(out.fields, dtype=np.float64)
    frw = np.zeros(2 + 4)
    rc = L.cgo_evolve(ctypes.byref(p), _ptr(f), steps, _ptr(frw))
    if rc != 0:
        raise RuntimeError(f"cgo_evolve failed: {rc}")
    out.fields = f
    out.step = state.step + steps
    out.frw_phi, out.frw_K = float(frw[0]), float(frw[1])
    out.fluids = tuple((float(frw[2 + i]), w) for i, (_, w) in enumerate(state.fluids))
    return out


def rhs(state, order: int, **kw) -> np.ndarray:
    L = lib()
    p = make_params(state, order, **kw)
    f = np.ascontiguousarray(state.fields, dtype=np.float64)
    out = np.zeros_like(f)
    rc = L.cgo_rhs(ctypes.byref(p), _ptr(f), _ptr(out))
    if rc != 0:
        raise RuntimeError(f"cgo_rhs failed: {rc}")
    return out


def constraints(state, order: int, **kw) -> dict:
    L = lib()
    p = make_params(state, order, **kw)
    f = np.ascontiguousarray(state.fields, dtype=np.float64)
    H, M = np.zeros(8), np.zeros(8)
    G, A, S = np.zeros(7), np.zeros(7), np.zeros(7)
    rc = L.cgo_constraints(ctypes.byref(p), _ptr(f), _ptr(H), _ptr(M), _ptr(G), _ptr(A), _ptr(S))
    if rc != 0:
        raise RuntimeError(f"cgo_constraints failed: {rc}")
    return {"H": H, "M": M, "G": G, "A": A, "S": S}


def field_statistics(state, order: int, **kw) -> np.ndarray:
    """io_bssn_dump_statistics columns after the step initialisation:
    volume-weighted mean and stdev of DIFFphi, DIFFK, DIFFr, ricci; volume
    average (cgo_field_statistics)."""
    L = lib()
    p = make_params(state, order, **kw)
    f = np.ascontiguousarray(state.fields, dtype=np.float64)
    out = np.zeros(9)
    rc = L.cgo_field_statistics(ctypes.byref(p), _ptr(f), _ptr(out))
    if rc != 0:
        raise RuntimeError(f"cgo_field_statistics failed: {rc}")
    return out


def frw_evolve(phi: float, K: float, fluids, h: float, steps: int):
    L = lib()
    st = np.array([phi, K] + [r for r, _ in fluids], dtype=np.float64)
    w = np.array([w for _, w in fluids] + [0.0], dtype=np.float64)
    L.cgo_frw_evolve(_ptr(st), _ptr(w), len(fluids), h, steps)
    return st


# ---------------------------------------------------------------------------
# the reference's own sources (oracle/_ref)
# ---------------------------------------------------------------------------

# gauge keys written only when a run sets them (BSSNGaugeHandler.h:137-147,
# bssn.cc:18); the reference's defaults apply otherwise
GAUGE_KEYS = ("shift", "gd_c", "gd_eta", "dw_mu_l", "dw_mu_s", "dw_p", "gauge_wave_dir", "k_driver_coeff")


def reference_config_text(lapse: str = "Harmonic", normalize_metric: int = 1,
                          ko_coeff: float = 0.0, a_adj_amp: float = 0.0,
                          k_damping_amp: float = 0.0, **extra) -> str:
    """The reference's `key = value` config keys read by the BSSN constructor
    (components/bssn/bssn.cc:15-22) and the gauge handler."""
    text = (f"lapse = {lapse}\nnormalize_metric = {normalize_metric}\n"
            f"KO_damping_coefficient = {ko_coeff!r}\na_adj_amp = {a_adj_amp!r}\n"
            f"k_damping_amp = {k_damping_amp!r}\n")
    for key in GAUGE_KEYS:
        if extra.get(key) is not None:
            v = extra[key]
            text += f"{key} = {v if isinstance(v, (str, int)) else repr(float(v))}\n"
    return text


def run_reference(binary: Path, mode: str, state, steps: int = 1, threads: int = 0,
                  timeout: float = 3600.0, **cfg):
    """Run an oracle/_ref binary on a state; returns (result, info)."""
    from cosmograph_b200 import state as cgstate

    env = dict(os.environ)
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    with tempfile.TemporaryDirectory(prefix="cg_ref_run_") as tmp:
        tmp = Path(tmp)
        (tmp / "config.txt").write_text(reference_config_text(**cfg))
        state.save(tmp / "in.bin")
        out = tmp / "out.bin"
        proc = subprocess.run([str(binary), mode, str(tmp / "config.txt"), str(tmp / "in.bin"),
                               str(out), str(steps)], capture_output=True, text=True,
                              env=env, timeout=timeout)
        if proc.returncode != 0:
            raise RuntimeError(f"{binary.name} failed ({proc.returncode}): {proc.stderr[-2000:]}")
        info = {}
        for line in proc.stdout.splitlines():
            if line.startswith("CGRESULT "):
                info = json.loads(line[len("CGRESULT "):])
        if mode == "constraints":
            res = {}
            for line in out.read_text().splitlines():
                parts = line.split()
                res[parts[0]] = np.array([float(x) for x in parts[1:]])
            return res, info
        return cgstate.load(out), info
