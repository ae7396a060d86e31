"""ctypes binding of the C ABI (include/cosmograph_b200.h).

The CUDA library is loaded from the package directory; there is no CPU
fallback: if libcosmograph_b200.so is missing or cannot be loaded, every call
raises.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import os

# CG_LIBRARY overrides the library file (an alternative build of the same ABI)
LIB_PATH = Path(os.environ.get("CG_LIBRARY") or Path(__file__).resolve().parent / "libcosmograph_b200.so")

CG_OK = 0
ERRORS = {-1: "invalid argument", -2: "CUDA error", -3: "out of memory", -4: "out of sequence",
          -10: "NaN detected"}

MATTER = {"vacuum": 0, "dust": 1, "scalar": 2, "static": 3}
LAPSE = {
    "Static": 0, "Harmonic": 1, "ConformalFLRW": 2, "ConformalSync": 3, "Anharmonic": 4,
    "OnePlusLog": 5, "AwAGaugeWave": 6, "AwAShiftedWave": 7, "DampedWave": 8,
}
PRECISION = {"fp64": 0, "fp64_fma": 1, "mixed": 2}
SHIFT = {"Static": 1, "GammaDriver": 2, "DampedWave": 3, "AwAShiftedWave": 4, "AijDriverShift": 5}
POTENTIAL = {"const": 0, "quadratic": 1}
STATUS_NAN, STATUS_NONFINITE, STATUS_TILE_TIMEOUT = 1, 2, 4

# every symbol include/cosmograph_b200.h declares
EXPORTS = (
    "cg_box_desc_default", "cg_create", "cg_destroy", "cg_set_stream", "cg_get_stream",
    "cg_num_fields", "cg_field_name", "cg_upload_state", "cg_download_state",
    "cg_upload_state_async", "cg_download_state_async", "cg_exchange_state_async", "cg_prefetch_state_async",
    "cg_upload_field", "cg_download_field",
    "cg_device_register", "cg_substep_input", "cg_background_sums", "cg_set_background",
    "cg_kavg_sums", "cg_set_kavg", "cg_step_init", "cg_rk_stage", "cg_step", "cg_synchronize",
    "cg_status", "cg_frw_state", "cg_step_count", "cg_last_error", "cg_version",
    "cg_conformal_average", "cg_conformal_average_noalloc", "cg_constraints", "cg_field_statistics",
    "cg_set_option", "cg_num_groups", "cg_group_info", "cg_ic_grf_dust", "cg_ic_grf_scalar", "cg_fp64_peak",
)
OPT_BATCH, OPT_GRAPH, OPT_AUTOTUNE, OPT_GROUP_GRID, OPT_TMA, OPT_TMA_WAIT = 1, 2, 3, 4, 5, 6


class BoxDesc(ctypes.Structure):
    """cg_box_desc"""
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("stencil_order", ctypes.c_int), ("matter", ctypes.c_int), ("lapse", ctypes.c_int),
        ("precision", ctypes.c_int), ("normalize_metric", ctypes.c_int),
        ("potential", ctypes.c_int), ("x_ghost", ctypes.c_int),
        ("dx", ctypes.c_double), ("dt", ctypes.c_double), ("lam", ctypes.c_double),
        ("ko_coeff", ctypes.c_double), ("a_adj_amp", ctypes.c_double),
        ("k_damping_amp", ctypes.c_double), ("gd_c", ctypes.c_double),
        ("dw_mu_l", ctypes.c_double), ("dw_p", ctypes.c_double),
        ("pot_const", ctypes.c_double), ("pot_mass", ctypes.c_double),
        ("frw_phi", ctypes.c_double), ("frw_K", ctypes.c_double),
        ("nfluids", ctypes.c_int), ("z4c", ctypes.c_int),
        ("fluid_rho", ctypes.c_double * 4), ("fluid_w", ctypes.c_double * 4),
        ("shift", ctypes.c_int), ("gauge_wave_dir", ctypes.c_int), ("gd_eta", ctypes.c_double),
        ("dw_mu_s", ctypes.c_double), ("k_driver_coeff", ctypes.c_double),
    ]


_lib = None


def load() -> ctypes.CDLL:
    """Load the CUDA library (raises if it is missing: there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing; build it with `python -m cosmograph_b200.build`")
    L = ctypes.CDLL(str(LIB_PATH))
    vp, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)
    i, sz = ctypes.c_int, ctypes.c_size_t
    sig = {
        "cg_box_desc_default": (None, [ctypes.POINTER(BoxDesc), i]),
        "cg_create": (i, [ctypes.POINTER(BoxDesc), i, ctypes.POINTER(vp)]),
        "cg_destroy": (i, [vp]),
        "cg_set_stream": (i, [vp, vp]),
        "cg_get_stream": (i, [vp, ctypes.POINTER(vp)]),
        "cg_num_fields": (i, [i]),
        "cg_field_name": (ctypes.c_char_p, [i, i]),
        "cg_upload_state": (i, [vp, i, dp, sz]),
        "cg_download_state": (i, [vp, i, dp, sz]),
        "cg_upload_state_async": (i, [vp, i, dp, sz]),
        "cg_download_state_async": (i, [vp, i, dp, sz]),
        "cg_exchange_state_async": (i, [vp, i, dp, dp, sz]),
        "cg_prefetch_state_async": (i, [vp, i, dp, sz]),
        "cg_upload_field": (i, [vp, i, i, ctypes.c_char, dp, sz]),
        "cg_download_field": (i, [vp, i, i, ctypes.c_char, dp, sz]),
        "cg_device_register": (i, [vp, i, ctypes.c_char, ctypes.POINTER(dp)]),
        "cg_substep_input": (i, [vp, i, ctypes.POINTER(vp), ctypes.POINTER(vp)]),
        "cg_background_sums": (i, [vp, i, dp, i]),
        "cg_set_background": (i, [vp, i, dp, i]),
        "cg_kavg_sums": (i, [vp, i, ctypes.POINTER(vp)]),
        "cg_set_kavg": (i, [vp, i, vp]),
        "cg_step_init": (i, [vp]),
        "cg_rk_stage": (i, [vp, i]),
        "cg_step": (i, [vp, i]),
        "cg_synchronize": (i, [vp]),
        "cg_status": (i, [vp, ctypes.POINTER(ctypes.c_uint32)]),
        "cg_frw_state": (i, [vp, i, dp, i]),
        "cg_step_count": (i, [vp, i, ctypes.POINTER(ctypes.c_int64)]),
        "cg_last_error": (ctypes.c_char_p, [vp]),
        "cg_conformal_average": (i, [vp, vp, vp, sz, ctypes.c_double, dp]),
        "cg_conformal_average_noalloc": (i, [vp, vp, sz, ctypes.c_double, vp, vp]),
        "cg_constraints": (i, [vp, i, dp, dp, dp, dp, dp]),
        "cg_field_statistics": (i, [vp, i, dp, i]),
        "cg_set_option": (i, [vp, i, i]),
        "cg_ic_grf_dust": (i, [vp, i, dp, ctypes.c_uint64, ctypes.c_double, ctypes.c_double, ctypes.c_double]),
        "cg_ic_grf_scalar": (i, [vp, i, dp, ctypes.c_uint64, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                 ctypes.c_double]),
        "cg_num_groups": (i, [vp, ctypes.POINTER(i)]),
        "cg_group_info": (i, [vp, i, ctypes.POINTER(i), i]),
        "cg_version": (i, []),
        "cg_fp64_peak": (i, [dp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


class CgError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


def check(rc: int, ctx=None) -> None:
    if rc != CG_OK:
        L = load()
        msg = L.cg_last_error(ctx)
        raise CgError(rc, msg.decode() if msg else "")
