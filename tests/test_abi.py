"""The C-ABI library: it builds, loads without a GPU, exports every symbol the
public header declares, and rejects bad descriptors before touching CUDA."""
import ctypes
import re
from pathlib import Path

import pytest

from cosmograph_b200 import _lib
from cosmograph_b200.build import build

HEADER = Path(__file__).resolve().parents[1] / "include" / "cosmograph_b200.h"


@pytest.fixture(scope="module")
def L():
    build()
    return _lib.load()


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"\b(cg_[a-z_0-9]+)\s*\(", text)))


def test_header_declares_what_the_binding_knows():
    assert declared_symbols() == sorted(_lib.EXPORTS)


def test_header_constants_match_the_binding():
    """Every CG_OPT_* / CG_STATUS_* value of the header is the binding's."""
    text = HEADER.read_text()
    consts = dict(re.findall(r"#define CG_((?:OPT|STATUS)_[A-Z_]+)\s+(\d+)u?", text))
    assert consts, "no constants parsed"
    for name, value in consts.items():
        assert getattr(_lib, name) == int(value), name


def test_library_exports_every_declared_symbol(L):
    for name in declared_symbols():
        assert hasattr(L, name), name


def test_host_only_entry_points(L):
    assert L.cg_version() == 1
    assert [L.cg_num_fields(m) for m in (0, 1, 2, 3)] == [18, 22, 23, 19]
    assert L.cg_field_name(3, 18) == b"DIFFD"
    assert L.cg_field_name(1, 0) == b"DIFFgamma11"
    assert L.cg_field_name(1, 21) == b"S3"
    assert L.cg_field_name(2, 22) == b"psi3"
    assert L.cg_field_name(0, 18) is None
    d = _lib.BoxDesc()
    L.cg_box_desc_default(ctypes.byref(d), 64)
    assert (d.nx, d.stencil_order, d.lapse, d.normalize_metric) == (64, 8, 1, 1)
    assert d.dx == 1.0 / 64 and d.dt == pytest.approx(0.1 / 64, rel=1e-15)


@pytest.mark.parametrize("field,value,msg", [
    ("stencil_order", 5, "stencil_order"),
    ("nx", 2, "at least"),
    ("z4c", 2, "z4c"),
    ("lapse", 42, "lapse"),
    ("nx", 5, None),         # with ko_coeff: order 8 dissipation needs 6 points per axis
    ("nfluids", 7, "fluids"),
    ("matter", 3, "constant lapse"),  # static matter with the default (Harmonic) lapse
    ("matter", 4, "matter"),
])
def test_create_rejects_bad_descriptors(L, field, value, msg):
    d = _lib.BoxDesc()
    L.cg_box_desc_default(ctypes.byref(d), 16)
    setattr(d, field, value)
    if msg is None:
        d.ko_coeff, msg = 0.5, "Kreiss-Oliger"
    h = ctypes.c_void_p()
    rc = L.cg_create(ctypes.byref(d), 1, ctypes.byref(h))
    assert rc == -1 and not h.value
    assert msg in L.cg_last_error(None).decode()


@pytest.mark.parametrize("changes,msg", [
    ({"shift": 6}, "unknown shift gauge"),
    ({"shift": 2, "precision": 1}, "CG_PREC_FP64 only"),
    ({"shift": 2, "precision": 2}, "CG_PREC_FP64 only"),
    ({"shift": 1, "matter": 3, "lapse": 0}, "static matter has no shift"),
    ({"shift": 1, "z4c": 1}, "do not combine"),
    ({"shift": 1, "nx": 3, "stencil_order": 2}, "4 points per axis"),
    ({"shift": 4, "gauge_wave_dir": 4}, "gauge_wave_dir"),
])
def test_create_rejects_bad_shift_descriptors(L, changes, msg):
    d = _lib.BoxDesc()
    L.cg_box_desc_default(ctypes.byref(d), 16)
    assert (d.shift, d.gauge_wave_dir, d.k_driver_coeff) == (0, 1, 0.04)
    for k, v in changes.items():
        setattr(d, k, v)
    h = ctypes.c_void_p()
    rc = L.cg_create(ctypes.byref(d), 1, ctypes.byref(h))
    assert rc == -1 and not h.value
    assert msg in L.cg_last_error(None).decode()


@pytest.mark.parametrize("n", [0, (1 << 30) + 1, 1 << 31, (1 << 32) + 5])
def test_noalloc_average_rejects_sizes_before_touching_cuda(L, n):
    """The allocation-free average checks n against its fixed scratch (at most
    CG_NOALLOC_MAX_POINTS = 2^30 points) before any CUDA call, so the check
    runs without a GPU."""
    rc = L.cg_conformal_average_noalloc(ctypes.c_void_p(16), ctypes.c_void_p(16), n, 0.0, ctypes.c_void_p(16), None)
    assert rc == -1
    assert b"n must be in 1.." in L.cg_last_error(None)


def test_conformal_average_rejects_a_null_context(L):
    rc = L.cg_conformal_average(None, ctypes.c_void_p(16), ctypes.c_void_p(16), 1 << 31, 0.0,
                                ctypes.byref(ctypes.c_double()))
    assert rc == -1
