"""Shared helpers for the parity tests: golden fixtures and error norms."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

from cosmograph_b200 import state as S

GOLDEN = Path(__file__).resolve().parent / "golden"


def golden_index() -> dict:
    return json.loads((GOLDEN / "index.json").read_text())


def _state_from(arr: np.ndarray, header: np.ndarray) -> S.BoxState:
    hdr = S._HDR.unpack(header.tobytes())
    st = S.BoxState(fields=np.array(arr, dtype=np.float64), matter=hdr[5], dx=hdr[9], dt=hdr[10],
                    step=hdr[6], frw_phi=hdr[11], frw_K=hdr[12],
                    fluids=tuple((hdr[13 + i], hdr[17 + i]) for i in range(hdr[7])), lam=hdr[21],
                    z4c=bool(hdr[8] & S.FLAG_Z4C), shift=bool(hdr[8] & S.FLAG_SHIFT))
    return st


def load_golden(name: str):
    """Returns (input BoxState, output BoxState | None, extra arrays, meta)."""
    z = np.load(GOLDEN / f"{name}.npz")
    meta = golden_index()[name]
    inp = _state_from(z["input"], z["input_header"])
    out = _state_from(z["output"], z["output_header"]) if "output" in z else None
    extra = {k[2:]: z[k] for k in z.files if k.startswith("c_")}
    return inp, out, extra, meta


def field_errors(got: np.ndarray, ref: np.ndarray, names, floor: float = 1e-15) -> dict:
    """Norm-wise relative error per field: max|got-ref| / max(max|ref|, floor)."""
    out = {}
    for f, n in enumerate(names):
        d = float(np.abs(got[f] - ref[f]).max())
        m = max(float(np.abs(ref[f]).max()), floor)
        out[n] = d / m
    return out


def worst(errs: dict):
    k = max(errs, key=errs.get)
    return k, errs[k]
