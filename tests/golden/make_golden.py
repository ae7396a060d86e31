"""Generate the golden fixtures in tests/golden/ from the reference's own sources.

Each fixture holds an input state and the reference's output on it, produced
by the reference's BSSN / Dust / Scalar / Lambda classes compiled unmodified
(strict FP build, oracle/build_ref.py; with USE_Z4c_DAMPING for the *_z4c
cases, with USE_BSSN_SHIFT and USE_GAMMA_DRIVER for the *_shift cases) and
driven by oracle/ref_driver.cc.
Needs the reference checkout, so it runs only where that exists; the
resulting .npz files are committed and need nothing at test time.

Usage: python tests/golden/make_golden.py [case ...]   (default: every case)
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
from oracle import build_ref  # noqa: E402
from cosmograph_b200 import ics  # noqa: E402
from cosmograph_b200 import state as S  # noqa: E402

OUT = Path(__file__).resolve().parent

# name, matter, shape, order, seed, amp, mode, steps, config
CASES = [
    ("dust_o4", S.DUST, (8, 10, 12), 4, 11, 2e-2, "evolve", 5, {"lapse": "Harmonic"}),
    ("dust_o8", S.DUST, (10, 9, 11), 8, 12, 2e-2, "evolve", 3, {"lapse": "Harmonic"}),
    ("scalar_o6", S.SCALAR, (8, 8, 10), 6, 13, 2e-2, "evolve", 3, {"lapse": "Harmonic"}),
    ("vacuum_o2", S.VACUUM, (8, 8, 8), 2, 14, 3e-2, "evolve", 4,
     {"lapse": "OnePlusLog", "a_adj_amp": 0.2, "k_damping_amp": 0.1}),
    ("dust_o4_rhs", S.DUST, (8, 10, 12), 4, 11, 2e-2, "rhs", 0, {"lapse": "Harmonic"}),
    ("dust_o8_constraints", S.DUST, (10, 9, 11), 8, 12, 2e-2, "constraints", 0, {"lapse": "Harmonic"}),
    ("scalar_o6_constraints", S.SCALAR, (8, 8, 10), 6, 13, 2e-2, "constraints", 0, {"lapse": "Harmonic"}),
    ("sinusoid_o4", S.DUST, (16, 4, 4), 4, 0, 0.0, "evolve", 20, {"lapse": "Harmonic"}),
    ("grf_dust_o4", S.DUST, (8, 8, 8), 4, 9, 0.0, "evolve", 5, {"lapse": "Harmonic"}),
    ("static_o4", S.STATIC, (10, 8, 12), 4, 15, 2e-2, "evolve", 4, {"lapse": "Static"}),
    ("static_o8", S.STATIC, (12, 10, 9), 8, 16, 2e-2, "evolve", 3, {"lapse": "ConformalFLRW"}),
    # Z4c damping: the reference built with USE_Z4c_DAMPING (flavour strict_z4c)
    ("dust_z4c_o4", S.DUST, (10, 8, 12), 4, 17, 2e-2, "evolve", 4, {"lapse": "Harmonic"}),
    ("scalar_z4c_o8", S.SCALAR, (9, 10, 8), 8, 18, 2e-2, "evolve", 3, {"lapse": "Harmonic"}),
    ("vacuum_z4c_o2", S.VACUUM, (8, 8, 10), 2, 19, 3e-2, "evolve", 4,
     {"lapse": "OnePlusLog", "ko_coeff": 0.2}),
    # the shift: the reference built with USE_BSSN_SHIFT and USE_GAMMA_DRIVER
    # (flavour strict_shift); beta^i at ten times the amplitude of the rest
    ("dust_shift_o4", S.DUST, (10, 8, 12), 4, 41, 2e-2, "evolve", 3,
     {"lapse": "Harmonic", "shift": "GammaDriver", "gd_eta": 0.5}),
    ("scalar_shift_o2", S.SCALAR, (8, 10, 8), 2, 42, 2e-2, "evolve", 3,
     {"lapse": "OnePlusLog", "shift": "AijDriverShift", "ko_coeff": 0.2}),
    ("vacuum_shift_o8", S.VACUUM, (10, 10, 9), 8, 43, 2e-2, "evolve", 2,
     {"lapse": "DampedWave", "shift": "DampedWave", "dw_mu_l": 0.2, "dw_mu_s": 0.3, "dw_p": 0.5,
      "ko_coeff": 0.1}),
    ("dust_shift_awa_o4", S.DUST, (8, 12, 10), 4, 44, 2e-2, "evolve", 3,
     {"lapse": "AwAShiftedWave", "shift": "AwAShiftedWave", "gauge_wave_dir": 2}),
    ("scalar_shift_o6", S.SCALAR, (9, 8, 10), 6, 45, 2e-2, "evolve", 2, {"lapse": "Harmonic", "shift": "Static"}),
]


def make_input(name, matter, shape, order, seed, amp):
    if name.startswith("sinusoid"):
        st = ics.sinusoid_dust(shape[0], peak_amplitude_frac=1e-3)
        f = st.fields[:, :, : shape[1], : shape[2]].copy()
        return S.BoxState(fields=f, matter=st.matter, dx=st.dx, dt=st.dt, lam=st.lam)
    if name.startswith("grf"):
        return ics.grf_dust(shape, seed=seed, rms_delta=1e-3, order=order)
    return ics.perturbed(shape, matter, seed=seed, amp=amp, z4c="_z4c" in name, shift="_shift" in name)


def main() -> int:
    if not build_ref.reference_available():
        print("reference checkout not found; nothing to do")
        return 1
    only = set(sys.argv[1:])
    index_path = OUT / "index.json"
    index = json.loads(index_path.read_text()) if only and index_path.exists() else {}
    for name, matter, shape, order, seed, amp, mode, steps, cfg in CASES:
        if only and name not in only:
            continue
        st = make_input(name, matter, shape, order, seed, amp)
        flavour = "strict_z4c" if st.z4c else ("strict_shift" if st.shift else "strict")
        binp = build_ref.build(*shape, order, flavour)
        res, info = oracle.run_reference(binp, mode, st, steps=steps, threads=1, **cfg)
        arrays = {"input": st.fields, "input_header": np.frombuffer(st.header_bytes(), dtype=np.uint8)}
        if mode == "constraints":
            for k, v in res.items():
                arrays[f"c_{k}"] = v
        else:
            arrays["output"] = res.fields
            arrays["output_header"] = np.frombuffer(res.header_bytes(), dtype=np.uint8)
        np.savez_compressed(OUT / f"{name}.npz", **arrays)
        index[name] = {"matter": matter, "shape": list(shape), "order": order, "mode": mode,
                       "steps": steps, "config": cfg, "generator": f"reference sources, {flavour} build",
                       "binary": binp.name}
        print(name, mode, info)
    index_path.write_text(json.dumps(index, indent=1, sort_keys=True) + "\n")
    return 0


if __name__ == "__main__":
    sys.exit(main())
