"""bench.py's output contract, checked on the CPU through its reference arm
(the reference's own sources timed on the host cores) on a small box: one
JSON line with the keys the benchmark consumers read."""
import json
import subprocess
import sys
from pathlib import Path

import pytest

from oracle import build_ref

ROOT = Path(__file__).resolve().parents[1]
KEYS = {"metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
        "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"}


def test_reference_arm_prints_one_contract_line():
    binp = build_ref.binary_path(16, 16, 16, 4, "fast")
    if not binp.exists():
        if not build_ref.reference_available():
            pytest.skip("no reference build for 16^3 and no reference sources to build it")
        build_ref.build(16, 16, 16, 4, "fast")
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--n", "16", "--order", "4",
                        "--steps", "2", "--warmup", "1"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert KEYS <= set(d), KEYS - set(d)
    assert d["impl"] == "reference" and d["value"] > 0 and d["higher_is_better"] is True
    assert d["config"]["workload"] == "bssn_dust_16cubed_o4"
    # the same workload description as the GPU arm prints
    import bench

    assert d["config"] == bench.box_config(16, 4, "fp64", 1)
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["value"] == d["value"]
