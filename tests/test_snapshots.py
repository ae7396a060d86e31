"""Converter of the driver's raw grid snapshots (`cosmograph_b200.snapshots`):
round trip through the gz raw format the driver writes, the reference's
dataset name "DS1", and the errors for a wrong name or size."""
import gzip

import numpy as np
import pytest

from cosmograph_b200 import snapshots


def _write(path, arr):
    with gzip.open(path, "wb") as f:
        f.write(np.ascontiguousarray(arr, dtype="<f8").tobytes())


def test_round_trip_3d_and_2d(tmp_path):
    rng = np.random.default_rng(3)
    g3 = rng.standard_normal((6, 5, 7))
    _write(tmp_path / "3D_DIFFphi_a10.3d_grid.f64.gz", g3)
    _write(tmp_path / "2D_D_a10.2d_grid.f64.gz", g3[0])
    out3 = snapshots.convert(tmp_path / "3D_DIFFphi_a10.3d_grid.f64.gz", 6, 5, 7)
    out2 = snapshots.convert(tmp_path / "2D_D_a10.2d_grid.f64.gz", 6, 5, 7)
    assert out3.name == "3D_DIFFphi_a10.3d_grid.npz" and out2.name == "2D_D_a10.2d_grid.npz"
    with np.load(out3) as z:
        assert list(z.keys()) == ["DS1"] and z["DS1"].dtype == np.float64
        assert np.array_equal(z["DS1"], g3)
    with np.load(out2) as z:
        assert np.array_equal(z["DS1"], g3[0])


def test_cli(tmp_path, capsys):
    g = np.arange(2 * 3 * 4, dtype=np.float64).reshape(2, 3, 4)
    p = tmp_path / "3D_K_a0.3d_grid.f64.gz"
    _write(p, g)
    assert snapshots.main(["2", "3", "4", str(p)]) == 0
    assert capsys.readouterr().out.strip().endswith("3D_K_a0.3d_grid.npz")
    assert snapshots.main(["2", "3"]) == 2


def test_errors(tmp_path):
    p = tmp_path / "3D_K_a0.3d_grid.f64.gz"
    _write(p, np.zeros(23))
    with pytest.raises(ValueError, match="expected 192"):
        snapshots.read_grid(p, 2, 3, 4)
    with pytest.raises(ValueError, match="not a grid snapshot"):
        snapshots.read_grid(tmp_path / "K.strip.dat.gz", 2, 3, 4)
