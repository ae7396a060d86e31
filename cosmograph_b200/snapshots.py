"""Field snapshots written by the config-file driver, and their converter.

The reference writes each 3-D snapshot as an HDF5 file holding one dataset
"DS1" of N^3 FP64 values (IO/io.cc:655-682, chunked 6^3, deflate 9) and each
2-D snapshot as "DS1" of the x = 0 plane.  HDF5 is not available in this
image, so the driver (`host/facade.cc`, `CosmoSim::outputSnapshots`) writes
the same values as gz-compressed raw little-endian FP64 in the box's memory
order (x-major, z fastest), named `3D_<field><step>.3d_grid.f64.gz` and
`2D_<field><step>.2d_grid.f64.gz`.  This module reads those files and
converts them to NumPy `.npz` archives that keep the reference's dataset
name, so analysis code that indexed `f["DS1"]` indexes `np.load(p)["DS1"]`.

    python -m cosmograph_b200.snapshots NX NY NZ FILE [FILE ...]

writes `<stem>.npz` beside each FILE (stem = the name without `.f64.gz`).
"""
from __future__ import annotations

import gzip
import sys
from pathlib import Path

import numpy as np

SUFFIX = ".f64.gz"


def grid_shape(path: str | Path, nx: int, ny: int, nz: int) -> tuple[int, ...]:
    """Shape of the grid in a snapshot file: (nx, ny, nz) for `.3d_grid`,
    (ny, nz) for `.2d_grid` (the x = 0 plane)."""
    name = Path(path).name
    if name.endswith(".3d_grid" + SUFFIX):
        return (nx, ny, nz)
    if name.endswith(".2d_grid" + SUFFIX):
        return (ny, nz)
    raise ValueError(f"not a grid snapshot (expected *.3d_grid{SUFFIX} or *.2d_grid{SUFFIX}): {name}")


def read_grid(path: str | Path, nx: int, ny: int, nz: int) -> np.ndarray:
    """The snapshot's values as an FP64 array of `grid_shape(...)`; raises
    ValueError when the file holds a different number of values."""
    shape = grid_shape(path, nx, ny, nz)
    with gzip.open(path, "rb") as f:
        raw = f.read()
    want = int(np.prod(shape)) * 8
    if len(raw) != want:
        raise ValueError(f"{path}: {len(raw)} bytes, expected {want} for a grid of shape {shape}")
    return np.frombuffer(raw, dtype="<f8").reshape(shape)


def convert(path: str | Path, nx: int, ny: int, nz: int, out: str | Path | None = None) -> Path:
    """Write the snapshot as a compressed `.npz` with the dataset "DS1";
    returns the output path (default: beside the input, `.f64.gz` replaced
    by `.npz`)."""
    path = Path(path)
    data = read_grid(path, nx, ny, nz)
    if out is None:
        out = path.with_name(path.name[: -len(SUFFIX)] + ".npz")
    out = Path(out)
    np.savez_compressed(out, DS1=data)
    return out


def main(argv: list[str] | None = None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    if len(argv) < 4:
        sys.stderr.write(__doc__.split("\n\n")[-2] + "\n")
        return 2
    nx, ny, nz = (int(v) for v in argv[:3])
    for p in argv[3:]:
        print(convert(p, nx, ny, nz))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
