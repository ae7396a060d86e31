"""Box state files: the checkpoint / interchange format of the evolved fields.

A state file holds the "_p" register of every evolved field of one periodic
box (the reference's RK4Register::_array_p, utils/RK4Register.h:27) as
little-endian FP64 arrays in the reference's memory order -- x slowest, z
fastest, NP_INDEX(i,j,k) = (NZ*NY)*i + NZ*j + k (cosmo_macros.h:118) -- plus
dx, dt, the step counter and the FRW reference background (utils/FRW.h:14-20).
The same bytes feed the reference CPU build, the CPU restatement and the CUDA
path, and a run can be resumed from one.

Field order is the reference's field-list order: BSSN_APPLY_TO_FIELDS
(components/bssn/bssn_macros.h:77-95), then the dust registers D, S1, S2, S3
(components/dust_fluid/dust.h:32-35), the scalar registers phi, Pi, psi1,
psi2, psi3 (components/scalar/scalar.h:35-39), or the static sims' fixed
density DIFFD (components/static/static.h:17), which no substep changes.
With Z4c damping theta follows, and with the shift beta1..3, auxB1..3, expN
(header flag bits 0 and 1).
"""
from __future__ import annotations

import dataclasses
import struct
from pathlib import Path

import numpy as np

MAGIC = b"CGSTATE1"
MAX_FLUIDS = 4

VACUUM, DUST, SCALAR, STATIC = 0, 1, 2, 3
MATTER_NAMES = {"vacuum": VACUUM, "dust": DUST, "scalar": SCALAR, "static": STATIC}

BSSN_FIELDS = (
    "DIFFgamma11", "DIFFgamma12", "DIFFgamma13", "DIFFgamma22", "DIFFgamma23",
    "DIFFgamma33", "DIFFphi", "A11", "A12", "A13", "A22", "A23", "A33", "DIFFK",
    "Gamma1", "Gamma2", "Gamma3", "DIFFalpha",
)
DUST_FIELDS = ("D", "S1", "S2", "S3")
SCALAR_FIELDS = ("phi", "Pi", "psi1", "psi2", "psi3")
STATIC_FIELDS = ("DIFFD",)  # the static sims' fixed density (components/static/static.h:17), not evolved
# Z4c damping (USE_Z4c_DAMPING, cosmo_macros.h:91-100): the constraint field
# theta (Z4c_APPLY_TO_FIELDS, bssn_macros.h:8-13), stored after the matter fields
Z4C_FIELDS = ("theta",)
FLAG_Z4C = 1  # header flags bit: the box carries theta
# the shift (USE_BSSN_SHIFT, cosmo_macros.h:43) with the Gamma-driver's
# auxiliary field (USE_GAMMA_DRIVER, :48) and expN (bssn_macros.h:18-50),
# stored after the matter fields and theta
SHIFT_FIELDS = ("beta1", "beta2", "beta3", "auxB1", "auxB2", "auxB3", "expN")
FLAG_SHIFT = 2  # header flags bit: the box carries the shift fields

# header layout (168 bytes); mirrors oracle/cg_state.h
_HDR = struct.Struct("<8s8i4d4d4dd3d")
assert _HDR.size == 168


def field_names(matter: int, z4c: bool = False, shift: bool = False) -> tuple[str, ...]:
    extra = (Z4C_FIELDS if z4c else ()) + (SHIFT_FIELDS if shift else ())
    if matter == DUST:
        return BSSN_FIELDS + DUST_FIELDS + extra
    if matter == SCALAR:
        return BSSN_FIELDS + SCALAR_FIELDS + extra
    if matter == STATIC:
        return BSSN_FIELDS + STATIC_FIELDS + extra
    return BSSN_FIELDS + extra


def num_fields(matter: int, z4c: bool = False, shift: bool = False) -> int:
    return len(field_names(matter, z4c, shift))


@dataclasses.dataclass
class BoxState:
    """One periodic box: fields[f] is an (nx, ny, nz) float64 array."""

    fields: np.ndarray                 # (nfields, nx, ny, nz) float64, C order
    matter: int
    dx: float
    dt: float
    step: int = 0
    frw_phi: float = 0.0
    frw_K: float = 0.0
    fluids: tuple[tuple[float, float], ...] = ()   # (rho, w) pairs
    lam: float = 0.0                   # rho_Lambda (Lambda::setLambda)
    z4c: bool = False                  # Z4c damping: theta after the matter fields
    shift: bool = False                # the shift fields after those

    @property
    def shape(self) -> tuple[int, int, int]:
        return tuple(self.fields.shape[1:])  # type: ignore[return-value]

    @property
    def names(self) -> tuple[str, ...]:
        return field_names(self.matter, self.z4c, self.shift)

    def field(self, name: str) -> np.ndarray:
        return self.fields[self.names.index(name)]

    def copy(self) -> "BoxState":
        return dataclasses.replace(self, fields=self.fields.copy())

    def header_bytes(self) -> bytes:
        nx, ny, nz = self.shape
        if len(self.fluids) > MAX_FLUIDS:
            raise ValueError("at most 4 FRW fluids")
        rho = [f[0] for f in self.fluids] + [0.0] * (MAX_FLUIDS - len(self.fluids))
        w = [f[1] for f in self.fluids] + [0.0] * (MAX_FLUIDS - len(self.fluids))
        return _HDR.pack(MAGIC, nx, ny, nz, self.fields.shape[0], self.matter,
                         self.step, len(self.fluids), self.flags, self.dx, self.dt,
                         self.frw_phi, self.frw_K, *rho, *w, self.lam, 0.0, 0.0, 0.0)

    @property
    def flags(self) -> int:
        return (FLAG_Z4C if self.z4c else 0) | (FLAG_SHIFT if self.shift else 0)

    def save(self, path: str | Path) -> None:
        f = np.ascontiguousarray(self.fields, dtype="<f8")
        if f.shape[0] != num_fields(self.matter, self.z4c, self.shift):
            raise ValueError("field count does not match the matter model")
        with open(path, "wb") as fh:
            fh.write(self.header_bytes())
            fh.write(f.tobytes())


def load(path: str | Path) -> BoxState:
    raw = Path(path).read_bytes()
    if len(raw) < _HDR.size:
        raise ValueError(f"{path}: truncated state header")
    h = _HDR.unpack_from(raw, 0)
    if h[0] != MAGIC:
        raise ValueError(f"{path}: not a state file")
    nx, ny, nz, nf, matter, step, nfl, flags = h[1:9]
    z4c, shift = bool(flags & FLAG_Z4C), bool(flags & FLAG_SHIFT)
    dx, dt, phi, K = h[9:13]
    rho, w, lam = h[13:17], h[17:21], h[21]
    if nf != num_fields(matter, z4c, shift) or not 0 <= nfl <= MAX_FLUIDS:
        raise ValueError(f"{path}: inconsistent header")
    n = nf * nx * ny * nz
    if len(raw) != _HDR.size + 8 * n:
        raise ValueError(f"{path}: truncated field data ({len(raw)} bytes)")
    fields = np.frombuffer(raw, dtype="<f8", count=n, offset=_HDR.size)
    return BoxState(fields=fields.reshape(nf, nx, ny, nz).astype(np.float64),
                    matter=matter, dx=dx, dt=dt, step=step, frw_phi=phi, frw_K=K,
                    fluids=tuple((rho[i], w[i]) for i in range(nfl)), lam=lam, z4c=z4c, shift=shift)
