"""Python front end of the C ABI: a context of periodic boxes on one GPU.

`Evolution` owns a cg_ctx; its methods follow the reference's sim-driver
sequence (sims/dust.cc:53-169): step_init() is BSSN::stepInit + Dust::stepInit
and the source pass, rk_stage(n) is one substep (RKEvolve + K{n}Finalize of
every field), step(n) runs whole RK4 steps.
"""
from __future__ import annotations

import ctypes
import dataclasses

import numpy as np

from . import _lib
from .state import BoxState, num_fields


@dataclasses.dataclass
class BoxConfig:
    """Per-box options (the reference's compile-time switches and config keys)."""

    order: int = 8
    lapse: str = "Harmonic"
    precision: str = "fp64"
    normalize_metric: int = 1
    potential: str = "const"
    pot_const: float = 3.0e-4
    pot_mass: float = 1.0
    ko_coeff: float = 0.0
    a_adj_amp: float = 0.0
    k_damping_amp: float = 0.0
    gd_c: float = 1.0
    dw_mu_l: float = 0.0
    dw_p: float = 0.0
    shift: str = "Static"   # the shift gauge of a box whose state carries the shift fields
    gd_eta: float = 0.0
    dw_mu_s: float = 0.0
    gauge_wave_dir: int = 1
    k_driver_coeff: float = 0.04
    x_ghost: int = 0  # > 0: the box is an x-slab with this many ghost planes per face (cosmograph_b200.slab)


def make_desc(state: BoxState, cfg: BoxConfig) -> _lib.BoxDesc:
    d = _lib.BoxDesc()
    d.nx, d.ny, d.nz = state.shape
    d.stencil_order = cfg.order
    d.matter = state.matter
    d.lapse = _lib.LAPSE[cfg.lapse]
    d.precision = _lib.PRECISION[cfg.precision]
    d.normalize_metric = cfg.normalize_metric
    d.potential = _lib.POTENTIAL[cfg.potential]
    d.dx, d.dt, d.lam = state.dx, state.dt, state.lam
    d.ko_coeff, d.a_adj_amp, d.k_damping_amp = cfg.ko_coeff, cfg.a_adj_amp, cfg.k_damping_amp
    d.gd_c, d.dw_mu_l, d.dw_p = cfg.gd_c, cfg.dw_mu_l, cfg.dw_p
    d.pot_const, d.pot_mass = cfg.pot_const, cfg.pot_mass
    d.x_ghost = cfg.x_ghost
    d.z4c = 1 if state.z4c else 0
    d.shift = _lib.SHIFT[cfg.shift] if state.shift else 0
    d.gauge_wave_dir, d.gd_eta, d.dw_mu_s = cfg.gauge_wave_dir, cfg.gd_eta, cfg.dw_mu_s
    d.k_driver_coeff = cfg.k_driver_coeff
    d.frw_phi, d.frw_K = state.frw_phi, state.frw_K
    d.nfluids = len(state.fluids)
    for n, (rho, w) in enumerate(state.fluids):
        d.fluid_rho[n], d.fluid_w[n] = rho, w
    return d


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Evolution:
    """A set of boxes evolved together on one GPU."""

    def __init__(self, states, configs):
        if isinstance(states, BoxState):
            states, configs = [states], [configs]
        if len(states) != len(configs):
            raise ValueError("one BoxConfig per box")
        self.L = _lib.load()
        self.templates = [s.copy() for s in states]
        descs = (_lib.BoxDesc * len(states))(*[make_desc(s, c) for s, c in zip(states, configs)])
        h = ctypes.c_void_p()
        rc = self.L.cg_create(descs, len(states), ctypes.byref(h))
        if rc != _lib.CG_OK:
            _lib.check(rc, None)
        self.ctx = h
        for b, s in enumerate(states):
            self.upload(b, s)

    # -- lifecycle ---------------------------------------------------------
    def close(self) -> None:
        if self.ctx:
            self.L.cg_destroy(self.ctx)
            self.ctx = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int) -> None:
        _lib.check(rc, self.ctx)

    # -- data movement -------------------------------------------------------
    def upload(self, box: int, state: BoxState) -> None:
        f = np.ascontiguousarray(state.fields, dtype=np.float64)
        self._check(self.L.cg_upload_state(self.ctx, box, _dptr(f), f.size))

    def download(self, box: int = 0) -> BoxState:
        t = self.templates[box]
        out = np.empty((num_fields(t.matter, t.z4c, t.shift),) + t.shape, dtype=np.float64)
        self._check(self.L.cg_download_state(self.ctx, box, _dptr(out), out.size))
        st = dataclasses.replace(t, fields=out)
        frw = np.zeros(2 + 4)
        self._check(self.L.cg_frw_state(self.ctx, box, _dptr(frw), frw.size))
        st.frw_phi, st.frw_K = float(frw[0]), float(frw[1])
        st.fluids = tuple((float(frw[2 + n]), w) for n, (_, w) in enumerate(t.fluids))
        cnt = ctypes.c_int64()
        self._check(self.L.cg_step_count(self.ctx, box, ctypes.byref(cnt)))
        st.step = t.step + int(cnt.value)
        return st

    def download_field(self, box: int, field: int, reg: str = "p") -> np.ndarray:
        t = self.templates[box]
        out = np.empty(t.shape, dtype=np.float64)
        self._check(self.L.cg_download_field(self.ctx, box, field, reg.encode(), _dptr(out), out.size))
        return out

    def upload_field(self, box: int, field: int, reg: str, data: np.ndarray) -> None:
        a = np.ascontiguousarray(data, dtype=np.float64)
        self._check(self.L.cg_upload_field(self.ctx, box, field, reg.encode(), _dptr(a), a.size))

    # -- stepping ----------------------------------------------------------------
    def step_init(self) -> None:
        self._check(self.L.cg_step_init(self.ctx))

    def rk_stage(self, n: int) -> None:
        self._check(self.L.cg_rk_stage(self.ctx, n))

    def step(self, nsteps: int = 1) -> None:
        self._check(self.L.cg_step(self.ctx, nsteps))

    def constraints(self, box: int = 0) -> dict:
        """BSSN::setConstraintCalcs statistics of the current state (between steps)."""
        arrs = {k: np.zeros(8 if k in "HM" else 7) for k in "HMGAS"}
        self._check(self.L.cg_constraints(self.ctx, box, *(_dptr(arrs[k]) for k in "HMGAS")))
        return arrs

    def field_statistics(self, box: int = 0) -> np.ndarray:
        """io_bssn_dump_statistics columns of the current state (between steps):
        volume-weighted mean and stdev of DIFFphi, DIFFK, DIFFr, ricci, then the
        volume average."""
        out = np.zeros(9)
        self._check(self.L.cg_field_statistics(self.ctx, box, _dptr(out), out.size))
        return out

    def synchronize(self) -> None:
        self._check(self.L.cg_synchronize(self.ctx))

    def status(self) -> int:
        f = ctypes.c_uint32()
        self._check(self.L.cg_status(self.ctx, ctypes.byref(f)))
        return int(f.value)

    def ic_grf_dust(self, box: int, seed: int = 9, rms_delta: float = 1.0e-4, ns: float = 0.96,
                    cutoff: float = 0.0, delta: np.ndarray | None = None) -> None:
        """GRF dust initial data built on the GPU (cg_ic_grf_dust); `delta`
        (host density contrast) replaces the GPU's own random field."""
        dptr = None
        if delta is not None:
            delta = np.ascontiguousarray(delta, dtype=np.float64)
            if delta.shape != self.templates[box].shape:
                raise ValueError("delta must have the box's shape")
            dptr = _dptr(delta)
        self._check(self.L.cg_ic_grf_dust(self.ctx, box, dptr, ctypes.c_uint64(seed), rms_delta, ns, cutoff))

    def ic_grf_scalar(self, box: int, seed: int = 9, phi0: float = 1.0e-2, rms: float = 1.0e-5, mass: float = 1.0,
                      cutoff: float = 0.0, dphi: np.ndarray | None = None) -> None:
        """GRF scalar initial data built on the GPU (cg_ic_grf_scalar); `dphi`
        (host fluctuation) replaces the GPU's own random field."""
        dptr = None
        if dphi is not None:
            dphi = np.ascontiguousarray(dphi, dtype=np.float64)
            if dphi.shape != self.templates[box].shape:
                raise ValueError("dphi must have the box's shape")
            dptr = _dptr(dphi)
        self._check(self.L.cg_ic_grf_scalar(self.ctx, box, dptr, ctypes.c_uint64(seed), phi0, rms, mass, cutoff))

    def set_option(self, option: str, value: int) -> None:
        """Launch options: "batch", "graph", "autotune", "group_grid", "tma",
        "tma_wait" (cg_set_option)."""
        code = {"batch": _lib.OPT_BATCH, "graph": _lib.OPT_GRAPH, "autotune": _lib.OPT_AUTOTUNE,
                "group_grid": _lib.OPT_GROUP_GRID, "tma": _lib.OPT_TMA, "tma_wait": _lib.OPT_TMA_WAIT}[option]
        self._check(self.L.cg_set_option(self.ctx, code, int(value)))

    def groups(self) -> list[dict]:
        """Launch groups: boxes, bricks, CTAs per launch, launch order, tuned."""
        n = ctypes.c_int()
        self._check(self.L.cg_num_groups(self.ctx, ctypes.byref(n)))
        out = []
        for g in range(n.value):
            info = (ctypes.c_int * 6)()
            self._check(self.L.cg_group_info(self.ctx, g, info, 6))
            out.append({"boxes": info[0], "bricks": info[1], "grid": info[2], "largest_first": info[3],
                        "tuned": bool(info[4]), "first_box": info[5]})
        return out

    def stream(self) -> int:
        s = ctypes.c_void_p()
        self._check(self.L.cg_get_stream(self.ctx, ctypes.byref(s)))
        return int(s.value or 0)

    def set_stream(self, stream_ptr: int) -> None:
        self._check(self.L.cg_set_stream(self.ctx, ctypes.c_void_p(stream_ptr)))


def evolve(state: BoxState, steps: int, cfg: BoxConfig | None = None) -> BoxState:
    """Evolve one box for `steps` RK4 steps on the GPU and return the new state."""
    cfg = cfg or BoxConfig()
    with Evolution(state, cfg) as ev:
        ev.step(steps)
        ev.synchronize()
        return ev.download(0)
