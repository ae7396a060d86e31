"""x-slab decomposition of one periodic box.

The reference evolves one box per process; a box too large for one GPU (or
spread over several for speed) is cut here into slabs along x, the slowest
index of the reference's memory order (``NP_INDEX``, cosmo_macros.h:118), so
each slab's planes are contiguous per field.  A slab is a box of its own
(``BoxConfig.x_ghost = g``) holding its ``nloc`` interior planes plus ``g``
ghost planes on each x face; the kernels update the interior only, and before
every substep the ghost planes of the arrays the substep reads with stencils
(the substep input and, for dust, its flux primitives, ``cg_substep_input``)
are refreshed from the neighbouring slabs' interior planes, periodically.
Everything else is pointwise, so the interior evolves exactly as the
corresponding planes of the undivided box.

Two exchanges:

* ``LocalHalo``: all slabs are boxes of one context on one GPU; ghost planes
  are device copies on the context's stream.
* ``DistHalo``: one slab per rank; ghost planes travel as point-to-point
  messages through ``torch.distributed`` (NCCL between GPUs, gloo on CPU).

Lapses that use the grid average of K need the whole box's K_avg before every
substep: each slab's two sums (``cg_kavg_sums``) are added up (across ranks:
an all-reduce) and handed back (``cg_set_kavg``).  FP32-mixed slabs hold FP32
perturbations about one uniform
background, which must be the whole box's: the slabs' sums of the background
fields are added up (across ranks: an all-reduce) and every slab gets the
same means (``cg_set_background``) before the first step.
"""
from __future__ import annotations

import ctypes
from dataclasses import replace

import numpy as np

from .evolution import BoxConfig, Evolution
from .state import BoxState

# dust flux primitives per point (alpha D, alpha S_1..3, v^1..3)
FLUX_ARRAYS = 7


def ghost_width(order: int, ko: bool = False) -> int:
    """Smallest valid ghost width: the stencil reach (the Kreiss-Oliger reach
    at orders 2 and 8 when dissipation is on), rounded up to the brick width 4."""
    reach = (5 if order == 8 else 2) if ko and order in (2, 8) else order // 2
    return -(-reach // 4) * 4


def slab_bounds(nx: int, nslabs: int, index: int) -> tuple[int, int]:
    """First interior plane and plane count of slab `index` (equal slabs)."""
    if nx % nslabs or (nx // nslabs) % 4:
        raise ValueError("nx must split into equal slabs of a multiple of 4 planes")
    nloc = nx // nslabs
    return index * nloc, nloc


def split(state: BoxState, nslabs: int, ghost: int) -> list[BoxState]:
    """The slabs of `state`, each with `ghost` periodic ghost planes per face."""
    nx = state.shape[0]
    out = []
    for s in range(nslabs):
        x0, nloc = slab_bounds(nx, nslabs, s)
        planes = np.arange(x0 - ghost, x0 + nloc + ghost) % nx
        out.append(replace(state.copy(), fields=np.ascontiguousarray(state.fields[:, planes])))
    return out


def assemble(slabs: list[BoxState], ghost: int) -> BoxState:
    """The undivided box from the slabs' interior planes."""
    fields = np.concatenate([s.fields[:, ghost:s.shape[0] - ghost] for s in slabs], axis=1)
    return replace(slabs[0].copy(), fields=np.ascontiguousarray(fields))


class _CudaArray:
    """__cuda_array_interface__ view of library-owned device memory."""

    def __init__(self, ptr: int, shape: tuple[int, ...], typestr: str):
        self.__cuda_array_interface__ = {"shape": shape, "typestr": typestr, "data": (ptr, False),
                                         "version": 2, "strides": None}


def _substep_arrays(ev: Evolution, box: int, nfields: int, shape, mixed: bool) -> list:
    """torch views of the arrays the next substep of `box` reads with stencils
    (FP32 perturbations for a mixed box)."""
    import torch

    inp, flux = ctypes.c_void_p(), ctypes.c_void_p()
    ev._check(ev.L.cg_substep_input(ev.ctx, box, ctypes.byref(inp), ctypes.byref(flux)))
    t = "<f4" if mixed else "<f8"
    out = [torch.as_tensor(_CudaArray(inp.value, (nfields, *shape), t), device="cuda")]
    if flux.value:
        out.append(torch.as_tensor(_CudaArray(flux.value, (FLUX_ARRAYS, *shape), t), device="cuda"))
    return out


def background_sums(ev: Evolution, box: int) -> np.ndarray:
    """Sums of K, phi, alpha, field 18 and field 19 of _p over the box's
    updated points, and their count (cg_background_sums)."""
    out = np.zeros(6)
    ev._check(ev.L.cg_background_sums(ev.ctx, box, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 6))
    return out


KAVG_LAPSES = ("ConformalFLRW", "Anharmonic", "OnePlusLog")


def _kavg_sums(ev: Evolution, box: int):
    """torch view of the box's two K_avg sums over its updated points (queued)."""
    import torch

    p = ctypes.c_void_p()
    ev._check(ev.L.cg_kavg_sums(ev.ctx, box, ctypes.byref(p)))
    return torch.as_tensor(_CudaArray(p.value, (2,), "<f8"), device="cuda")


def _set_kavg(ev: Evolution, box: int, sums) -> None:
    ev._check(ev.L.cg_set_kavg(ev.ctx, box, ctypes.c_void_p(sums.data_ptr())))


def set_background(ev: Evolution, box: int, sums: np.ndarray) -> None:
    means = np.ascontiguousarray(sums[:5] / sums[5])
    ev._check(ev.L.cg_set_background(ev.ctx, box, means.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 5))


def fill_ghosts(arrays_by_slab: list[list], ghost: int) -> None:
    """Periodic ghost refresh among slabs held by one process: slab s's low
    ghosts from slab s-1's top interior planes, its high ghosts from slab
    s+1's bottom interior planes (arrays of shape (fields, nx_s, ny, nz))."""
    n = len(arrays_by_slab)
    for s in range(n):
        left, right = arrays_by_slab[(s - 1) % n], arrays_by_slab[(s + 1) % n]
        for a, al, ar in zip(arrays_by_slab[s], left, right):
            nxl = al.shape[1]
            a[:, :ghost].copy_(al[:, nxl - 2 * ghost:nxl - ghost])
            a[:, a.shape[1] - ghost:].copy_(ar[:, ghost:2 * ghost])


class LocalHalo:
    """Ghost planes among slabs that are boxes of one context (one GPU)."""

    def __init__(self, ev: Evolution, ghost: int, mixed: bool = False):
        self.ev, self.ghost, self.mixed = ev, ghost, mixed

    def exchange(self) -> None:
        ev = self.ev
        arrays = [_substep_arrays(ev, b, t.fields.shape[0], t.shape, self.mixed) for b, t in enumerate(ev.templates)]
        fill_ghosts(arrays, self.ghost)

    def kavg(self) -> None:
        """The whole box's K_avg for every slab's next substep."""
        ev = self.ev
        total = sum(_kavg_sums(ev, b) for b in range(len(ev.templates)))
        for b in range(len(ev.templates)):
            _set_kavg(ev, b, total)

    def background(self) -> None:
        """One background for every slab: the whole box's means."""
        total = sum(background_sums(self.ev, b) for b in range(len(self.ev.templates)))
        for b in range(len(self.ev.templates)):
            set_background(self.ev, b, total)


class DistHalo:
    """Ghost planes between ranks, one slab per rank, periodic ring: each rank
    sends its bottom interior planes to rank-1 and its top ones to rank+1 and
    receives its ghosts from them (``torch.distributed`` point-to-point; every
    rank takes the same steps in the same order).  Messages carry no tags
    (NCCL has none): with two ranks both neighbours are the same rank, and the
    fixed issue order -- send up, send down, receive from below, receive from
    above -- pairs each receive with the right send."""

    def __init__(self, ghost: int, group=None):
        import torch.distributed as dist

        self.dist, self.ghost, self.group = dist, ghost, group
        self.rank = dist.get_rank(group)
        self.size = dist.get_world_size(group)

    def exchange_arrays(self, arrays: list) -> None:
        g, dist = self.ghost, self.dist
        if self.size == 1:
            fill_ghosts([arrays], g)
            return
        left, right = (self.rank - 1) % self.size, (self.rank + 1) % self.size
        gl = dist.get_global_rank(self.group, left) if self.group is not None else left
        gr = dist.get_global_rank(self.group, right) if self.group is not None else right
        # one field's x-planes are one contiguous block: every field's planes
        # are sent from and received into the arrays themselves (no staging
        # copies, no allocation), all fields in one batch, waited for once
        ops = []
        for a in arrays:
            nx = a.shape[1]
            for f in range(a.shape[0]):
                ops += [dist.P2POp(dist.isend, a[f, nx - 2 * g:nx - g], gr, self.group),
                        dist.P2POp(dist.isend, a[f, g:2 * g], gl, self.group),
                        dist.P2POp(dist.irecv, a[f, :g], gl, self.group),
                        dist.P2POp(dist.irecv, a[f, nx - g:], gr, self.group)]
        for r in dist.batch_isend_irecv(ops):
            r.wait()

    def exchange(self, ev: Evolution, mixed: bool = False) -> None:
        t = ev.templates[0]
        self.exchange_arrays(_substep_arrays(ev, 0, t.fields.shape[0], t.shape, mixed))

    def kavg(self, ev: Evolution) -> None:
        """The whole box's K_avg for this rank's next substep: the slabs' sums
        all-reduced in place (the same call on every rank)."""
        sums = _kavg_sums(ev, 0)
        if self.size > 1:
            self.dist.all_reduce(sums, group=self.group)
        _set_kavg(ev, 0, sums)

    def background(self, ev: Evolution) -> None:
        """One background for every rank's slab: the all-reduced sums."""
        import torch

        sums = torch.from_numpy(background_sums(ev, 0))
        if self.size > 1:
            if self.dist.get_backend(self.group) == "nccl":
                sums = sums.cuda()
            self.dist.all_reduce(sums, group=self.group)
        set_background(ev, 0, sums.cpu().numpy())


class SlabEvolution:
    """RK4 steps of a box cut into x-slabs: the substeps of every slab with the
    ghost exchange before each (the sequence of ``cg_step``, which slab boxes
    cannot use).

    local:  ``SlabEvolution(split(state, P, g), cfg, g)``: all slabs in one
            context on this GPU.
    ranks:  ``SlabEvolution([my_slab], cfg, g, halo=DistHalo(g))``.
    """

    def __init__(self, slabs: list[BoxState], cfg: BoxConfig, ghost: int, halo=None):
        import torch

        cfg = replace(cfg, x_ghost=ghost)
        self.ev = Evolution(slabs, [cfg] * len(slabs))
        # the halo copies (or messages) and the kernels share one stream (not
        # the legacy default stream, which the library's handle 0 does not name)
        self.stream = torch.cuda.Stream()
        self.ev.set_stream(self.stream.cuda_stream)
        self.ghost = ghost
        self.halo = halo
        self.mixed = cfg.precision == "mixed"
        self.needs_kavg = cfg.lapse in KAVG_LAPSES
        self.local = LocalHalo(self.ev, ghost, self.mixed) if halo is None else None
        self.started = False
        if self.mixed:  # the whole box's uniform background in every slab
            if self.local is not None:
                self.local.background()
            else:
                self.halo.background(self.ev)

    def _exchange(self) -> None:
        import torch

        with torch.cuda.stream(self.stream):
            if self.local is not None:
                self.local.exchange()
            else:
                self.halo.exchange(self.ev, self.mixed)
            if self.needs_kavg:
                (self.local.kavg() if self.local is not None else self.halo.kavg(self.ev))

    def step(self, nsteps: int = 1) -> None:
        for _ in range(nsteps):
            if not self.started:
                self.ev.step_init()
                self.started = True
            for n in (1, 2, 3, 4):
                self._exchange()
                self.ev.rk_stage(n)

    def refresh(self) -> None:
        """Ghost planes of the next substep's input (before constraints)."""
        if not self.started:
            self.ev.step_init()
            self.started = True
        self._exchange()

    def download(self) -> list[BoxState]:
        return [self.ev.download(b) for b in range(len(self.ev.templates))]

    def close(self) -> None:
        self.ev.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


__all__ = ["ghost_width", "slab_bounds", "split", "assemble", "fill_ghosts", "background_sums", "set_background",
           "LocalHalo", "DistHalo", "SlabEvolution", "FLUX_ARRAYS", "KAVG_LAPSES"]
