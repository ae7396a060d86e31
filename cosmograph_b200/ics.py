"""Initial data for periodic BSSN boxes (host side, FP64, numpy).

Initial data is built once on the host and is not part of the timed path.
Three families:

* `sinusoid_dust` -- a single-mode perturbation of a dust FRW box, following
  the reference's sinusoid construction (components/static/static_ic.cc:287-401)
  loaded into the conserved dust density D = e^{6 phi} rho the way
  `dust_ic_set_random` stores it (components/dust_fluid/dust_ic.cc:135).
* `grf_dust` -- a seeded Gaussian random density field turned into
  synchronous-gauge BSSN + dust data by the steps of `dust_ic_set_random`
  (components/dust_fluid/dust_ic.cc:23-140) with the spectral inverse
  Laplacian of `Fourier::inverseLaplacian` (utils/Fourier.h:251-298).
* `grf_scalar` -- a homogeneous scalar field plus a seeded Gaussian random
  fluctuation, psi_i = d_i phi and K from the local energy density.
* `perturbed` -- every field perturbed by a few smooth random periodic modes;
  not physical, used to exercise every term of the right-hand side.
"""
from __future__ import annotations

import math

import numpy as np

from .state import BSSN_FIELDS, DUST, SCALAR, STATIC, VACUUM, BoxState, field_names

PI = math.pi
RHO_FRW = 3.0 / PI / 8.0        # dust_ic.cc:29, H0 = 1


def default_dt(dx: float, dt_frac: float = 0.1) -> float:
    """dt = dt_frac * dx evaluated in long double and rounded to double, as
    cosmo.cc:41-42 does with stold()."""
    return float(np.longdouble(str(dt_frac)) * np.longdouble(dx))


# ---------------------------------------------------------------------------
# periodic finite differences (utils/math.h:74-1085), axis a = 0, 1, 2
# ---------------------------------------------------------------------------

def _sh(f: np.ndarray, a: int, n: int) -> np.ndarray:
    """f at offset +n along axis a (periodic)."""
    return np.roll(f, -n, axis=a)


def derivative(f: np.ndarray, a: int, dx: float, order: int) -> np.ndarray:
    V = lambda n: _sh(f, a, n)  # noqa: E731
    if order == 2:
        return (-1.0 / 2.0 * V(-1) + 1.0 / 2.0 * V(1)) / dx
    if order == 4:
        return (+1.0 / 12.0 * V(-2) - 2.0 / 3.0 * V(-1) + 2.0 / 3.0 * V(1) - 1.0 / 12.0 * V(2)) / dx
    if order == 6:
        return (-1.0 / 60.0 * V(-3) + 3.0 / 20.0 * V(-2) - 3.0 / 4.0 * V(-1) + 3.0 / 4.0 * V(1)
                - 3.0 / 20.0 * V(2) + 1.0 / 60.0 * V(3)) / dx
    return ((1.0 / 280.0 * V(-4) - 1.0 / 280.0 * V(4)) - (4.0 / 105.0 * V(-3) - 4.0 / 105.0 * V(3))
            + (1.0 / 5.0 * V(-2) - 1.0 / 5.0 * V(2)) - (4.0 / 5.0 * V(-1) - 4.0 / 5.0 * V(1))) / dx


def double_derivative(f: np.ndarray, a: int, b: int, dx: float, order: int) -> np.ndarray:
    if a == b:
        V = lambda n: _sh(f, a, n)  # noqa: E731
        if order == 2:
            return (V(-1) - 2.0 * V(0) + V(1)) / dx / dx
        if order == 4:
            return (-1.0 / 12.0 * V(-2) + 4.0 / 3.0 * V(-1) - 5.0 / 2.0 * V(0) + 4.0 / 3.0 * V(1)
                    - 1.0 / 12.0 * V(2)) / dx / dx
        if order == 6:
            return (1.0 / 90.0 * V(-3) - 3.0 / 20.0 * V(-2) + 3.0 / 2.0 * V(-1) - 49.0 / 18.0 * V(0)
                    + 3.0 / 2.0 * V(1) - 3.0 / 20.0 * V(2) + 1.0 / 90.0 * V(3)) / dx / dx
        return (-1.0 / 560.0 * V(-4) + 8.0 / 315.0 * V(-3) - 1.0 / 5.0 * V(-2) + 8.0 / 5.0 * V(-1)
                - 205.0 / 72.0 * V(0) + 8.0 / 5.0 * V(1) - 1.0 / 5.0 * V(2) + 8.0 / 315.0 * V(3)
                - 1.0 / 560.0 * V(4)) / dx / dx
    a, b = min(a, b), max(a, b)

    def P(n):
        s = lambda p, q: np.roll(np.roll(f, -p, axis=a), -q, axis=b)  # noqa: E731
        return -s(n, -n) + s(n, n) + s(-n, -n) - s(-n, n)

    if order == 2:
        return P(1) / 4.0 / dx / dx
    if order == 4:
        return (P(1) - 1.0 / 16.0 * P(2)) / 3.0 / dx / dx
    if order == 6:
        return (135.0 * P(1) - 27.0 / 2.0 * P(2) + P(3)) / 360.0 / dx / dx
    return (2.0 / 5.0 * P(1) - 1.0 / 20.0 * P(2) + 2.0 / 315.0 * P(3) - 1.0 / 2240.0 * P(4)) / dx / dx


def laplacian(f, dx, order):
    return (double_derivative(f, 0, 0, dx, order) + double_derivative(f, 1, 1, dx, order)
            + double_derivative(f, 2, 2, dx, order))


def _kgrid(shape):
    nx, ny, nz = shape
    px = np.fft.fftfreq(nx) * nx
    py = np.fft.fftfreq(ny) * ny
    pz = np.fft.rfftfreq(nz) * nz
    return np.meshgrid(px, py, pz, indexing="ij")


def inverse_laplacian(f: np.ndarray, box_len: float) -> np.ndarray:
    """Spectral inverse Laplacian with the zero mode removed
    (utils/Fourier.h:251-298)."""
    px, py, pz = _kgrid(f.shape)
    p2 = (px ** 2 + py ** 2 + pz ** 2) * (2.0 * PI / box_len) ** 2
    fk = np.fft.rfftn(f, axes=(0, 1, 2))
    with np.errstate(divide="ignore", invalid="ignore"):
        fk = fk / (-p2)
    fk[0, 0, 0] = 0.0
    return np.fft.irfftn(fk, s=f.shape, axes=(0, 1, 2))


def gaussian_random_field(shape, seed: int, spectrum, rms: float) -> np.ndarray:
    """Zero-mean Gaussian random field with power spectrum `spectrum(k)`
    (k in units of the fundamental mode), normalised to the given rms."""
    rng = np.random.Generator(np.random.MT19937(seed))
    px, py, pz = _kgrid(shape)
    k = np.sqrt(px ** 2 + py ** 2 + pz ** 2)
    with np.errstate(divide="ignore", invalid="ignore"):
        amp = np.sqrt(np.where(k > 0, spectrum(np.maximum(k, 1e-30)), 0.0))
    noise = rng.standard_normal(k.shape) + 1j * rng.standard_normal(k.shape)
    field = np.fft.irfftn(amp * noise, s=shape, axes=(0, 1, 2))
    field -= field.mean()
    s = field.std()
    return field * (rms / s) if s > 0 else field


def _empty(shape, matter, dx, dt, z4c: bool = False, shift: bool = False, **kw) -> BoxState:
    return BoxState(fields=np.zeros((len(field_names(matter, z4c, shift)),) + tuple(shape)), matter=matter,
                    dx=dx, dt=dt, z4c=z4c, shift=shift, **kw)


# ---------------------------------------------------------------------------
# initial data families
# ---------------------------------------------------------------------------

def sinusoid_dust(n: int, box_len: float = 1.0, peak_amplitude_frac: float = 1.0e-3,
                  omega_l: float = 0.0, phix: float = 0.0, dt_frac: float = 0.1) -> BoxState:
    """Single-mode dust box (static_ic.cc:287-401 in dust form).  The FRW
    reference stays trivial (the dust sim never sets it, bssn.cc:25), so DIFFK
    and D carry the full K and density."""
    dx = box_len / n
    st = _empty((n, n, n), DUST, dx, default_dt(dx, dt_frac))
    rho_m = (1.0 - omega_l) * RHO_FRW
    st.lam = omega_l * RHO_FRW
    A = box_len * box_len * peak_amplitude_frac
    twopi_L = 2.0 * PI / box_len
    x = np.arange(n, dtype=np.float64) / n
    phi1 = A * np.sin(2.0 * PI * x + phix)
    drho1 = -np.exp(-4.0 * phi1) / PI / 2.0 * ((twopi_L * A * np.cos(2.0 * PI * x + phix)) ** 2
                                               - twopi_L * twopi_L * A * np.sin(2.0 * PI * x + phix))
    phi = np.broadcast_to(phi1[:, None, None], (n, n, n))
    rho = rho_m + np.broadcast_to(drho1[:, None, None], (n, n, n))
    if rho.min() < 0.0:
        raise ValueError("negative density in some regions")
    st.field("DIFFphi")[...] = phi
    st.field("DIFFK")[...] = -math.sqrt(24.0 * PI * RHO_FRW)
    st.field("D")[...] = np.exp(6.0 * phi) * rho
    return st


def grf_dust(n, seed: int = 9, rms_delta: float = 1.0e-4, order: int = 4, box_len: float = 1.0,
             omega_l: float = 1.0e-6, ns: float = 0.96, dt_frac: float = 0.1) -> BoxState:
    """Synchronous-gauge BSSN + dust from a Gaussian random density field,
    P(k) ~ k^ns T(k)^2 with T a Gaussian cutoff at k = N/4, by the steps of
    dust_ic_set_random (components/dust_fluid/dust_ic.cc:59-136)."""
    shape = (n, n, n) if np.isscalar(n) else tuple(n)
    nmin = min(shape)
    dx = box_len / shape[0]
    st = _empty(shape, DUST, dx, default_dt(dx, dt_frac))
    rho_L = omega_l * RHO_FRW
    st.lam = rho_L
    kc = nmin / 4.0
    delta = gaussian_random_field(shape, seed, lambda k: k ** ns * np.exp(-(k / kc) ** 2), rms_delta)
    # Newtonian potential: lap Phi_N = 4 pi rho_FRW delta = (3/2) delta
    phi_N = inverse_laplacian(1.5 * delta, box_len)
    lap_phi_N = laplacian(phi_N, dx, order)
    dphi = np.log1p(-10.0 / 3.0 * phi_N) / 4.0                       # dust_ic.cc:70
    dK = -3.0 * (1.0 + 2.0 * phi_N) + 2.0 / 3.0 * lap_phi_N         # dust_ic.cc:71
    e6p = np.exp(6.0 * dphi)
    W = []
    for a in range(3):                                               # dust_ic.cc:76-95
        inv = inverse_laplacian(e6p * derivative(dK, a, dx, order), box_len)
        W.append(-derivative(phi_N, a, dx, order) / 3.0 + inv / 2.0)
    c = np.exp(-6.0 * dphi)                                           # dust_ic.cc:98-114
    DkWk = sum(derivative(W[a], a, dx, order) for a in range(3))
    Aij = {}
    for i in range(3):
        for j in range(i, 3):
            v = derivative(W[j], i, dx, order) + derivative(W[i], j, dx, order) \
                + 2.0 / 3.0 * double_derivative(phi_N, i, j, dx, order)
            if i == j:
                v = v - 2.0 / 3.0 * DkWk - 2.0 / 9.0 * lap_phi_N
            Aij[(i, j)] = c * v
    AijAij = (Aij[0, 0] ** 2 + Aij[1, 1] ** 2 + Aij[2, 2] ** 2
              + 2.0 * (Aij[0, 1] ** 2 + Aij[0, 2] ** 2 + Aij[1, 2] ** 2))
    lap_e_p = np.exp(dphi) * (laplacian(dphi, dx, order)
                              + sum(derivative(dphi, a, dx, order) ** 2 for a in range(3)))
    rho_ADM = 1.0 / 2.0 / PI * (dK * dK / 12.0 - AijAij / 8.0 - np.exp(-5.0 * dphi) * lap_e_p)
    rho_0 = rho_ADM - rho_L
    if rho_0.min() < 0.0:
        raise ValueError("negative density in some regions")
    st.field("DIFFphi")[...] = dphi
    st.field("DIFFK")[...] = dK
    for (i, j), v in Aij.items():
        st.field(f"A{i + 1}{j + 1}")[...] = v
    st.field("D")[...] = e6p * rho_0
    return st


def grf_dust_gpu(n, seed: int = 9, rms_delta: float = 1.0e-4, order: int = 4, box_len: float = 1.0,
                 omega_l: float = 1.0e-6, ns: float = 0.96, dt_frac: float = 0.1, delta=None,
                 host_delta: bool = False) -> BoxState:
    """grf_dust built on the GPU (cg_ic_grf_dust): the same construction with
    cuFFT inverse Laplacians.  The random field comes from the GPU's own
    generator unless `delta` is given; host_delta=True draws it on the host
    exactly as grf_dust does, so the result equals grf_dust's to rounding."""
    from .evolution import BoxConfig, Evolution

    shape = (n, n, n) if np.isscalar(n) else tuple(n)
    if host_delta and delta is None:
        kc = min(shape) / 4.0
        delta = gaussian_random_field(shape, seed, lambda k: k ** ns * np.exp(-(k / kc) ** 2), rms_delta)
    dx = box_len / shape[0]
    st = _empty(shape, DUST, dx, default_dt(dx, dt_frac))
    st.lam = omega_l * RHO_FRW
    with Evolution(st, BoxConfig(order=order)) as ev:
        ev.ic_grf_dust(0, seed=seed, rms_delta=rms_delta, ns=ns, cutoff=min(shape) / 4.0, delta=delta)
        out = ev.download(0)
    out.step = 0
    return out


def grf_scalar(n, seed: int = 9, phi0: float = 1.0e-2, rms: float = 1.0e-5, mass: float = 1.0,
               order: int = 8, box_len: float = 1.0, dt_frac: float = 0.1) -> BoxState:
    """BSSN + scalar field: phi = phi0 + a Gaussian random fluctuation with a
    k^-3 spectrum cut off at N/4, Pi = 0, psi_i = d_i phi (the relation the
    reference's wave data sets, components/scalar/scalar_ic.cc:43-48), and
    K = -sqrt(24 pi rho) from the local energy density with V = m^2 phi^2 / 2."""
    shape = (n, n, n) if np.isscalar(n) else tuple(n)
    dx = box_len / shape[0]
    st = _empty(shape, SCALAR, dx, default_dt(dx, dt_frac))
    kc = min(shape) / 4.0
    dphi = gaussian_random_field(shape, seed, lambda k: np.where(k <= kc, k ** -3.0, 0.0), rms)
    phi = phi0 + dphi
    st.field("phi")[...] = phi
    grad2 = 0.0
    for a in range(3):
        d = derivative(phi, a, dx, order)
        st.field(f"psi{a + 1}")[...] = d
        grad2 = grad2 + d * d
    rho = 0.5 * mass * mass * phi * phi + 0.5 * grad2
    st.field("DIFFK")[...] = -np.sqrt(24.0 * PI * rho)
    return st


def grf_scalar_gpu(n, seed: int = 9, phi0: float = 1.0e-2, rms: float = 1.0e-5, mass: float = 1.0,
                   order: int = 8, box_len: float = 1.0, dt_frac: float = 0.1, dphi=None,
                   host_field: bool = False) -> BoxState:
    """grf_scalar built on the GPU (cg_ic_grf_scalar).  The fluctuation comes
    from the GPU's own generator unless `dphi` is given; host_field=True draws
    it on the host exactly as grf_scalar does, so the result equals
    grf_scalar's to rounding."""
    from .evolution import BoxConfig, Evolution

    shape = (n, n, n) if np.isscalar(n) else tuple(n)
    kc = min(shape) / 4.0
    if host_field and dphi is None:
        dphi = gaussian_random_field(shape, seed, lambda k: np.where(k <= kc, k ** -3.0, 0.0), rms)
    dx = box_len / shape[0]
    st = _empty(shape, SCALAR, dx, default_dt(dx, dt_frac))
    with Evolution(st, BoxConfig(order=order)) as ev:
        ev.ic_grf_scalar(0, seed=seed, phi0=phi0, rms=rms, mass=mass, cutoff=kc, dphi=dphi)
        out = ev.download(0)
    out.step = 0
    return out


def perturbed(shape, matter: int, seed: int = 1, amp: float = 1.0e-2, modes: int = 3,
              box_len: float = 1.0, dt_frac: float = 0.1, z4c: bool = False,
              shift: bool = False) -> BoxState:
    """Every field = background + amp * (a few random smooth periodic modes,
    each a product of one sine per axis).  Backgrounds: DIFFK = -3,
    D = 3/(8 pi), alpha = 1 (DIFFalpha = 0), scalar phi = 0.1; everything
    else 0 (with z4c, theta too; with the shift, beta^i, auxB^i and expN,
    beta^i at ten times the amplitude, so that the advection terms of both
    signs matter).  Not a solution of the constraints: it
    exercises every term of the right-hand side."""
    shape = tuple(shape)
    dx = box_len / shape[0]
    st = _empty(shape, matter, dx, default_dt(dx, dt_frac), z4c=z4c, shift=shift)
    rng = np.random.Generator(np.random.MT19937(seed))
    x = [np.arange(m, dtype=np.float64) / m for m in shape]
    for f, name in enumerate(st.names):
        v = np.zeros(shape)
        for _ in range(modes):
            a = rng.uniform(-1, 1)
            s1 = [np.sin(2 * PI * int(rng.integers(0, 3)) * xi + rng.uniform(0, 2 * PI)) for xi in x]
            v += (a * s1[0])[:, None, None] * s1[1][None, :, None] * s1[2][None, None, :]
        v *= amp / modes
        base = {"DIFFK": -3.0, "D": RHO_FRW, "phi": 0.1}.get(name, 0.0)
        if name in ("D", "S1", "S2", "S3", "DIFFD"):
            v = RHO_FRW * v            # keep the density positive
        if matter == STATIC and name == "DIFFK":
            base = 0.0                 # K sits in the FRW background
        if name.startswith("beta"):
            v = 10.0 * v
        st.fields[f] = base + v
    if matter in (DUST, STATIC):
        st.lam = 1.0e-6 * RHO_FRW
    if matter == STATIC:
        # the static sims' FRW background: one pressureless fluid at the
        # density of H = 1, K = -3 (FRW::addFluid, utils/FRW.h:60-76)
        st.fluids = ((RHO_FRW, 0.0),)
        st.frw_K = -3.0
    return st


__all__ = ["sinusoid_dust", "grf_dust", "grf_scalar", "grf_scalar_gpu", "perturbed", "derivative",
           "double_derivative", "laplacian", "inverse_laplacian", "default_dt",
           "gaussian_random_field", "BSSN_FIELDS", "VACUUM", "DUST", "SCALAR", "STATIC"]
