"""Initial conditions for the hydro step.

The reference sets its initial state in init_conditions() (a user-edited file;
ICFILES/ holds variants).  Every generator here returns the reference's global
arrays in the reference layout -- cons (ng,5), u (ng,3), p (ng,), adindx (ng,) --
together with the HydroParams of the run, so the same arrays can be handed to
the GPU path (bx_upload) and to any checker.

* `sod_reference`: init_conditions.f90:26-77 verbatim in meaning (split on y<0,
  outer ghost layer set to small_rho / small_eps).
* `sod_x`: the 512x4x4-interior Sod tube split on x at the box centre.
* `turbulent_box`: seeded lognormal density and solenoidal velocity (power
  spectrum k^-2), uniform pressure, outflow walls.
* `riemann_box`: one Riemann problem along a chosen axis (batched ensemble).
"""
from __future__ import annotations

import dataclasses

import numpy as np

from . import grid as G
from .params import HydroParams


@dataclasses.dataclass
class State:
    params: HydroParams
    cons: np.ndarray      # (ng,5)
    u: np.ndarray         # (ng,3)
    p: np.ndarray         # (ng,)
    adindx: np.ndarray    # (ng,)

    def copy(self):
        return State(dataclasses.replace(self.params), self.cons.copy(), self.u.copy(),
                     self.p.copy(), self.adindx.copy())


def sod_reference(params: HydroParams, axis: str = "y", x0: float = 0.0,
                  left=(1.0, 1.0), right=(0.125, 0.1)) -> State:
    """init_conditions.f90:26-77: (rho,p)=left where coordinate<x0, else right;
    v=0; E=p/(gamma-1); then the outer ghost layer (boundary 1) is set to
    rho=small_rho, m=0, E=small_eps while p keeps its value."""
    hp = params
    ng = hp.ngrid
    x, y, z = G.cell_centres(hp.nx, hp.ny, hp.nz, hp.dx, hp.dy, hp.dz)
    coord = {"x": x, "y": y, "z": z}[axis]
    lm = coord < x0
    cons = np.zeros((ng, 5))
    p = np.where(lm, left[1], right[1]).astype(np.float64)
    adindx = np.full(ng, hp.gammafix)
    cons[:, 0] = np.where(lm, left[0], right[0])
    cons[:, 4] = p / (adindx - 1.0)
    u = np.zeros((ng, 3))
    b = G.boundary_flags(hp.nx, hp.ny, hp.nz)
    ob = b == 1
    cons[ob, 0] = hp.small_rho
    cons[ob, 1:4] = 0.0
    cons[ob, 4] = hp.small_eps
    return State(hp, cons, u, p, adindx)


def sod_params(n_active: int = 512, ny: int = 8, nz: int = 4, gamma: float = 1.4,
               cfl: float = 0.1) -> HydroParams:
    """Sod tube with n_active interior cells along x, reflective walls,
    cell size 1/n_active, reference hydro defaults of in.nml.sod."""
    d = 1.0 / n_active
    return HydroParams(nx=n_active + 4, ny=ny, nz=nz, dx=d, dy=d, dz=d, cfl=cfl,
                       small_rho=1e-12, small_eps=1e-40, vlimit=10.0, gammafix=gamma,
                       h2stat=-1, endtime=0.2)


def sod_x(n_active: int = 512, ny: int = 8, nz: int = 4, gamma: float = 1.4) -> State:
    """Sod shock tube split on x at the box centre (x=0.5 of [0,1])."""
    return sod_reference(sod_params(n_active, ny, nz, gamma), axis="x")


def shipped_sod_params() -> HydroParams:
    """The reference's shipped in.nml (8x200x1, dx=0.01, gamma=1.4, t=0.4)."""
    return HydroParams(nx=8, ny=200, nz=1, dx=0.01, dy=0.01, dz=0.01, small_rho=1e-12,
                       small_eps=1e-40, vlimit=10.0, endtime=0.4, dtout=4.0,
                       gammafix=1.4, h2stat=-1, starttime=0.0)


def _grf(rng, shape, slope=-2.0):
    """Unit-variance Gaussian random field with power spectrum P(k) ~ k^slope."""
    white = rng.standard_normal(shape)
    fk = np.fft.rfftn(white)
    k = _kmag(shape)
    amp = np.zeros_like(k)
    nz = k > 0
    amp[nz] = k[nz] ** (slope / 2.0)
    fk *= amp
    f = np.fft.irfftn(fk, s=shape, axes=(0, 1, 2))
    f -= f.mean()
    f /= f.std()
    return f


def _kvec(shape):
    kz = np.fft.fftfreq(shape[0]) * shape[0]
    ky = np.fft.fftfreq(shape[1]) * shape[1]
    kx = np.fft.rfftfreq(shape[2]) * shape[2]
    return np.meshgrid(kz, ky, kx, indexing="ij")


def _kmag(shape):
    kz, ky, kx = _kvec(shape)
    return np.sqrt(kx * kx + ky * ky + kz * kz)


def _solenoidal(rng, shape, slope=-2.0):
    """Divergence-free Gaussian vector field, P(k) ~ k^slope, components (vx,vy,vz).
    The Nyquist planes of an even grid (a wavenumber component of n/2) carry no
    field: a real field's mode there has no spectral derivative, so the
    projection cannot make it divergence-free."""
    kz, ky, kx = _kvec(shape)
    k2 = kx * kx + ky * ky + kz * kz
    k2[0, 0, 0] = 1.0
    amp = np.where(k2 > 0, np.sqrt(k2) ** (slope / 2.0), 0.0)
    amp[0, 0, 0] = 0.0
    for kc, n in ((kz, shape[0]), (ky, shape[1]), (kx, shape[2])):
        if n % 2 == 0:
            amp[np.abs(kc) == n // 2] = 0.0
    comps = [np.fft.rfftn(rng.standard_normal(shape)) * amp for _ in range(3)]
    vx, vy, vz = comps
    div = (kx * vx + ky * vy + kz * vz) / k2
    vx = vx - kx * div
    vy = vy - ky * div
    vz = vz - kz * div
    return [np.fft.irfftn(c, s=shape, axes=(0, 1, 2)) for c in (vx, vy, vz)]


def turbulent_params(n: int = 256, gamma: float = 1.6666666666666667, cfl: float = 0.4):
    d = 1.0 / n
    nz = n + 4 if n + 4 >= 6 else n
    return HydroParams(nx=n + 4, ny=n + 4, nz=nz, dx=d, dy=d, dz=d, cfl=cfl,
                       small_rho=1e-12, small_eps=1e-40, vlimit=10.0, gammafix=gamma,
                       h2stat=-1, no_outflow_xl=False, no_outflow_xr=False,
                       no_outflow_yl=False, no_outflow_yr=False, no_outflow_zl=False,
                       no_outflow_zr=False, endtime=1e30)


def _assemble(hp: HydroParams, rho3, v3, p3) -> State:
    """Interior fields (nz,ny,nx) -> full arrays, ghosts filled by zero-gradient
    copies (what outflow ghost filling produces), m = v*rho, u = m/rho,
    E = p/(gamma-1) + rho*0.5*|u|^2 (state.f90:32 ordering)."""
    nx, ny, nz = hp.nx, hp.ny, hp.nz
    zs, ys, xs = G.active_slices(nx, ny, nz)
    full = np.zeros((nz, ny, nx, 5))
    full[zs, ys, xs, 0] = rho3
    full[zs, ys, xs, 1] = v3[0]
    full[zs, ys, xs, 2] = v3[1]
    full[zs, ys, xs, 3] = v3[2]
    full[zs, ys, xs, 4] = p3
    G.clamp_fill(full, nz >= 6)
    rho = full[..., 0].ravel()
    p = full[..., 4].ravel().copy()
    cons = np.zeros((hp.ngrid, 5))
    cons[:, 0] = rho
    for d in range(3):
        cons[:, 1 + d] = full[..., 1 + d].ravel() * rho
    u = cons[:, 1:4] / cons[:, 0:1]
    ekin = rho * 0.5 * (u[:, 0] * u[:, 0] + u[:, 1] * u[:, 1] + u[:, 2] * u[:, 2])
    cons[:, 4] = p / (hp.gammafix - 1.0) + ekin
    adindx = np.full(hp.ngrid, hp.gammafix)
    return State(hp, cons, np.ascontiguousarray(u), p, adindx)


def turbulent_box(n: int = 256, seed: int = 1234, sigma_ln: float = 0.5, mach: float = 1.0,
                  gamma: float = 1.6666666666666667, cfl: float = 0.4) -> State:
    """Lognormal density rho = exp(sigma*g - sigma^2/2) with g a unit-variance
    k^-2 Gaussian random field; uniform p=1; solenoidal k^-2 velocity scaled so
    the 3-D RMS speed equals mach * sqrt(gamma*p/<rho>)."""
    hp = turbulent_params(n, gamma, cfl)
    rng = np.random.default_rng(seed)
    shape = (n, n, n)
    g = _grf(rng, shape)
    rho = np.exp(sigma_ln * g - 0.5 * sigma_ln * sigma_ln)
    v = _solenoidal(rng, shape)
    vrms = np.sqrt(np.mean(v[0] ** 2 + v[1] ** 2 + v[2] ** 2))
    cs = np.sqrt(gamma * 1.0 / rho.mean())
    v = [c * (mach * cs / vrms) for c in v]
    p = np.ones(shape)
    return _assemble(hp, rho, v, p)


def sod_blob_box(n: int = 128, seed: int = 4, amp: float = 0.05, width: float = 0.08,
                 gamma: float = 1.6666666666666667, cfl: float = 0.4, blob: bool = True) -> State:
    """Sod state split on x at the box centre ((rho,p) = (1,1) | (0.125,0.1), v=0) in
    an n^3-interior box with outflow walls, times a seeded Gaussian density blob
    rho *= 1 + amp*exp(-|r-r0|^2/(2 width^2)) with r0 uniform in [0.3,0.7]^3 of the
    unit box (pressure unchanged).  blob=False gives the unperturbed state."""
    hp = turbulent_params(n, gamma, cfl)
    rng = np.random.default_rng(seed)
    r0 = rng.uniform(0.3, 0.7, 3)
    c = (np.arange(n) + 0.5) / n
    zz, yy, xx = np.meshgrid(c, c, c, indexing="ij")
    rho = np.where(xx < 0.5, 1.0, 0.125)
    p = np.where(xx < 0.5, 1.0, 0.1)
    if blob:
        r2 = (xx - r0[0]) ** 2 + (yy - r0[1]) ** 2 + (zz - r0[2]) ** 2
        rho = rho * (1.0 + amp * np.exp(-r2 / (2.0 * width * width)))
    v = [np.zeros((n, n, n)) for _ in range(3)]
    return _assemble(hp, rho, v, p)


def riemann_params(side: int, gamma: float, cfl: float = 0.1) -> HydroParams:
    d = 1.0 / side
    return HydroParams(nx=side + 4, ny=side + 4, nz=side + 4, dx=d, dy=d, dz=d, cfl=cfl,
                       small_rho=1e-12, small_eps=1e-40, vlimit=10.0, gammafix=gamma,
                       h2stat=-1, no_outflow_xl=False, no_outflow_xr=False,
                       no_outflow_yl=False, no_outflow_yr=False, no_outflow_zl=False,
                       no_outflow_zr=False, endtime=1e30)


def riemann_box(side: int, axis: int, left, right, gamma: float, cfl: float = 0.1) -> State:
    """One Riemann problem: (rho, v_normal, p) = left where the coordinate along
    `axis` (0=x,1=y,2=z) is below the box centre, else right; outflow walls."""
    hp = riemann_params(side, gamma, cfl)
    n = side
    coord = np.arange(n) - (n - 1) / 2.0
    shp = [1, 1, 1]
    shp[2 - axis] = n
    c = np.broadcast_to(coord.reshape(shp), (n, n, n))
    lm = c < 0
    rho = np.where(lm, left[0], right[0]).astype(np.float64)
    vn = np.where(lm, left[1], right[1]).astype(np.float64)
    p = np.where(lm, left[2], right[2]).astype(np.float64)
    v = [np.zeros((n, n, n)) for _ in range(3)]
    v[axis] = vn
    return _assemble(hp, rho, v, p)


def riemann_box_cons(side: int, axis: int, left, right, gamma: float) -> np.ndarray:
    """cons (ng,5) of `riemann_box` built from a 1-D profile (same values, far
    fewer temporaries): every cell equals the interior cell nearest to it along
    `axis`, which is also what the outflow ghost fill gives the ghosts."""
    n = side
    N = n + 4
    idx = np.clip(np.arange(N) - 2, 0, n - 1)
    lm = (idx - (n - 1) / 2.0) < 0
    rho = np.where(lm, left[0], right[0]).astype(np.float64)
    vn = np.where(lm, left[1], right[1]).astype(np.float64)
    p = np.where(lm, left[2], right[2]).astype(np.float64)
    prof = np.zeros((N, 5))
    prof[:, 0] = rho
    prof[:, 1 + axis] = vn * rho
    u = prof[:, 1:4] / prof[:, 0:1]
    ekin = rho * 0.5 * (u[:, 0] * u[:, 0] + u[:, 1] * u[:, 1] + u[:, 2] * u[:, 2])
    prof[:, 4] = p / (gamma - 1.0) + ekin
    shp = [1, 1, 1, 5]
    shp[2 - axis] = N
    full = np.broadcast_to(prof.reshape(shp), (N, N, N, 5))
    return np.ascontiguousarray(full).reshape(N * N * N, 5)


def riemann_ensemble_spec(nbox: int = 4096, seed: int = 2024, sides=(32, 48, 64, 96)):
    """Seeded per-box draws: side, axis, gamma, left and right (rho, v, p)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(nbox):
        side = int(rng.choice(sides))
        axis = int(rng.integers(0, 3))
        gamma = float(rng.choice([1.4, 1.6666666666666667]))
        lr = []
        for _ in range(2):
            rho = float(np.exp(rng.uniform(np.log(0.1), np.log(10.0))))
            pr = float(np.exp(rng.uniform(np.log(0.1), np.log(10.0))))
            vn = float(rng.uniform(-1.0, 1.0))
            lr.append((rho, vn, pr))
        out.append(dict(side=side, axis=axis, gamma=gamma, left=lr[0], right=lr[1]))
    return out
