"""celldump files of the reference, as numpy arrays.

The reference writes its hydro snapshots with write_files.f90:55-63 and restarts
from them with read_hydro.f90:122-134: Fortran unformatted sequential files,
built with gfortran -frecord-marker=4 (Makefile:20), so every record is framed
by a little-endian int32 byte count on both sides:

    1  int32 readtest = 1234
    2  float64 time, int32 step
    3  8 x float64 units (derived_types.f90:14-15 order: length, time, mass,
       density, rgas, eps, kelvin, vel), from units.f90:10-17
    4.. one record per cell in reference order (x fastest):
       float64 x, y, z, rho, p, u1, u2, u3, phi, E, muc; int32 boundary

This module reads and writes that layout on the host (analysis scripts, and
the independent check of the library's bx_write_celldump/bx_read_celldump).
"""
from __future__ import annotations

import numpy as np

from . import grid as G

UNIT_NAMES = ("length", "time", "mass", "density", "rgas", "eps", "kelvin", "vel")
CELL_FIELDS = ("x", "y", "z", "rho", "p", "u1", "u2", "u3", "phi", "E", "muc")
CELL_RECORD = np.dtype([("n0", "<i4"), ("v", "<f8", (11,)), ("boundary", "<i4"), ("n1", "<i4")])
HEADER_BYTES = (4 + 4 + 4) + (4 + 12 + 4) + (4 + 64 + 4)


def units() -> np.ndarray:
    """The 8 units of units.f90:10-17 (constants of parameters.f90:7-11), in the
    record order of derived_types.f90:14-15."""
    pi, gcgs, rgas_cgs = 3.1415926535897931, 6.67e-8, 8.254e7
    length = 1.496e13
    time = (3600.0 * 365.25 * 24.0) / (2.0 * pi)
    density = 1.0 / (gcgs * (time * time))
    mass = density * (length * length * length)
    vel = length / time
    eps = vel * vel * mass / (length * length * length)
    kelvin = 1.0
    rgas = rgas_cgs / (vel * vel / kelvin)
    return np.array([length, time, mass, density, rgas, eps, kelvin, vel])


def write(path, time, step, x, y, z, rho, p, u, phi, E, muc, boundary, unit_values=None):
    """Write a celldump; per-cell arguments are arrays of ngrid (u: (ngrid, 3))."""
    ng = len(rho)
    cells = np.empty(ng, CELL_RECORD)
    cells["n0"] = 92
    cells["n1"] = 92
    v = cells["v"]
    for k, a in enumerate((x, y, z, rho, p)):
        v[:, k] = a
    v[:, 5:8] = u
    v[:, 8] = 0.0 if phi is None else phi
    v[:, 9] = E
    v[:, 10] = muc
    cells["boundary"] = boundary
    uv = units() if unit_values is None else np.asarray(unit_values, dtype="<f8")
    with open(path, "wb") as f:
        f.write(np.array([4, 1234, 4], "<i4").tobytes())
        f.write(np.array([12], "<i4").tobytes() + np.array([time], "<f8").tobytes()
                + np.array([step, 12], "<i4").tobytes())
        f.write(np.array([64], "<i4").tobytes() + uv.astype("<f8").tobytes()
                + np.array([64], "<i4").tobytes())
        f.write(cells.tobytes())


def read(path) -> dict:
    """Read a celldump into a dict of arrays (keys: time, step, readtest, units,
    the CELL_FIELDS, u (ngrid, 3) and boundary)."""
    raw = np.fromfile(path, dtype=np.uint8)
    hdr = raw[:HEADER_BYTES].tobytes()
    i4 = np.frombuffer(hdr, "<i4")
    if i4[0] != 4 or i4[2] != 4 or i4[3] != 12 or i4[7] != 12 or i4[8] != 64:
        raise ValueError(f"{path}: header records are not (int), (double, int), (8 doubles)")
    out = {"readtest": int(i4[1]),
           "time": float(np.frombuffer(hdr[16:24], "<f8")[0]),
           "step": int(np.frombuffer(hdr[24:28], "<i4")[0]),
           "units": np.frombuffer(hdr[36:100], "<f8").copy()}
    body = raw[HEADER_BYTES:]
    if body.size % CELL_RECORD.itemsize:
        raise ValueError(f"{path}: cell records are not 100-byte (92 + markers) records")
    cells = np.frombuffer(body.tobytes(), CELL_RECORD)
    if np.any(cells["n0"] != 92) or np.any(cells["n1"] != 92):
        raise ValueError(f"{path}: a cell record has a length other than 92 bytes")
    for k, name in enumerate(CELL_FIELDS):
        out[name] = cells["v"][:, k].copy()
    out["u"] = cells["v"][:, 5:8].copy()
    out["boundary"] = cells["boundary"].copy()
    return out


def from_arrays(params, cons, u, p, time, step, phi=None, path=None):
    """The celldump write_files would write for reference arrays that state() has
    already updated (cons (ngrid,5), u (ngrid,3), p (ngrid,))."""
    x, y, z = G.cell_centres(params.nx, params.ny, params.nz, params.dx, params.dy, params.dz)
    b = G.boundary_flags(params.nx, params.ny, params.nz)
    muc = np.full(params.ngrid, params.muc)
    if path is not None:
        write(path, time, step, x, y, z, cons[:, 0], p, u, phi, cons[:, 4], muc, b)
    return dict(x=x, y=y, z=z, rho=cons[:, 0], p=p, u=u, E=cons[:, 4], muc=muc, boundary=b)


def restart_arrays(params, d):
    """read_hydro.f90:122-180 on a read celldump: (cons, u, p) before its state()
    call -- m = u*rho, adindx = gammafix, the outermost layer reset."""
    ng = params.ngrid
    cons = np.empty((ng, 5))
    cons[:, 0] = d["rho"]
    cons[:, 4] = d["E"]
    u = d["u"].copy()
    cons[:, 1:4] = u * cons[:, 0:1]
    b = G.boundary_flags(params.nx, params.ny, params.nz)
    outer = b == 1
    cons[outer, 0] = params.small_rho
    cons[outer, 1:4] = 0.0
    cons[outer, 4] = params.small_eps
    return cons, u, d["p"].copy()


__all__ = ["UNIT_NAMES", "CELL_FIELDS", "units", "write", "read", "from_arrays",
           "restart_arrays"]
