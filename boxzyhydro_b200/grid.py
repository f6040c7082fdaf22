"""Grid geometry of the reference (init_grid.f90:7-265), vectorised.

Cell index (0-based) = ix + iy*nx + iz*nx*ny with ix fastest, the reference's
igrid-1.  Two ghost layers per side in x and y always, and in z only when
nz >= 6; with nz < 6 every z plane is interior and z neighbours are the cell
itself.  Boundary flag: 0 interior, 1 outer ghost layer, 2 inner ghost layer.
"""
from __future__ import annotations

import numpy as np


def index_grids(nx: int, ny: int, nz: int):
    """1-based (ix, iy, iz) arrays over all cells in reference order."""
    iz, iy, ix = np.meshgrid(np.arange(1, nz + 1), np.arange(1, ny + 1),
                             np.arange(1, nx + 1), indexing="ij")
    return ix.ravel(), iy.ravel(), iz.ravel()


def boundary_flags(nx: int, ny: int, nz: int) -> np.ndarray:
    """grid(:)%boundary as set by init_grid.f90:82-118."""
    ix, iy, iz = index_grids(nx, ny, nz)
    f1 = (ix == 1) | (ix == nx) | (iy == 1) | (iy == ny)
    f2 = (ix == 2) | (ix == nx - 1) | (iy == 2) | (iy == ny - 1)
    if nz >= 6:
        f1 |= (iz == 1) | (iz == nz)
        f2 |= (iz == 2) | (iz == nz - 1)
    b = np.zeros(nx * ny * nz, dtype=np.int32)
    b[f2] = 2
    b[f1] = 1
    return b


def cell_centres(nx, ny, nz, dx, dy, dz):
    """grid(:)%x,y,z (init_grid.f90:85,89,93): centred on the box middle."""
    ix, iy, iz = index_grids(nx, ny, nz)
    x = dx * (ix.astype(np.float64) - (float(nx) + 1.0) / 2.0)
    y = dy * (iy.astype(np.float64) - (float(ny) + 1.0) / 2.0)
    z = dz * (iz.astype(np.float64) - (float(nz) + 1.0) / 2.0)
    return x, y, z


def active_slices(nx, ny, nz):
    """Slices of a (nz,ny,nx) array that select the interior cells."""
    zs = slice(0, nz) if nz < 6 else slice(2, nz - 2)
    return zs, slice(2, ny - 2), slice(2, nx - 2)


def clamp_fill(field3d: np.ndarray, nz_ghosts: bool) -> np.ndarray:
    """Fill ghost layers of a (nz,ny,nx[,k]) array with the nearest interior
    value (zero-gradient).  This is what the reference's outflow ghost fill
    produces for every ghost cell."""
    f = field3d
    nz, ny, nx = f.shape[:3]
    f[:, :, 0] = f[:, :, 2]
    f[:, :, 1] = f[:, :, 2]
    f[:, :, nx - 1] = f[:, :, nx - 3]
    f[:, :, nx - 2] = f[:, :, nx - 3]
    f[:, 0] = f[:, 2]
    f[:, 1] = f[:, 2]
    f[:, ny - 1] = f[:, ny - 3]
    f[:, ny - 2] = f[:, ny - 3]
    if nz_ghosts:
        f[0] = f[2]
        f[1] = f[2]
        f[nz - 1] = f[nz - 3]
        f[nz - 2] = f[nz - 3]
    return f
