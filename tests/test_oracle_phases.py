"""The oracle's per-phase subroutines against numpy restatements of the
reference's formulas, bit for bit (the same operations in the same order):
state() with the stale velocity and its low-density branch (state.f90:29-59),
velocity() with the limiter (velocity.f90:18-53), courant() over every cell
including ghosts (courant.f90:17-29) and source() with a force on the interior
cells (source.f90:148-191)."""
import numpy as np
import pytest

import oracle as O
from boxzyhydro_b200 import grid as G
from tests.helpers import small_random_box


@pytest.fixture
def box():
    st = small_random_box(nx=11, ny=10, nz=9, walls=(0,) * 6, seed=13, amp=0.4)
    return st


def fresh(st, u=None, p=None):
    hp = st.params
    o = O.Oracle(hp)
    o.set_state(st.cons, st.u if u is None else u, st.p if p is None else p,
                np.full(hp.ngrid, hp.gammafix))
    return o


def test_state_uses_the_stale_velocity_and_the_low_density_branch(box):
    hp = box.params
    rng = np.random.default_rng(1)
    cons = box.cons.copy()
    low = rng.random(hp.ngrid) < 0.2
    cons[low, 0] = 10.0 ** rng.uniform(-7, -4.5, low.sum())  # below 1e-4
    u_stale = box.u * 0.9 + 0.01  # not m/rho: state() must use this array
    p_in = np.abs(box.p) + 0.1
    o = O.Oracle(hp)
    o.set_state(cons, u_stale, p_in, np.full(hp.ngrid, hp.gammafix))
    o.state()
    c1, _, p1, g1 = o.get_state()
    o.close()
    gam, mu, R = hp.gammafix, hp.muc, hp.rgas
    ekin = cons[:, 0] * 0.5 * (u_stale[:, 0] * u_stale[:, 0] + u_stale[:, 1] * u_stale[:, 1] +
                               u_stale[:, 2] * u_stale[:, 2])
    eps = np.maximum(cons[:, 4] - ekin, hp.small_eps)
    p_want = eps * (gam - 1.0)
    e_want = cons[:, 4].copy()
    lo = cons[:, 0] < 1e-4
    tk = np.minimum(5e3, p_in[lo] / (cons[lo, 0] * R) * mu)
    p_want[lo] = cons[lo, 0] * tk * R / mu
    e_want[lo] = p_want[lo] / (gam - 1.0) + ekin[lo]
    assert lo.any() and (~lo).any()
    assert np.array_equal(p1, p_want)
    assert np.array_equal(c1[:, 4], e_want)
    assert np.all(g1 == gam)


def test_velocity_and_the_limiter(box):
    hp = box.params
    cons = box.cons.copy()
    vlimit = hp.vlimit
    fast = np.arange(hp.ngrid) % 7 == 0
    cons[fast, 1] = cons[fast, 0] * (1.5 * vlimit)  # |u1| above the limit
    o = fresh(box)
    o.set_state(cons, box.u, box.p, np.full(hp.ngrid, hp.gammafix))
    o.velocity()
    c1, u1, _, _ = o.get_state()
    o.close()
    u = cons[:, 1:4] / cons[:, 0:1]
    c = cons.copy()
    flag = (np.abs(u) > vlimit).any(axis=1)
    f = flag
    ekin = 0.5 * (c[f, 1] * c[f, 1] + c[f, 2] * c[f, 2] + c[f, 3] * c[f, 3]) / c[f, 0]
    speed = np.sqrt(((0.0 + u[f, 0] * u[f, 0]) + u[f, 1] * u[f, 1]) + u[f, 2] * u[f, 2])
    uf = u[f] * vlimit / speed[:, None]
    u[f] = uf
    c[f, 1:4] = uf * c[f, 0:1]
    e = c[f, 4] - ekin
    ekin2 = 0.5 * (c[f, 1] * c[f, 1] + c[f, 2] * c[f, 2] + c[f, 3] * c[f, 3]) / c[f, 0]
    c[f, 4] = np.maximum(e, hp.small_eps) + ekin2
    assert flag.sum() == fast.sum()
    assert np.array_equal(u1, u) and np.array_equal(c1, c)
    sp = np.sqrt((u1[f] ** 2).sum(axis=1))
    assert np.allclose(sp, vlimit, rtol=1e-15, atol=0)


def test_courant_over_every_cell(box):
    hp = box.params
    p = np.abs(box.p) + 0.05
    u = box.u.copy()
    b = G.boundary_flags(hp.nx, hp.ny, hp.nz)
    gi = np.flatnonzero(b > 0)[3]
    u[gi, 0] = 50.0  # the fastest cell is a ghost: it still sets dt
    o = fresh(box, u=u, p=p)
    o.courant()
    dt = o.clock()["dt"]
    o.close()
    sound = np.sqrt(hp.gammafix * p / box.cons[:, 0])
    r = ((sound + np.abs(u[:, 0])) / hp.dx + (sound + np.abs(u[:, 1])) / hp.dy +
         (sound + np.abs(u[:, 2])) / hp.dz)
    assert r.argmax() == gi
    assert dt == hp.cfl / r.max()


def test_source_with_a_force_on_the_interior(box):
    hp = box.params
    rng = np.random.default_rng(3)
    g3 = rng.standard_normal((hp.ngrid, 3))
    dt = 1e-3
    o = fresh(box)
    o.set_gforce(g3)
    o.set_clock(0.0, dt, 0.0, 0)
    o.source(0)
    c1 = o.get_state()[0]
    o.close()
    inner = G.boundary_flags(hp.nx, hp.ny, hp.nz) == 0
    c = box.cons[inner].copy()
    g = g3[inner]
    u = box.u[inner]
    c[:, 2] = c[:, 2] + (c[:, 0] * g[:, 1]) * dt
    c[:, 1] = c[:, 1] + (c[:, 0] * g[:, 0]) * dt
    c[:, 3] = c[:, 3] + (g[:, 2] * c[:, 0]) * dt
    ekin = 0.5 * (c[:, 1] * c[:, 1] + c[:, 2] * c[:, 2] + c[:, 3] * c[:, 3]) / c[:, 0]
    work = dt * c[:, 0] * ((u[:, 0] * g[:, 0] + u[:, 1] * g[:, 1]) + u[:, 2] * g[:, 2])
    c[:, 4] = np.maximum(c[:, 4] - ekin + work, hp.small_eps) + ekin
    assert np.array_equal(c1[inner], c)


def avisc_numpy(hp, u, avmag):
    """avisc.f90:13-23 from the grid coordinates: the neighbour table of
    init_grid.f90:178-261 (outer ghost layer: its donor two cells inward in
    slot 1, the other slots unset; inner ghost layer: +y, -y, +x, -x, +z, -z, the
    z pair the cell itself when nz < 6), each neighbour in a ghost layer -- or
    unset -- replaced by the cell (get_boundary, utils.f90:62-73)."""
    nx, ny, nz = hp.nx, hp.ny, hp.nz
    flag = G.boundary_flags(nx, ny, nz)
    qq = np.zeros((hp.ngrid, 3))
    for i in np.nonzero(flag > 0)[0]:
        x, y, z = i % nx, (i // nx) % ny, i // (nx * ny)
        nb = [None] * 6
        if flag[i] == 1:
            if x == 0: nb[0] = i + 2
            elif x == nx - 1: nb[0] = i - 2
            elif y == 0: nb[0] = i + 2 * nx
            elif y == ny - 1: nb[0] = i - 2 * nx
            elif z == 0: nb[0] = i if nz < 6 else i + 2 * nx * ny
            else: nb[0] = i if nz < 6 else i - 2 * nx * ny
        else:
            zs = 0 if nz < 6 else nx * ny
            nb = [i + nx, i - nx, i + 1, i - 1, i + zs, i - zs]
        b = [i if (j is None or flag[j] > 0) else j for j in nb]
        m1 = min(0.0, u[b[2], 0] - u[b[3], 0])
        m2 = min(0.0, u[b[0], 1] - u[b[1], 1])
        m3 = min(0.0, u[b[4], 2] - u[b[5], 2])
        qq[i] = (avmag[0] * (m1 * m1), avmag[1] * (m2 * m2), avmag[2] * (m3 * m3))
    return qq


@pytest.mark.parametrize("shape", [(11, 10, 9), (12, 9, 4), (8, 8, 6)])
def test_avisc_matches_the_formula_on_the_ghost_layers(shape):
    """qq on the boundary > 0 cells (the reference's condition as written),
    zero on the interior, bit for bit; zero everywhere at the default avmag = 0."""
    nx, ny, nz = shape
    st = small_random_box(nx=nx, ny=ny, nz=nz, walls=(0,) * 6, seed=nx * ny + nz, amp=0.4)
    o = fresh(st)
    avmag = (0.7, 1.3, 2.1)
    qq = o.avisc(*avmag)
    ref = avisc_numpy(st.params, st.u, avmag)
    assert np.array_equal(qq, ref)
    flag = G.boundary_flags(nx, ny, nz)
    assert not qq[flag == 0].any()
    assert qq[flag > 0].any()  # compressions in a random field
    assert not o.avisc().any()
