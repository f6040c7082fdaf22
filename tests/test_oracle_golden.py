"""The oracle (CPU restatement) pinned against the reference's own golden files.

The reference's only test is its Sod shock tube run (README:6-33): the final
density profile is plotted against analysis/sodtest.dat ("the curves should be
on top of each other") and the exact solution analysis/sod.ana.  These tests
run the shipped in.nml case (8x200x1, dx=0.01, gamma=1.4, reflective walls,
t=0.4) through the oracle and check it against both files, and pin this
package's exact Riemann solver against sod.ana.
"""
import os

import numpy as np
import pytest

import oracle as O
from boxzyhydro_b200 import grid as G
from boxzyhydro_b200 import ic, riemann


def test_exact_riemann_matches_sod_ana(golden_dir):
    a = np.loadtxt(os.path.join(golden_dir, "sod_exact_t0.4.txt"))
    r, u, p = riemann.sod_profile(a[:, 0], 0.4)
    # sod.ana is printed with 7 significant digits
    assert np.abs(r - a[:, 1]).max() < 2e-7
    assert np.abs(u - a[:, 2]).max() < 2e-7
    assert np.abs(p - a[:, 3]).max() < 2e-7
    ps, us = riemann.star_state(1.0, 0.0, 1.0, 0.125, 0.0, 0.1, 1.4)
    assert abs(ps - 0.30313) < 1e-5 and abs(us - 0.92745) < 1e-5


@pytest.fixture(scope="module")
def shipped_sod():
    hp = ic.shipped_sod_params()
    st = ic.sod_reference(hp, axis="y")
    o = O.Oracle(hp)
    o.set_state(st.cons, st.u, st.p, st.adindx)
    n = o.run(endtime=hp.endtime)
    c, u, p, _ = o.get_state()
    return hp, o, n, c, u, p


def test_shipped_sod_reaches_endtime(shipped_sod):
    hp, o, n, c, u, p = shipped_sod
    clk = o.clock()
    assert clk["time"] == hp.endtime
    assert n == clk["step"] > 100


def test_shipped_sod_vs_exact(shipped_sod, golden_dir):
    hp, o, n, c, u, p = shipped_sod
    x, y, z = G.cell_centres(hp.nx, hp.ny, hp.nz, hp.dx, hp.dy, hp.dz)
    b = G.boundary_flags(hp.nx, hp.ny, hp.nz)
    a = np.loadtxt(os.path.join(golden_dir, "sod_exact_t0.4.txt"))
    for xc in (-0.015, -0.005, 0.005, 0.015):
        m = (b == 0) & np.isclose(x, xc)
        re = np.interp(y[m], a[:, 0], a[:, 1])
        pe = np.interp(y[m], a[:, 0], a[:, 3])
        assert np.abs(c[m, 0] - re).mean() < 6e-3
        assert np.abs(p[m] - pe).mean() < 5e-3
        plateau = (y[m] > 0.05) & (y[m] < 0.25)
        assert abs(c[m, 0][plateau].mean() - 0.42632) < 2e-3


def test_shipped_sod_on_top_of_sodtest(shipped_sod, golden_dir):
    """README:32-33: the density curve lies on the stored reference run."""
    hp, o, n, c, u, p = shipped_sod
    x, y, z = G.cell_centres(hp.nx, hp.ny, hp.nz, hp.dx, hp.dy, hp.dz)
    b = G.boundary_flags(hp.nx, hp.ny, hp.nz)
    col = np.loadtxt(os.path.join(golden_dir, "sodtest_column.txt"))
    m = (b == 0) & np.isclose(x, -0.005)
    ref = col[2:-2]  # interior rows of the stored 200-cell column
    assert np.allclose(y[m], ref[:, 0])
    assert np.abs(c[m, 0] - ref[:, 1]).max() < 0.02
    assert np.abs(c[m, 0] - ref[:, 1]).mean() < 3e-3
    assert np.abs(p[m] - ref[:, 2]).mean() < 3e-3


def test_oracle_free_stream_is_preserved():
    """A uniform moving state with outflow walls stays uniform (HLL of equal
    states is the exact Euler flux, slopes vanish)."""
    hp = ic.HydroParams(nx=12, ny=10, nz=9, dx=0.125, dy=0.125, dz=0.125, cfl=0.4,
                        small_rho=1e-12, small_eps=1e-40, vlimit=10, gammafix=1.4, h2stat=-1,
                        no_outflow_xl=False, no_outflow_xr=False, no_outflow_yl=False,
                        no_outflow_yr=False, no_outflow_zl=False, no_outflow_zr=False)
    ng = hp.ngrid
    cons = np.zeros((ng, 5))
    cons[:, 0] = 1.0
    cons[:, 1] = 0.5
    cons[:, 2] = -0.25
    cons[:, 3] = 0.125
    u = cons[:, 1:4] / cons[:, :1]
    cons[:, 4] = 1.0 / 0.4 + 0.5 * (u ** 2).sum(1)
    o = O.Oracle(hp)
    o.set_state(cons, u, np.ones(ng), np.full(ng, 1.4))
    o.run(nsteps=5)
    c, _, _, _ = o.get_state()
    assert np.allclose(c, c[0], rtol=1e-14, atol=1e-14)


def test_oracle_sod_x_stays_one_dimensional():
    """A Sod tube split on x keeps every (y,z) column identical, bit for bit."""
    st = ic.sod_x(n_active=64, ny=8, nz=4)
    hp = st.params
    o = O.Oracle(hp)
    o.set_state(st.cons, st.u, st.p, st.adindx)
    o.run(nsteps=20)
    c, _, _, _ = o.get_state()
    zs, ys, xs = G.active_slices(hp.nx, hp.ny, hp.nz)
    c3 = c.reshape(hp.nz, hp.ny, hp.nx, 5)[zs, ys, xs]
    assert np.array_equal(c3, np.broadcast_to(c3[:1, :1], c3.shape))
    assert np.all(c3[..., 2:4] == 0.0)


def test_flux_ang_keeps_a_uniform_state_at_rest():
    """flux_ang.f90: the pressure terms of the radial and angular momentum fluxes
    cancel between the two faces of a cell for a uniform state, so a state at
    rest stays exactly at rest (self-check of the oracle's restatement)."""
    import dataclasses

    from tests.helpers import small_random_box
    st = small_random_box(nx=12, ny=10, nz=8, amp=0.0, seed=0)
    hp = dataclasses.replace(st.params, fluxangmom=True, yoffset=0.25)
    o = O.Oracle(hp)
    o.set_state(st.cons, st.u, st.p, st.adindx)
    for _ in range(3):
        o.step()
    c, u, p, _ = o.get_state()
    assert np.array_equal(c, st.cons) and np.all(u == 0.0)
    o.close()
