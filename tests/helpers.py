"""Shared helpers of the parity tests: run the oracle and the GPU path side by
side on the same seeded inputs and compare the reference's arrays."""
import numpy as np

import oracle as O
from boxzyhydro_b200 import ic
from boxzyhydro_b200.hydro import Hydro


def small_random_box(nx=14, ny=12, nz=10, walls=(0, 0, 0, 0, 0, 0), gamma=1.4, seed=0,
                     amp=0.3, dx=1.0 / 16, cfl=0.3, vlimit=10.0):
    """A seeded smooth-plus-noise 3-D state with the given walls."""
    hp = ic.HydroParams(nx=nx, ny=ny, nz=nz, dx=dx, dy=dx, dz=dx, cfl=cfl, small_rho=1e-12,
                        small_eps=1e-40, vlimit=vlimit, gammafix=gamma, h2stat=-1,
                        no_outflow_xl=bool(walls[0]), no_outflow_xr=bool(walls[1]),
                        no_outflow_yl=bool(walls[2]), no_outflow_yr=bool(walls[3]),
                        no_outflow_zl=bool(walls[4]), no_outflow_zr=bool(walls[5]))
    rng = np.random.default_rng(seed)
    ng = hp.ngrid
    rho = 1.0 + amp * rng.uniform(-1, 1, ng)
    v = amp * rng.uniform(-1, 1, (ng, 3))
    p = 1.0 + amp * rng.uniform(-1, 1, ng)
    cons = np.zeros((ng, 5))
    cons[:, 0] = rho
    cons[:, 1:4] = v * rho[:, None]
    u = cons[:, 1:4] / cons[:, 0:1]
    cons[:, 4] = p / (gamma - 1.0) + rho * 0.5 * (u ** 2).sum(1)
    return ic.State(hp, cons, u, p, np.full(ng, gamma))


def make_pair(st, phase_only=False):
    o = O.Oracle(st.params)
    o.set_state(st.cons, st.u, st.p, st.adindx)
    g = Hydro(st.params, phase_only=phase_only)
    g.upload(st.cons, st.u, st.p)
    return o, g


def compare(o, g, what="", u_and_p=True):
    c0, u0, p0, _ = o.get_state()
    c1, u1, p1 = g.download()
    bad = []
    if not np.array_equal(c0, c1):
        d = np.abs(c0 - c1)
        i = np.unravel_index(np.nanargmax(d), d.shape)
        bad.append(f"cons differs: max|d|={np.nanmax(d):.3e} at {i} ({c0[i]!r} vs {c1[i]!r}), "
                   f"{int((c0 != c1).sum())} values")
    if u_and_p and not np.array_equal(u0, u1):
        bad.append(f"u differs: max|d|={np.nanmax(np.abs(u0 - u1)):.3e}")
    if u_and_p and not np.array_equal(p0, p1):
        bad.append(f"p differs: max|d|={np.nanmax(np.abs(p0 - p1)):.3e}")
    assert not bad, what + ": " + "; ".join(bad)


def step_both(o, g, nsteps, endtime=1e300, check_every=1):
    for k in range(nsteps):
        ro = o.step(endtime)
        rg = g.step(endtime)
        assert ro == rg
        if not ro:
            break
        if (k + 1) % check_every == 0 or k == nsteps - 1:
            co, cg = o.clock(), g.clock()
            for key in ("time", "dt", "dtold", "step"):
                assert co[key] == cg[key], f"step {k + 1}: clock {key} {co[key]!r} vs {cg[key]!r}"
            compare(o, g, f"after step {k + 1}")


def synthetic_eos_table(neos=40, neos_rho=9, seed=0):
    """Tables in the layout of the eos module for the tabulated state() path
    (tests/eos_tables.py)."""
    from tests.eos_tables import synthetic_table
    return synthetic_table(neos, neos_rho, seed)
