"""Angular-momentum fluxing (fluxangmom=.true., flux_ang.f90) on the per-phase
kernels and on the fused stage kernels against the oracle's restatement: whole
steps and single flux calls, with and without yoffset, outflow and reflective
walls, a force switched on and off."""
import dataclasses

import numpy as np
import pytest

from tests.helpers import compare, make_pair, small_random_box, step_both

pytestmark = pytest.mark.gpu


def ang_box(dims, walls, yoffset, seed):
    st = small_random_box(nx=dims[0], ny=dims[1], nz=dims[2], walls=walls, seed=seed)
    st.params = dataclasses.replace(st.params, fluxangmom=True, yoffset=yoffset)
    return st


@pytest.mark.parametrize("dims,walls,yoffset", [((14, 12, 10), (0,) * 6, 0.0),
                                                ((16, 10, 8), (1,) * 6, 0.3),
                                                ((18, 12, 4), (1, 0, 0, 1, 0, 0), -0.45)])
def test_flux_ang_steps(dims, walls, yoffset):
    """Steps bit-identical to the oracle; after the first step (per-phase, from
    the upload) the grids the fused kernels take run them with the transformed
    momenta (tile shape 3), the reflective 3-D box stays on the per-phase
    kernels."""
    st = ang_box(dims, walls, yoffset, seed=5)
    o, g = make_pair(st)
    step_both(o, g, 4)
    reflective_3d = dims[2] >= 6 and any(walls[4:])
    assert g.status()[1] == (0 if reflective_3d else 1)
    o.close()
    g.close()


def test_flux_ang_turbulent_box_runs_fused():
    """The turbulent box with the rotation axis below the box (yoffset 0.75):
    every step on the fused kernels with no guard fired, bit-identical to the
    oracle."""
    from boxzyhydro_b200 import ic
    st = ic.turbulent_box(n=40, seed=3)
    st.params = dataclasses.replace(st.params, fluxangmom=True, yoffset=0.75)
    o, g = make_pair(st)
    step_both(o, g, 1)
    g.status()
    step_both(o, g, 4)
    assert g.status() == (0, 1)
    o.close()
    g.close()


def test_flux_ang_fused_with_a_force_leaves_and_returns():
    """A force moves a flux_ang grid to the per-phase kernels (the force
    instances have the fixed-gamma, fixed-frame tile shape); clearing it lets
    the next clean step return to the fused kernels, bit-identical throughout."""
    from boxzyhydro_b200 import grid as G
    st = ang_box((20, 18, 14), (0,) * 6, 0.25, seed=9)
    o, g = make_pair(st)
    step_both(o, g, 2)
    assert g.status()[1] == 1
    hp = st.params
    x, y, z = G.cell_centres(hp.nx, hp.ny, hp.nz, hp.dx, hp.dy, hp.dz)
    phi = -0.05 / np.sqrt(x * x + y * y + z * z + 0.01)
    g.set_phi(phi)
    o.set_gforce(o.calc_gforce(phi))
    step_both(o, g, 2)
    assert g.status()[1] == 0
    g.set_phi(None)
    o.set_gforce(None)
    step_both(o, g, 3)
    assert g.status()[1] == 1
    o.close()
    g.close()


def test_flux_ang_single_calls():
    st = ang_box((14, 12, 10), (0,) * 6, 0.2, seed=8)
    o, g = make_pair(st)
    o.set_clock(dt=0.002)
    g.set_dt(0.002)
    for obj in (o, g):
        obj.state()
        obj.velocity()
        obj.save_cons_old()
    o.flux(0); g.flux(0); compare(o, g, "flux_ang(0)")
    for obj in (o, g):
        obj.state()
        obj.velocity()
    o.flux(1); g.flux(1); compare(o, g, "flux_ang(1)")
    # the second call reads cons_old as the first left it (transformed and back)
    o.flux(1); g.flux(1); compare(o, g, "flux_ang(1) again")
    o.close()
    g.close()
