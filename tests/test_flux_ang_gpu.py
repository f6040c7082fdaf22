"""Angular-momentum fluxing (fluxangmom=.true., flux_ang.f90) on the per-phase
kernels against the oracle's restatement: whole steps and single flux calls,
with and without yoffset, outflow and reflective walls."""
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
    st = ang_box(dims, walls, yoffset, seed=5)
    o, g = make_pair(st)
    step_both(o, g, 4)
    assert g.status()[1] == 0  # flux_ang runs on the per-phase kernels
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
