"""Gravity coupling: a potential from the host (bx_set_phi) becomes gforce by
calc_gforce (utils.f90:549-571) on the device, and source() applies it
(source.f90:148-191); compared with the oracle given the same potential."""
import numpy as np
import pytest

from boxzyhydro_b200 import grid as G
from tests.helpers import compare, make_pair, small_random_box, step_both

pytestmark = pytest.mark.gpu


def potential(hp, seed, t=0.0):
    x, y, z = G.cell_centres(hp.nx, hp.ny, hp.nz, hp.dx, hp.dy, hp.dz)
    rng = np.random.default_rng(seed)
    a = rng.uniform(0.5, 1.5, 3)
    return -1.0 / np.sqrt((x - 0.1 * t) ** 2 + y ** 2 + z ** 2 + a[0] * 0.1) + a[1] * 0.05 * x * y


@pytest.mark.parametrize("walls,dims", [((0,) * 6, (14, 12, 10)), ((1,) * 6, (16, 10, 4))])
def test_potential_each_step(walls, dims):
    st = small_random_box(nx=dims[0], ny=dims[1], nz=dims[2], walls=walls, seed=9)
    hp = st.params
    o, g = make_pair(st)
    for k in range(4):
        phi = potential(hp, 3, t=float(k))
        o.set_gforce(o.calc_gforce(phi))
        g.set_phi(phi)
        step_both(o, g, 1)
    # removing the potential returns to the force-free step
    o.set_gforce(None)
    g.set_phi(None)
    step_both(o, g, 2)
    compare(o, g, "after the force-free steps")
    o.close()
    g.close()
