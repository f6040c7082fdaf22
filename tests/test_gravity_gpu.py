"""Gravity coupling: a potential from the host (bx_set_phi) becomes gforce by
calc_gforce (utils.f90:549-571) on the device, and source() applies it
(source.f90:148-191); compared with the oracle given the same potential, bit
for bit (cons, u and p).  Grids the fused path takes run the stage kernels with
the force terms after their first step; the others the per-phase kernels."""
import numpy as np
import pytest

from boxzyhydro_b200 import grid as G
from boxzyhydro_b200 import ic
from tests.helpers import compare, make_pair, small_random_box, step_both

pytestmark = pytest.mark.gpu


def potential(hp, seed, t=0.0):
    x, y, z = G.cell_centres(hp.nx, hp.ny, hp.nz, hp.dx, hp.dy, hp.dz)
    rng = np.random.default_rng(seed)
    a = rng.uniform(0.5, 1.5, 3)
    return -1.0 / np.sqrt((x - 0.1 * t) ** 2 + y ** 2 + z ** 2 + a[0] * 0.1) + a[1] * 0.05 * x * y


@pytest.mark.parametrize("walls,dims,fused", [((0,) * 6, (14, 12, 10), True),
                                               ((1,) * 6, (16, 10, 4), True),
                                               ((0, 1, 1, 0, 0, 1), (23, 14, 12), True),
                                               ((1,) * 6, (13, 12, 10), False)])
def test_potential_each_step(walls, dims, fused):
    st = small_random_box(nx=dims[0], ny=dims[1], nz=dims[2], walls=walls, seed=9)
    hp = st.params
    o, g = make_pair(st)
    for k in range(4):
        phi = potential(hp, 3, t=float(k))
        o.set_gforce(o.calc_gforce(phi))
        g.set_phi(phi)
        step_both(o, g, 1)
    assert g.status()[1] == (1 if fused else 0)
    # removing the potential returns to the force-free step
    o.set_gforce(None)
    g.set_phi(None)
    step_both(o, g, 2)
    compare(o, g, "after the force-free steps")
    o.close()
    g.close()


def test_turbulent_box_with_a_point_mass():
    """The stage kernels with the force terms on a turbulent box: a fixed
    softened point-mass potential for several steps (arrays compared after each),
    switched off and on again between fused steps."""
    st = ic.turbulent_box(n=40, seed=11)
    hp = st.params
    x, y, z = G.cell_centres(hp.nx, hp.ny, hp.nz, hp.dx, hp.dy, hp.dz)
    phi = -0.05 / np.sqrt(x * x + y * y + z * z + 0.02)
    o, g = make_pair(st)
    gf = o.calc_gforce(phi)
    o.set_gforce(gf)
    g.set_phi(phi)
    step_both(o, g, 4)
    assert g.status()[1] == 1
    o.set_gforce(None)
    g.set_phi(None)
    step_both(o, g, 2)
    o.set_gforce(gf)
    g.set_phi(phi)
    step_both(o, g, 3)
    assert g.status()[1] == 1
    o.close()
    g.close()
