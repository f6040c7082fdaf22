"""Tabulated EOS (H2STAT >= 0): state() through get_gamma2 (eos.f90:653-699,
state.f90:60-79) on the device against the oracle given the same tables --
3-D grids and the nz == 1 disk branch, clamps at both ends of the energy range,
the low-density branch, then whole steps: per-phase kernels with per-cell gamma,
and the fused stage kernels with gamma reconstructed as a primitive."""
import dataclasses

import numpy as np
import pytest

from boxzyhydro_b200 import celldump as CD
from tests.helpers import compare, make_pair, small_random_box, step_both, synthetic_eos_table

pytestmark = pytest.mark.gpu


def tab_box(dims, walls, seed):
    st = small_random_box(nx=dims[0], ny=dims[1], nz=dims[2], walls=walls, seed=seed)
    st.params = dataclasses.replace(st.params, h2stat=1)
    c = st.cons
    rng = np.random.default_rng(seed + 1)
    k = rng.choice(st.params.ngrid, size=12, replace=False)
    c[k[:4], 4] *= 1e3    # above the table's energies
    c[k[4:8], 4] *= 1e-3  # below them
    c[k[8:], 0] = 1e-5    # low-density branch
    c[k[8:], 1:4] = 1e-5 * st.u[k[8:]]
    return st


@pytest.mark.parametrize("dims,walls", [((14, 12, 10), (0,) * 6), ((16, 14, 1), (1,) * 6)])
def test_tabulated_state_and_steps(tmp_path, dims, walls):
    st = tab_box(dims, walls, seed=6)
    tab = synthetic_eos_table()
    o, g = make_pair(st)
    o.set_eos_table(tab)
    g.set_eos_table(tab)
    o.state(); g.state(); compare(o, g, "state with tables")
    # per-cell mu through the celldump writer (state() again on both sides)
    path = tmp_path / "celldump.00000000"
    g.write_celldump(path)
    o.state()
    assert np.array_equal(CD.read(path)["muc"], o.muc_array())
    step_both(o, g, 3)
    # nz == 1 (the scale-height branch reads the previous gamma) stays on the
    # per-phase kernels; the 3-D grid leaves them once no cell is below the
    # low-density threshold
    if dims[2] == 1:
        assert g.status()[1] == 0
    o.close()
    g.close()


def test_steps_need_the_table():
    st = tab_box((12, 10, 8), (0,) * 6, seed=2)
    o, g = make_pair(st)
    with pytest.raises(Exception, match="bx_set_eos_table"):
        g.step()
    o.close()
    g.close()


@pytest.mark.parametrize("dims,walls", [((20, 18, 14), (0,) * 6),
                                        ((40, 30, 4), (0, 1, 1, 0, 0, 0)),
                                        ((37, 21, 13), (1, 1, 0, 0, 0, 0))])
def test_tabulated_eos_on_the_fused_path(tmp_path, dims, walls):
    """Without low-density cells the grid takes the fused stage kernels with the
    tables (32 x 6 tiles, gamma reconstructed as a primitive): steps
    bit-identical to the oracle (cells above and below the table's energies,
    so get_gamma2's clamps run in the stage kernels), and the reference arrays
    after the fused steps (p, gamma and mu from state() with the tables)."""
    st = small_random_box(nx=dims[0], ny=dims[1], nz=dims[2], walls=walls, seed=31)
    st.params = dataclasses.replace(st.params, h2stat=1)
    rng = np.random.default_rng(32)
    k = rng.choice(st.params.ngrid, size=8, replace=False)
    st.cons[k[:4], 4] *= 1e3
    st.cons[k[4:], 4] *= 1e-3
    tab = synthetic_eos_table()
    o, g = make_pair(st)
    o.set_eos_table(tab)
    g.set_eos_table(tab)
    step_both(o, g, 5)
    assert g.status()[1] == 1, "expected the fused stage kernels"
    path = tmp_path / "celldump.00000000"
    g.write_celldump(path)
    o.state()
    assert np.array_equal(CD.read(path)["muc"], o.muc_array())
    o.close()
    g.close()


def test_tabulated_eos_with_a_force_leaves_the_fused_path():
    """A force on a grid with the tabulated EOS: the steps run on the per-phase
    kernels (the fused force instances have the fixed-gamma tile shape), still
    bit-identical to the oracle, and the fused path comes back once the force
    is cleared."""
    st = small_random_box(nx=20, ny=18, nz=14, walls=(0,) * 6, seed=33)
    st.params = dataclasses.replace(st.params, h2stat=1)
    tab = synthetic_eos_table()
    o, g = make_pair(st)
    o.set_eos_table(tab)
    g.set_eos_table(tab)
    step_both(o, g, 2)
    assert g.status()[1] == 1
    hp = st.params
    from boxzyhydro_b200 import grid as G
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
