"""Tabulated EOS (H2STAT >= 0): state() through get_gamma2 (eos.f90:653-699,
state.f90:60-79) on the device against the oracle given the same tables --
3-D grids and the nz == 1 disk branch, clamps at both ends of the energy range,
the low-density branch, then whole steps (per-phase kernels with per-cell gamma)."""
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
