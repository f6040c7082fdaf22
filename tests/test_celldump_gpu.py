"""celldump writer and restart reader of the library (bx_write_celldump,
bx_read_celldump) against the oracle: the file holds the reference's arrays
after state() (write_files.f90:32-63), and a restart reproduces read_hydro.f90
and continues bit for bit."""
import numpy as np
import pytest

import oracle as O
from boxzyhydro_b200 import celldump as CD
from boxzyhydro_b200 import grid as G
from boxzyhydro_b200.hydro import Hydro
from tests.helpers import compare, make_pair, small_random_box, step_both

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("walls,dims", [((0,) * 6, (14, 12, 10)), ((1,) * 6, (16, 9, 4))])
def test_write_then_restart(tmp_path, walls, dims):
    st = small_random_box(nx=dims[0], ny=dims[1], nz=dims[2], walls=walls, seed=2)
    hp = st.params
    o, g = make_pair(st)
    step_both(o, g, 3)
    path = tmp_path / "celldump.00000003"
    rng = np.random.default_rng(4)
    phi = rng.standard_normal(hp.ngrid)
    g.write_celldump(path, phi=phi)
    o.state()  # write_files calls state() first, with its effect on the arrays
    compare(o, g, "arrays after the dump's state()")
    c0, u0, p0, _ = o.get_state()
    d = CD.read(path)
    clk = o.clock()
    assert d["readtest"] == 1234 and d["time"] == clk["time"] and d["step"] == clk["step"] == 3
    assert np.array_equal(d["units"], CD.units())
    x, y, z = G.cell_centres(hp.nx, hp.ny, hp.nz, hp.dx, hp.dy, hp.dz)
    assert np.array_equal(d["x"], x) and np.array_equal(d["y"], y) and np.array_equal(d["z"], z)
    assert np.array_equal(d["rho"], c0[:, 0]) and np.array_equal(d["E"], c0[:, 4])
    assert np.array_equal(d["p"], p0) and np.array_equal(d["u"], u0)
    assert np.array_equal(d["phi"], phi) and np.all(d["muc"] == hp.muc)
    assert np.array_equal(d["boundary"], G.boundary_flags(hp.nx, hp.ny, hp.nz))

    # restart: read_hydro on the oracle side (m = u rho, outer layer reset, state())
    g2 = Hydro(hp)
    t, s, ph = g2.read_celldump(path, want_phi=True)
    assert t == d["time"] and s == 3 and np.array_equal(ph, phi)
    cons, u, p = CD.restart_arrays(hp, d)
    o2 = O.Oracle(hp)
    o2.set_state(cons, u, p, np.full(hp.ngrid, hp.gammafix))
    o2.state()
    o2.set_clock(time=t, dt=0.0, dtold=0.0, step=s)
    compare(o2, g2, "arrays after the restart")
    ck = g2.clock()
    assert ck["time"] == t and ck["dtold"] == 0.0 and ck["step"] == 3
    step_both(o2, g2, 3)
    o.close()
    o2.close()
    g.close()
    g2.close()


def test_read_rejects_a_short_file(tmp_path):
    st = small_random_box(nx=10, ny=9, nz=7, seed=1)
    hp = st.params
    path = tmp_path / "celldump.00000001"
    CD.from_arrays(hp, st.cons, st.u, st.p, time=0.0, step=1, path=path)
    raw = path.read_bytes()
    path.write_bytes(raw[:-100])
    g = Hydro(hp)
    with pytest.raises(Exception, match="fewer cell records"):
        g.read_celldump(path)
    g.close()
