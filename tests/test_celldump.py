"""celldump codec (write_files.f90:55-63, read_hydro.f90:122-134) on the host:
record framing, header values, round trip, restart arrays."""
import numpy as np

import oracle as O
from boxzyhydro_b200 import celldump as CD
from boxzyhydro_b200 import grid as G
from tests.helpers import small_random_box


def test_units_match_the_oracle():
    u = CD.units()
    assert dict(zip(CD.UNIT_NAMES, u))["rgas"] == O.rgas_code_units()
    assert u[CD.UNIT_NAMES.index("kelvin")] == 1.0


def test_record_framing_and_round_trip(tmp_path):
    st = small_random_box(nx=9, ny=7, nz=6, seed=3)
    hp = st.params
    path = tmp_path / "celldump.00000012"
    rng = np.random.default_rng(1)
    phi = rng.standard_normal(hp.ngrid)
    d0 = CD.from_arrays(hp, st.cons, st.u, st.p, time=0.375, step=12, phi=phi, path=path)
    raw = path.read_bytes()
    assert len(raw) == CD.HEADER_BYTES + 100 * hp.ngrid
    head = np.frombuffer(raw[:12], "<i4")
    assert list(head) == [4, 1234, 4]
    assert np.frombuffer(raw[12:16], "<i4")[0] == 12
    assert np.frombuffer(raw[16:24], "<f8")[0] == 0.375
    assert list(np.frombuffer(raw[24:32], "<i4")) == [12, 12]
    assert list(np.frombuffer(raw[32:36], "<i4")) == [64]
    first = raw[CD.HEADER_BYTES:CD.HEADER_BYTES + 100]
    assert np.frombuffer(first[:4], "<i4")[0] == 92 and np.frombuffer(first[96:], "<i4")[0] == 92
    v = np.frombuffer(first[4:92], "<f8")
    x, y, z = G.cell_centres(hp.nx, hp.ny, hp.nz, hp.dx, hp.dy, hp.dz)
    assert (v[0], v[1], v[2]) == (x[0], y[0], z[0])
    assert v[3] == st.cons[0, 0] and v[9] == st.cons[0, 4] and v[8] == phi[0]
    d = CD.read(path)
    assert d["readtest"] == 1234 and d["time"] == 0.375 and d["step"] == 12
    assert np.array_equal(d["units"], CD.units())
    for k in ("x", "y", "z", "rho", "p", "E", "muc", "boundary"):
        assert np.array_equal(d[k], d0[k]), k
    assert np.array_equal(d["u"], st.u) and np.array_equal(d["phi"], phi)


def test_restart_arrays_follow_read_hydro(tmp_path):
    st = small_random_box(nx=8, ny=8, nz=7, seed=5)
    hp = st.params
    path = tmp_path / "celldump.00000003"
    CD.from_arrays(hp, st.cons, st.u, st.p, time=1.5, step=3, path=path)
    cons, u, p = CD.restart_arrays(hp, CD.read(path))
    b = G.boundary_flags(hp.nx, hp.ny, hp.nz)
    inner = b != 1
    assert np.array_equal(cons[inner, 0], st.cons[inner, 0])
    assert np.array_equal(cons[inner, 1:4], st.u[inner] * st.cons[inner, 0:1])
    assert np.all(cons[b == 1] == [hp.small_rho, 0, 0, 0, hp.small_eps])
    assert np.array_equal(u, st.u) and np.array_equal(p, st.p)
