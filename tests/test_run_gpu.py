"""bx_run on the fused form: the steps go out in runs of up to 32 without a host
round trip per step; a step whose guard fires is rolled back on the device and
taken again by bx_step.  Compared with the oracle's loop, bit for bit (cons, u,
p and the clock): runs longer than one chunk, a step count and an end time
that stop inside a chunk, the velocity limiter firing inside a run, a gravity
force, and against a step-by-step loop on the same handle type."""
import numpy as np
import pytest

from boxzyhydro_b200 import grid as G
from boxzyhydro_b200 import ic
from tests.helpers import compare, make_pair, small_random_box

pytestmark = pytest.mark.gpu


def clocks_equal(o, g):
    co, cg = o.clock(), g.clock()
    for key in ("time", "dt", "dtold", "step"):
        assert co[key] == cg[key], f"clock {key} {co[key]!r} vs {cg[key]!r}"


def test_long_run_and_step_count():
    st = ic.turbulent_box(n=40, seed=21)
    o, g = make_pair(st)
    assert o.run(nsteps=70) == g.run(nsteps=70) == 70
    clocks_equal(o, g)
    compare(o, g, "after 70 steps")
    assert g.status()[1] == 1
    assert o.run(nsteps=45) == g.run(nsteps=45) == 45
    clocks_equal(o, g)
    compare(o, g, "after 115 steps")


def test_end_time_inside_a_chunk():
    st = ic.turbulent_box(n=32, seed=22)
    o, g = make_pair(st)
    o.run(nsteps=3)
    g.run(nsteps=3)
    end = o.clock()["time"] + 12.5 * o.clock()["dt"]
    n_o = o.run(endtime=end)
    n_g = g.run(endtime=end)
    assert n_o == n_g and g.clock()["time"] == end
    clocks_equal(o, g)
    compare(o, g, "at the end time")
    assert g.run(endtime=end) == 0


def test_limiter_fires_inside_a_run():
    """|u| > vlimit in some steps: those are rolled back and redone on the
    per-phase kernels, the run goes on."""
    st = small_random_box(nx=16, ny=13, nz=9, walls=(0,) * 6, seed=8, amp=0.6, vlimit=0.55)
    o, g = make_pair(st)
    assert o.run(nsteps=40) == g.run(nsteps=40) == 40
    clocks_equal(o, g)
    compare(o, g, "after 40 steps")
    assert g.status()[0] & 1


def test_run_with_gravity():
    st = ic.turbulent_box(n=32, seed=23)
    hp = st.params
    x, y, z = G.cell_centres(hp.nx, hp.ny, hp.nz, hp.dx, hp.dy, hp.dz)
    phi = -0.05 / np.sqrt(x * x + y * y + z * z + 0.02)
    o, g = make_pair(st)
    o.set_gforce(o.calc_gforce(phi))
    g.set_phi(phi)
    assert o.run(nsteps=40) == g.run(nsteps=40) == 40
    clocks_equal(o, g)
    compare(o, g, "after 40 steps with a force")
    assert g.status()[1] == 1
