"""bx_step_host -- one main-loop iteration on a state held on the host, with the
copies overlapped with the step -- against the three calls it stands for
(bx_upload_conserved, bx_step, bx_download of cons) and against the oracle, bit
for bit: several z slabs, reflective and outflow walls, a 2-D grid, a state the
fused path rejects (dirty ghosts), steps the velocity limiter redoes, the end
time, in place and into a second array, pageable and page-locked memory."""
import numpy as np
import pytest
import torch

import oracle as O
from boxzyhydro_b200 import grid as G
from boxzyhydro_b200 import ic
from boxzyhydro_b200.hydro import Hydro

from .helpers import small_random_box

pytestmark = pytest.mark.gpu


_PINNED = []  # the tensors that own the page-locked buffers


def pinned_copy(a):
    t = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
    _PINNED.append(t)
    out = t.numpy()
    out[:] = a
    return out


def three_calls(g, cons, endtime=1e300):
    g.upload_conserved(cons)
    ran = g.step(endtime)
    return g.download()[0], ran


def oracle_set(o, params, cons):
    """The oracle's arrays at the state bx_upload_conserved makes of cons:
    u = m/rho, p from state() with that u (the clock is kept)."""
    gam = params.gammafix
    u = cons[:, 1:4] / cons[:, 0:1]
    ek = cons[:, 0] * 0.5 * (u[:, 0] * u[:, 0] + u[:, 1] * u[:, 1] + u[:, 2] * u[:, 2])
    p = np.maximum(cons[:, 4] - ek, params.small_eps) * (gam - 1.0)
    o.set_state(cons, u, p, np.full(len(cons), gam))


def run_pair(st, nsteps, pinned, in_place, endtime=1e300, modify=None, phi=None):
    """Steps through bx_step_host (handle a), the three calls (handle b) and the
    oracle from the same cons; `modify(k, cons)` changes the host state in place
    before step k (the same change on all three); `phi(k)` gives the potential
    of step k (or None: no force)."""
    ga, gb = Hydro(st.params), Hydro(st.params)
    c0 = np.ascontiguousarray(st.cons)
    ca = pinned_copy(c0) if pinned else c0.copy()
    cb = c0.copy()
    out = ca if in_place else (pinned_copy(c0) if pinned else np.empty_like(c0))
    o = O.Oracle(st.params)
    oracle_set(o, st.params, c0)
    src = ca
    for k in range(nsteps):
        if modify is not None and modify(k, src):
            cb[:] = src
            oracle_set(o, st.params, src)
        if phi is not None:
            ph = phi(k)
            ga.set_phi(ph)
            gb.set_phi(ph)
            o.set_gforce(None if ph is None else o.calc_gforce(ph))
        ra = ga.step_host(src, out, endtime)
        cb, rb = three_calls(gb, cb, endtime)
        assert ra == rb, f"step {k + 1}: ran {ra} vs {rb}"
        assert np.array_equal(out, cb), f"step {k + 1}: cons differs from the three calls " \
            f"(max |d| {np.nanmax(np.abs(out - cb)):.3e}, {int((out != cb).sum())} values)"
        ka, kb = ga.clock(), gb.clock()
        for key in ("time", "dt", "dtold", "step"):
            assert ka[key] == kb[key], f"step {k + 1}: clock {key} {ka[key]!r} vs {kb[key]!r}"
        assert o.step(endtime) == ra
        assert np.array_equal(out, o.get_state()[0]), f"step {k + 1}: cons differs from the oracle"
        assert o.clock()["time"] == ka["time"]
        if not in_place:
            src[:] = out
    return ga, gb


def test_turbulent_box_many_slabs_pinned_in_place():
    st = ic.turbulent_box(n=64, seed=5)
    ga, _ = run_pair(st, 4, pinned=True, in_place=True)
    assert ga.status()[1] == 1


def test_walls_ragged_pageable_two_arrays():
    st = small_random_box(nx=37, ny=21, nz=19, walls=(0, 1, 1, 0, 0, 1), seed=21)
    ga, _ = run_pair(st, 4, pinned=False, in_place=False)
    assert ga.status()[1] == 1


def test_grid_off_the_fused_path():
    """Reflective walls on all six sides of a 3-D grid: the fused path does not
    take it, and the call runs the three calls in sequence."""
    st = small_random_box(nx=13, ny=12, nz=10, walls=(1,) * 6, seed=2)
    ga, _ = run_pair(st, 3, pinned=True, in_place=True)
    assert ga.status()[1] == 0


def test_two_dimensional_grid():
    st = small_random_box(nx=40, ny=30, nz=4, walls=(0, 1, 1, 0, 0, 0), seed=22)
    run_pair(st, 4, pinned=True, in_place=False)


def test_dirty_ghosts_take_the_reference_flow():
    """Ghost values that are not copies of their donors: the fused path does not
    take the state, the step runs the per-phase kernels like the three calls."""
    st = small_random_box(nx=20, ny=18, nz=16, walls=(0,) * 6, seed=23)
    st.cons[0, 4] *= 1.5  # a corner ghost
    ga, gb = run_pair(st, 3, pinned=True, in_place=True)
    sa, sb = ga.status(), gb.status()
    assert sa == sb


def test_velocity_limiter_redo():
    """|u| > vlimit: the fused step is redone on the per-phase kernels and the
    copies already made are replaced."""
    st = small_random_box(nx=16, ny=13, nz=9, walls=(0,) * 6, seed=8, amp=0.6, vlimit=0.55)
    ga, gb = run_pair(st, 5, pinned=True, in_place=True)
    sa, sb = ga.status(), gb.status()
    assert sa[0] & 1 and sa == sb


def test_host_changes_the_state_between_steps():
    """The step is started with dt from the rate the device holds for the state
    it left; a host that changes the state between the calls gets the step of
    the state it passed (a change of the maximum rate restarts the step, others
    keep it)."""
    st = ic.turbulent_box(n=48, seed=7)

    def modify(k, c):
        if k == 2:  # every momentum: the maximum rate changes
            c[:, 1:4] *= 1.001
            return True
        if k == 4:  # one interior cell's energy, far from the maximum rate
            i = (st.params.nx * st.params.ny) * 20 + st.params.nx * 20 + 20
            c[i, 4] *= 1.0 + 1e-9
            return True
        return False

    ga, _ = run_pair(st, 6, pinned=True, in_place=True, modify=modify)
    assert ga.status()[1] == 1


def test_potential_from_the_host():
    """A potential from the host's solver before every step (a point mass that
    moves, off for one step): the force terms of the stage kernels."""
    st = ic.turbulent_box(n=48, seed=9)
    hp = st.params
    x, y, z = G.cell_centres(hp.nx, hp.ny, hp.nz, hp.dx, hp.dy, hp.dz)

    def phi(k):
        if k == 3:
            return None
        return -0.05 / np.sqrt((x - 0.02 * k) ** 2 + y * y + z * z + 0.02)

    ga, _ = run_pair(st, 6, pinned=True, in_place=True, phi=phi)
    assert ga.status()[1] == 1


def test_end_time_reached():
    st = ic.turbulent_box(n=32, seed=6)
    ga, gb = run_pair(st, 2, pinned=True, in_place=False, endtime=0.0)
    assert ga.clock()["step"] == 0


def test_profiled_call_gives_a_timeline_and_the_same_state():
    """With the timeline on, a call records its per-slab events (ordered as the
    pipeline orders them) and gives the same state as without it."""
    st = ic.turbulent_box(n=64, seed=6)
    ga, gb = Hydro(st.params), Hydro(st.params)
    c = pinned_copy(np.ascontiguousarray(st.cons))
    ref = c.copy()
    ga.step_host(c, c)
    gb.step_host(ref, ref)
    ga.step_host_profile(True)
    ga.step_host(c, c)
    gb.step_host(ref, ref)
    assert np.array_equal(c, ref)
    tl = ga.step_host_timeline()
    assert tl.shape[0] > 4 and tl.shape[1] == 7
    assert np.all(tl >= 0.0)
    up0, up1, s0, s1, cv, dn0, dn1 = tl.T
    # events on one stream are ordered; across streams (a wait on another
    # stream's event, then an event here) the two timestamps may differ by the
    # few microseconds between the waited-on event and the one recorded beside it
    tol = 0.05
    assert np.all(up1 >= up0) and np.all(dn1 >= dn0)
    assert np.all(cv >= s1 - tol) and np.all(dn0 >= cv - tol)
    assert np.all(np.diff(up1) >= 0.0)  # the uploads run in order on one stream
    ga.step_host_profile(False)
    ga.close()
    gb.close()
