"""Batched ensembles: every box of a batch run evolves exactly as the same box
run alone through bx_step (cons, u, p and clock identical after the run),
with and without the CUDA graph, including a box that leaves the fused path
(velocity limiter) and finishes on its own handle."""
import numpy as np
import pytest

from boxzyhydro_b200 import ic
from boxzyhydro_b200.batch import Batch
from boxzyhydro_b200.hydro import BoxzyError, Hydro

pytestmark = pytest.mark.gpu


def ensemble(n, seed, sides=(8, 12, 20, 13)):
    spec = ic.riemann_ensemble_spec(nbox=n, seed=seed, sides=sides)
    return [ic.riemann_box(s["side"], s["axis"], s["left"], s["right"], s["gamma"]) for s in spec]


def alone(st, nsteps):
    h = Hydro(st.params)
    h.upload(st.cons, st.u, st.p)
    h.run(nsteps=nsteps)
    out = h.download(), h.clock()
    h.close()
    return out


@pytest.mark.parametrize("graph", [True, False])
def test_batch_matches_single_grid_runs(graph):
    boxes = ensemble(14, seed=5)
    b = Batch([st.params for st in boxes])
    for i, st in enumerate(boxes):
        b.upload(i, st.cons)
    b.run(6, graph=graph)
    b.run(5, graph=graph)
    assert b.info()["solo_boxes"] == 0
    for i, st in enumerate(boxes):
        (c0, u0, p0), clk0 = alone(st, 11)
        c1, u1, p1 = b.download(i)
        assert np.array_equal(c0, c1), f"box {i}"
        assert np.array_equal(u0, u1) and np.array_equal(p0, p1), f"box {i}"
        clk1 = b.clock(i)
        for k in ("time", "dt", "dtold", "step"):
            assert clk0[k] == clk1[k], (i, k)
    b.close()


@pytest.mark.parametrize("graph", [True, False])
def test_persistent_launch_matches_single_grid_runs(graph):
    """One persistent launch per run (items taken from a queue, per-box waits):
    every box as it would run alone, bit for bit, over two runs; three launches
    per run."""
    boxes = ensemble(14, seed=21, sides=(8, 12, 20, 13, 40))
    b = Batch([st.params for st in boxes])
    b.set_persistent(True)
    assert b.persistent
    for i, st in enumerate(boxes):
        b.upload(i, st.cons)
    b.run(6, graph=graph)
    assert b.info()["launches"] == 3
    b.run(5, graph=graph)
    for i, st in enumerate(boxes):
        (c0, u0, p0), clk0 = alone(st, 11)
        c1, u1, p1 = b.download(i)
        assert np.array_equal(c0, c1) and np.array_equal(u0, u1) and np.array_equal(p0, p1), i
        clk1 = b.clock(i)
        for k in ("time", "dt", "dtold", "step"):
            assert clk0[k] == clk1[k], (i, k)
    b.close()


@pytest.mark.parametrize("persistent", [False, True])
def test_16x16_tiles_match_single_grid_runs(persistent):
    """The second tile shape (16 x 16 columns) in both launch forms: every box as
    it would run alone, bit for bit."""
    boxes = ensemble(10, seed=33, sides=(8, 12, 20, 13, 40, 18))
    b = Batch([st.params for st in boxes])
    b.set_tile_shape(1)
    assert b.tile_shape[:3] == (1, 16, 16)
    b.set_persistent(persistent)
    for i, st in enumerate(boxes):
        b.upload(i, st.cons)
    b.run(4)
    b.run(3)
    for i, st in enumerate(boxes):
        (c0, u0, p0), clk0 = alone(st, 7)
        c1, u1, p1 = b.download(i)
        assert np.array_equal(c0, c1) and np.array_equal(u0, u1) and np.array_equal(p0, p1), i
        clk1 = b.clock(i)
        for k in ("time", "dt", "dtold", "step"):
            assert clk0[k] == clk1[k], (i, k)
    b.close()


def test_persistent_launch_with_a_box_leaving_the_fused_path():
    boxes = ensemble(6, seed=9)
    boxes[2].params.vlimit = 0.6
    boxes[2].params.validate()
    b = Batch([s.params for s in boxes])
    b.set_persistent(True)
    for i, s in enumerate(boxes):
        b.upload(i, s.cons)
    b.run(7)
    assert b.info()["solo_boxes"] >= 1
    for i, s in enumerate(boxes):
        (c0, u0, p0), clk0 = alone(s, 7)
        c1, u1, p1 = b.download(i)
        assert np.array_equal(c0, c1) and np.array_equal(u0, u1) and np.array_equal(p0, p1), i
        assert b.clock(i)["step"] == clk0["step"] == 7
    b.close()


def test_persistent_wait_gives_up_at_its_poll_limit():
    """The wait of the persistent launch on a counter nothing advances ends by
    itself after its poll limit and reports it, with the device usable after."""
    from boxzyhydro_b200.batch import wait_selftest
    gave_up, ms = wait_selftest(2000)
    assert gave_up and 0.0 < ms < 1000.0
    boxes = ensemble(3, seed=2)
    b = Batch([s.params for s in boxes])
    for i, s in enumerate(boxes):
        b.upload(i, s.cons)
    b.run(2)
    b.close()


def test_batch_box_leaving_the_fused_path():
    boxes = ensemble(6, seed=9)
    # a box whose velocity limiter fires: |v| up to 1 against vlimit 0.6
    st = boxes[2]
    st.params.vlimit = 0.6
    st.params.validate()
    b = Batch([s.params for s in boxes])
    for i, s in enumerate(boxes):
        b.upload(i, s.cons)
    b.run(7)
    assert b.info()["solo_boxes"] >= 1
    for i, s in enumerate(boxes):
        (c0, u0, p0), clk0 = alone(s, 7)
        c1, u1, p1 = b.download(i)
        assert np.array_equal(c0, c1) and np.array_equal(u0, u1) and np.array_equal(p0, p1), i
        assert b.clock(i)["step"] == clk0["step"] == 7
    b.close()


def test_autotune_leaves_the_ensemble_as_it_was():
    """The tile-depth autotuner times trial steps from the current states; the
    boxes then continue exactly as if it had not run, with the tiling it chose,
    and so does a box already on its own handle."""
    boxes = ensemble(10, seed=12, sides=(8, 12, 20, 26))
    boxes[3].params.vlimit = 0.6
    boxes[3].params.validate()
    b = Batch([st.params for st in boxes])
    for i, st in enumerate(boxes):
        b.upload(i, st.cons)
    b.run(3)
    solo = b.info()["solo_boxes"]
    zc, ms = b.autotune(reps=2)
    assert ms > 0 and (zc in (0, 8, 16, 32, 64) or zc >= 1 << 30)
    assert b.tile_shape[0] in (0, 1) and b.tile_shape[3] == zc
    assert b.info()["solo_boxes"] == solo
    for i in range(len(boxes)):
        assert b.clock(i)["step"] == 3
    b.run(5)
    for i, st in enumerate(boxes):
        (c0, u0, p0), clk0 = alone(st, 8)
        c1, u1, p1 = b.download(i)
        assert np.array_equal(c0, c1) and np.array_equal(u0, u1) and np.array_equal(p0, p1), i
        clk1 = b.clock(i)
        for k in ("time", "dt", "dtold", "step"):
            assert clk0[k] == clk1[k], (i, k)
    b.close()


def test_batch_rejects_state_it_cannot_start_from():
    st = ic.sod_x(n_active=16, ny=8, nz=8)
    st.params.no_outflow_xl = st.params.no_outflow_xr = False
    st.params.no_outflow_yl = st.params.no_outflow_yr = False
    st.params.no_outflow_zl = st.params.no_outflow_zr = False
    b = Batch([st.params])
    with pytest.raises(BoxzyError):
        b.upload(0, st.cons)   # outer ghost layer holds small_rho, not the fill
    b.close()
