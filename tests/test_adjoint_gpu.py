"""Discrete adjoint of a run (bx_adj_*): dot-product test against the tangent-linear
model (oracle/tangent.py), finite differences of the GPU forward and of the CPU
oracle, checkpoint schedules, and the torch.autograd.Function."""
import numpy as np
import pytest

import oracle as O
import tangent as TLM
from boxzyhydro_b200 import grid as G
from boxzyhydro_b200.adjoint import AdjointEngine, AdjointRun, device_bytes, plan
from tests.helpers import small_random_box

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    return torch


def interior_mask(hp):
    return G.boundary_flags(hp.nx, hp.ny, hp.nz) == 0


def setup(walls=(0,) * 6, dims=(14, 12, 11), nsteps=4, snaps=2, seed=0, amp=0.25,
          dx=1.0 / 16):
    st = small_random_box(nx=dims[0], ny=dims[1], nz=dims[2], walls=walls, seed=seed, amp=amp,
                          cfl=0.4, dx=dx)
    # ghosts as the donor rule fills them, so the oracle starts from the same state
    from boxzyhydro_b200.hydro import apply_ghost_plan, ghost_plan
    pl = ghost_plan(st.params)
    st.cons[:] = apply_ghost_plan(st.cons, pl["src2"], pl["sgn2"], pl["dst"])
    st.u[:] = st.cons[:, 1:4] / st.cons[:, :1]
    eng = AdjointEngine(st.params, nsteps, snaps)
    return st, eng


def fwd(eng, cons, frozen):
    torch = _torch()
    c0 = torch.tensor(np.ascontiguousarray(cons.T), device="cuda")
    out = torch.empty_like(c0)
    torch.cuda.synchronize()
    eng.forward_ptr(c0.data_ptr(), out.data_ptr(), frozen=frozen)
    return out.cpu().numpy().T.copy()


def bwd(eng, lamT):
    torch = _torch()
    l = torch.tensor(np.ascontiguousarray(lamT.T), device="cuda")
    out = torch.empty_like(l)
    torch.cuda.synchronize()
    eng.backward_ptr(l.data_ptr(), out.data_ptr())
    return out.cpu().numpy().T.copy()


def rand_dir(hp, rng, scale):
    m = interior_mask(hp)
    v = rng.standard_normal((hp.ngrid, 5)) * scale
    v[~m] = 0.0
    return v


@pytest.mark.parametrize("walls,dims,dx", [((0,) * 6, (14, 12, 11), 1.0 / 16),
                                           ((1, 1, 1, 1, 1, 1), (40, 9, 4), 1.0 / 16),
                                           ((0, 1, 1, 0, 0, 1), (13, 12, 10), 1.0 / 16),
                                           ((0,) * 6, (15, 13, 12), 1.0 / 12)])
def test_dot_product(walls, dims, dx):
    st, eng = setup(walls, dims, dx=dx)
    hp = st.params
    consT = fwd(eng, st.cons, frozen=False)
    dts = eng.dts()
    rng = np.random.default_rng(7)
    scale = np.array([1.0, 0.3, 0.3, 0.3, 2.0])
    v = rand_dir(hp, rng, scale)
    cT, dT = TLM.run(hp, st.cons, v, dts)
    m = interior_mask(hp)
    assert np.allclose(cT[m], consT[m], rtol=1e-13, atol=0), "TLM forward differs from GPU"
    lamT = rand_dir(hp, rng, np.ones(5))
    lam0 = bwd(eng, lamT)
    assert np.all(lam0[~m] == 0.0)
    d1 = float(np.sum(lamT[m] * dT[m]))
    d2 = float(np.sum(lam0[m] * v[m]))
    assert abs(d1 - d2) <= 1e-12 * abs(d1), (d1, d2)
    eng.close()


def test_reflective_3d_box_takes_the_per_phase_dt_sequence():
    """A reflective 3-D box: its two-sweep ghost plan leaves corner ghosts
    lagging, which enter only the Courant maximum, so the engine takes the dt
    sequence of the per-phase kernels and runs the fused stage arithmetic with
    it.  The forward equals the oracle's run of the reference loop bit for bit
    (dt sequence included), and the dot-product test holds to 1e-12."""
    from boxzyhydro_b200.hydro import apply_ghost_plan, ghost_plan
    walls, dims = (1,) * 6, (14, 12, 11)
    st, eng = setup(walls, dims, nsteps=6, snaps=3)
    hp = st.params
    pl = ghost_plan(hp)
    assert not pl["fused_ok"]
    consT = fwd(eng, st.cons, frozen=False)
    dts = eng.dts()
    # the oracle from the state the engine starts from: two calls of the fill
    c = st.cons.copy()
    for _ in range(2):
        c = apply_ghost_plan(c, pl["src2"], pl["sgn2"], pl["dst"])
    o = O.Oracle(hp)
    o.set_state(c, c[:, 1:4] / c[:, :1], np.ones(hp.ngrid), np.full(hp.ngrid, hp.gammafix))
    odts = []
    for _ in range(6):
        assert o.step()
        odts.append(o.clock()["dt"])
    m = interior_mask(hp)
    assert np.array_equal(np.array(odts), dts)
    assert np.array_equal(o.get_state()[0][m], consT[m])
    o.close()
    rng = np.random.default_rng(9)
    v = rand_dir(hp, rng, np.array([1.0, 0.3, 0.3, 0.3, 2.0]))
    cT, dT = TLM.run(hp, st.cons, v, dts)
    assert np.allclose(cT[m], consT[m], rtol=1e-13, atol=0), "TLM forward differs from GPU"
    lamT = rand_dir(hp, rng, np.ones(5))
    lam0 = bwd(eng, lamT)
    d1 = float(np.sum(lamT[m] * dT[m]))
    d2 = float(np.sum(lam0[m] * v[m]))
    assert abs(d1 - d2) <= 1e-12 * abs(d1), (d1, d2)
    eng.close()


def test_dot_product_32cubed_twenty_steps():
    """The dot-product test on a 32^3-interior box over 20 steps with 5 snapshots
    (the checkpoint schedule recomputes), 1e-12 relative."""
    st, eng = setup((0,) * 6, (36, 36, 36), nsteps=20, snaps=5, dx=1.0 / 32)
    hp = st.params
    consT = fwd(eng, st.cons, frozen=False)
    dts = eng.dts()
    rng = np.random.default_rng(17)
    v = rand_dir(hp, rng, np.array([1.0, 0.3, 0.3, 0.3, 2.0]))
    cT, dT = TLM.run(hp, st.cons, v, dts)
    m = interior_mask(hp)
    assert np.allclose(cT[m], consT[m], rtol=1e-13, atol=0), "TLM forward differs from GPU"
    lamT = rand_dir(hp, rng, np.ones(5))
    lam0 = bwd(eng, lamT)
    assert eng.stats()["recomputed_steps"] > 0
    d1 = float(np.sum(lamT[m] * dT[m]))
    d2 = float(np.sum(lam0[m] * v[m]))
    assert abs(d1 - d2) <= 1e-12 * abs(d1), (d1, d2)
    eng.close()


def test_finite_differences_gpu_and_oracle():
    st, eng = setup()
    hp = st.params
    fwd(eng, st.cons, frozen=False)
    dts = eng.dts()
    rng = np.random.default_rng(11)
    m = interior_mask(hp)
    lamT = np.zeros((hp.ngrid, 5))
    lamT[m, 0] = rng.standard_normal(m.sum())
    lam0 = bwd(eng, lamT)
    for k in range(3):
        v = rand_dir(hp, rng, np.array([1.0, 0.3, 0.3, 0.3, 2.0]))
        adj = float(np.sum(lam0[m] * v[m]))
        h = 1e-7
        # GPU forward with the frozen dt sequence
        fp = fwd(eng, st.cons + h * v, frozen=True)
        fm = fwd(eng, st.cons - h * v, frozen=True)
        fd = float(np.sum(lamT[m] * (fp[m] - fm[m]))) / (2 * h)
        assert abs(fd - adj) <= 1e-6 * abs(adj), (fd, adj)
        # the oracle (CPU restatement of the reference loop) with the same dts
        vals = []
        for sgn in (1.0, -1.0):
            c = st.cons + sgn * h * v
            from boxzyhydro_b200.hydro import apply_ghost_plan, ghost_plan
            pl = ghost_plan(hp)
            c = apply_ghost_plan(c, pl["src2"], pl["sgn2"], pl["dst"])
            o = O.Oracle(hp)
            o.set_state(c, c[:, 1:4] / c[:, :1], np.ones(hp.ngrid), np.full(hp.ngrid, hp.gammafix))
            for dt in dts:
                o.step_dt(dt)
            vals.append(o.get_state()[0])
            o.close()
        fdo = float(np.sum(lamT[m] * (vals[0][m] - vals[1][m]))) / (2 * h)
        assert abs(fdo - adj) <= 1e-6 * abs(adj), (fdo, adj)
    eng.close()


def fwd_branches(eng, base, pert):
    torch = _torch()
    b = torch.tensor(np.ascontiguousarray(base.T), device="cuda")
    p = torch.tensor(np.ascontiguousarray(pert.T), device="cuda")
    ob, op = torch.empty_like(b), torch.empty_like(p)
    torch.cuda.synchronize()
    eng.forward_branches_ptr(b.data_ptr(), p.data_ptr(), ob.data_ptr(), op.data_ptr())
    return ob.cpu().numpy().T.copy(), op.cpu().numpy().T.copy()


@pytest.mark.parametrize("walls,dims", [((0,) * 6, (20, 18, 16)), ((1, 1, 1, 1, 0, 0), (30, 12, 4))])
def test_frozen_branch_differences_on_a_state_with_ties(walls, dims):
    """A state with flat regions at rest (a split state plus a blob, like the
    128^3 adjoint configuration): genminmod and the HLL wave speeds sit on ties
    there, so central differences of the step itself do not converge.  With the
    branches held where the base run takes them (bx_adj_forward_branches) they
    match the adjoint to 1e-6.  The base of that run is bx_adj_forward's run bit
    for bit, and a perturbed run from the base state is the base run."""
    from boxzyhydro_b200 import ic
    nx, ny, nz = dims
    hp = small_random_box(nx=nx, ny=ny, nz=nz, walls=walls, cfl=0.4, dx=1.0 / 16).params
    g = G.cell_centres(hp.nx, hp.ny, hp.nz, hp.dx, hp.dy, hp.dz)
    x, y, z = g
    rho = np.where(x < 0.0, 1.0, 0.125) * (1.0 + 0.05 * np.exp(-((x - 0.1) ** 2 + y ** 2 + z ** 2) / 0.01))
    p = np.where(x < 0.0, 1.0, 0.1)
    cons = np.zeros((hp.ngrid, 5))
    cons[:, 0] = rho
    cons[:, 4] = p / (hp.gammafix - 1.0)
    from boxzyhydro_b200.hydro import apply_ghost_plan, ghost_plan
    pl = ghost_plan(hp)
    cons = apply_ghost_plan(cons, pl["src2"], pl["sgn2"], pl["dst"])
    eng = AdjointEngine(hp, 6, 2)
    consT = fwd(eng, cons, frozen=False)
    m = interior_mask(hp)
    ob, op = fwd_branches(eng, cons, cons)
    assert np.array_equal(ob[m], consT[m]), "base run differs from the forward run"
    assert np.array_equal(op[m], ob[m]), "perturbed run from the base state differs"
    rng = np.random.default_rng(31)
    lamT = np.zeros((hp.ngrid, 5))
    lamT[m, 0] = rng.standard_normal(m.sum())
    lam0 = bwd(eng, lamT)
    h = 1e-7
    free, frozen = [], []
    for k in range(4):
        v = rand_dir(hp, rng, np.array([1.0, 0.3, 0.3, 0.3, 2.0]))
        adj = float(np.sum(lam0[m] * v[m]))
        _, fp = fwd_branches(eng, cons, cons + h * v)
        _, fm = fwd_branches(eng, cons, cons - h * v)
        frozen.append(abs(float(np.sum(lamT[m] * (fp[m] - fm[m]))) / (2 * h) - adj) / abs(adj))
        gp = fwd(eng, cons + h * v, frozen=True)
        gm = fwd(eng, cons - h * v, frozen=True)
        free.append(abs(float(np.sum(lamT[m] * (gp[m] - gm[m]))) / (2 * h) - adj) / abs(adj))
    assert max(frozen) <= 1e-6, (frozen, free)
    eng.close()


def test_checkpoint_schedules_agree():
    st, eng1 = setup(nsteps=6, snaps=1)
    hp = st.params
    fwd(eng1, st.cons, frozen=False)
    rng = np.random.default_rng(3)
    lamT = rand_dir(hp, rng, np.ones(5))
    ref = bwd(eng1, lamT)
    s1 = eng1.stats()
    assert s1["recomputed_steps"] == plan(6, 1)["recomputed_first"]
    eng1.close()
    for snaps in (2, 3, 6):
        eng = AdjointEngine(hp, 6, snaps)
        fwd(eng, st.cons, frozen=False)
        got = bwd(eng, lamT)
        assert np.array_equal(got, ref), snaps
        st_ = eng.stats()
        assert st_["recomputed_steps"] <= s1["recomputed_steps"]
        # the host's plan of the schedule is the walk the engine took
        assert st_["recomputed_steps"] == plan(6, snaps)["recomputed_first"], snaps
        assert st_["device_bytes"] == device_bytes(hp, 6, snaps), snaps
        eng.close()


def test_kept_stage0_results_give_the_same_gradient():
    st, eng = setup(nsteps=5, snaps=2)
    hp = st.params
    fwd(eng, st.cons, frozen=False)
    rng = np.random.default_rng(5)
    lamT = rand_dir(hp, rng, np.ones(5))
    ref = bwd(eng, lamT)
    r0 = eng.stats()["recomputed_steps"]
    eng.keep_stage0(True)
    fwd(eng, st.cons, frozen=False)
    got = bwd(eng, lamT)
    assert np.array_equal(got, ref)
    assert eng.stats()["recomputed_steps"] == r0
    eng.close()


def test_stage0_cache_sizes_give_the_same_gradient():
    """The backward pass's cache of stage-0 results changes what is recomputed,
    not the gradient: 2, 3 and 8 entries, a backward repeated after a resize."""
    st, eng = setup(nsteps=24, snaps=3)
    hp = st.params
    fwd(eng, st.cons, frozen=False)
    rng = np.random.default_rng(6)
    lamT = rand_dir(hp, rng, np.ones(5))
    ref = bwd(eng, lamT)
    for entries in (3, 8, 2):
        eng.stage0_cache(entries)
        fwd(eng, st.cons, frozen=False)
        assert np.array_equal(bwd(eng, lamT), ref), entries
    eng.close()


def test_host_level_gives_the_same_gradient():
    """States every `stride` steps in pinned host memory, the segments between
    them reversed one by one: the same gradient bit for bit as the device-only
    schedule, each state recomputed once when a segment fits the free plane sets,
    and a second backward of the same run (segment starts fetched again) equal
    to the first."""
    from boxzyhydro_b200._lib import BoxzyError
    st, eng = setup(nsteps=23, snaps=8)
    hp = st.params
    fwd(eng, st.cons, frozen=False)
    rng = np.random.default_rng(8)
    lamT = rand_dir(hp, rng, np.ones(5))
    ref = bwd(eng, lamT)
    for stride, entries in ((7, 2), (5, 8), (2, 2)):
        eng.stage0_cache(entries)
        nbytes = eng.host_level(stride)
        assert nbytes == ((23 - 1) // stride) * 5 * hp.ngrid * 8
        fwd(eng, st.cons, frozen=False)
        got = bwd(eng, lamT)
        assert np.array_equal(got, ref), stride
        # six free plane sets: every segment reversed with each state computed once
        nseg = (23 + stride - 1) // stride
        assert eng.stats()["recomputed_steps"] == 23 - nseg, stride
        assert np.array_equal(bwd(eng, lamT), ref), stride
    # the level set after the forward run: refused until the forward runs again
    eng.host_level(4)
    with pytest.raises(BoxzyError):
        bwd(eng, lamT)
    eng.host_level(0)
    fwd(eng, st.cons, frozen=False)
    assert np.array_equal(bwd(eng, lamT), ref)
    with pytest.raises(BoxzyError):
        eng.host_level(1)
    eng.close()
    _, small = setup(nsteps=10, snaps=2)
    with pytest.raises(BoxzyError):
        small.host_level(3)
    small.close()


def test_torch_autograd_function():
    torch = _torch()
    st, eng = setup()
    hp = st.params
    m = torch.tensor(interior_mask(hp), device="cuda")
    c0 = torch.tensor(np.ascontiguousarray(st.cons.T), device="cuda", requires_grad=True)
    cT = AdjointRun.apply(c0, eng)
    target = cT.detach()[0] * 1.01
    loss = 0.5 * torch.sum(((cT[0] - target) * m) ** 2)
    loss.backward()
    lamT = torch.zeros_like(cT)
    lamT[0] = (cT.detach()[0] - target) * m
    ref = torch.empty_like(lamT)
    eng.backward_ptr(lamT.contiguous().data_ptr(), ref.data_ptr())
    torch.cuda.synchronize()
    assert torch.equal(c0.grad, ref)
    assert float(torch.abs(c0.grad).sum()) > 0
    eng.close()
