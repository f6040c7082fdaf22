"""The tangent-linear model (oracle/tangent.py), which checks the GPU adjoint by the
dot-product test, checked here on its own against the CPU oracle: its values
follow the oracle's run with the same dt sequence, and its tangents match central
finite differences of the oracle's run along random directions."""
import numpy as np
import pytest

import oracle as O
import tangent as TLM
from boxzyhydro_b200 import grid as G
from boxzyhydro_b200.hydro import apply_ghost_plan, ghost_plan
from tests.helpers import small_random_box


def start_state(walls, dims, seed, dx=1.0 / 16):
    st = small_random_box(nx=dims[0], ny=dims[1], nz=dims[2], walls=walls, seed=seed,
                          amp=0.25, cfl=0.4, dx=dx)
    pl = ghost_plan(st.params)
    st.cons[:] = apply_ghost_plan(st.cons, pl["src2"], pl["sgn2"], pl["dst"])
    return st


def oracle_run(hp, cons, dts=None, nsteps=0):
    """The reference loop from cons: with the given dt sequence, or nsteps by the
    CFL rule (then the dt of each step is returned)."""
    c = apply_ghost_plan(cons, *(lambda p: (p["src2"], p["sgn2"], p["dst"]))(ghost_plan(hp)))
    o = O.Oracle(hp)
    o.set_state(c, c[:, 1:4] / c[:, :1], np.ones(hp.ngrid), np.full(hp.ngrid, hp.gammafix))
    out_dts = []
    if dts is None:
        for _ in range(nsteps):
            o.step()
            out_dts.append(o.clock()["dt"])
    else:
        for dt in dts:
            o.step_dt(dt)
    res = o.get_state()[0]
    o.close()
    return res, np.array(out_dts)


def rand_dir(hp, rng, scale):
    m = G.boundary_flags(hp.nx, hp.ny, hp.nz) == 0
    v = rng.standard_normal((hp.ngrid, 5)) * scale
    v[~m] = 0.0
    return v


@pytest.mark.parametrize("walls,dims", [((0,) * 6, (14, 12, 11)),
                                        ((0, 1, 1, 0, 0, 1), (13, 12, 10)),
                                        ((1, 1, 1, 1, 1, 1), (40, 9, 4))])
def test_tangent_model_against_oracle_finite_differences(walls, dims):
    st = start_state(walls, dims, seed=3)
    hp = st.params
    m = G.boundary_flags(hp.nx, hp.ny, hp.nz) == 0
    cref, dts = oracle_run(hp, st.cons, nsteps=4)
    rng = np.random.default_rng(8)
    scale = np.array([1.0, 0.3, 0.3, 0.3, 2.0])
    for k in range(3):
        v = rand_dir(hp, rng, scale)
        cT, dT = TLM.run(hp, st.cons, v, dts)
        # values: the fused map the model follows gives the reference loop's result
        assert np.allclose(cT[m], cref[m], rtol=1e-13, atol=0)
        # tangents: central differences of the oracle with the dt sequence held
        h = 1e-7
        fp = oracle_run(hp, st.cons + h * v, dts=dts)[0]
        fm = oracle_run(hp, st.cons - h * v, dts=dts)[0]
        fd = (fp[m] - fm[m]) / (2 * h)
        err = np.linalg.norm(fd - dT[m]) / np.linalg.norm(dT[m])
        assert err < 1e-6, (k, err)
        # and projected on a random adjoint direction, as the GPU test projects
        lam = rng.standard_normal(fd.shape)
        a, b = float(np.sum(lam * fd)), float(np.sum(lam * dT[m]))
        assert abs(a - b) <= 1e-6 * abs(b), (a, b)


def test_tangent_is_linear_in_the_direction():
    """J(a v + b w) = a J v + b J w: the tangent carries no value-dependent
    branching of its own."""
    st = start_state((0,) * 6, (12, 11, 10), seed=4)
    hp = st.params
    _, dts = oracle_run(hp, st.cons, nsteps=3)
    rng = np.random.default_rng(9)
    v = rand_dir(hp, rng, np.ones(5))
    w = rand_dir(hp, rng, np.ones(5))
    _, dv = TLM.run(hp, st.cons, v, dts)
    _, dw = TLM.run(hp, st.cons, w, dts)
    _, dvw = TLM.run(hp, st.cons, 2.0 * v - 0.5 * w, dts)
    assert np.allclose(dvw, 2.0 * dv - 0.5 * dw, rtol=1e-12, atol=1e-12 * np.abs(dvw).max())
