"""Checkpoint schedule of the discrete adjoint (bx_adj_plan, host only): the steps
the backward pass recomputes against the optimum of the recursion it follows.

Reversing l steps with s free snapshot slots beside the held state costs
C(l, s) = min_m m + C(l-m, s-1) + C(m, s), C(l, 0) = l(l-1)/2, C(1, s) = 0, whose
closed form is Griewank's (1992): with c = s + 1 checkpoints and r the smallest
integer with (c+r over c) >= l, C(l, s) = r l - (c+1+r-1 over c+1).  The first
backward after a forward run reverses the chain of snapshots the forward stored
without advancing to them: F(l, s) = min_m F(l-m, s-1) + C(m, s), F(l, 0) = C(l, 0).
The library solves the recursion by dynamic programming up to l^2 s = 4e8 and by
closed-form split rules beyond; both are checked here, the second at sizes no GPU
test reaches.  bx_adj_device_bytes, the engine's memory computed on the host, is
checked against the device bytes the engine reported in the adjoint bench runs."""
from math import comb

import numpy as np
import pytest

from boxzyhydro_b200._lib import BoxzyError
from boxzyhydro_b200 import ic
from boxzyhydro_b200.adjoint import device_bytes, plan


def closed_c(l, s):
    """Griewank's minimal number of recomputed steps (s free slots)."""
    if l <= 1:
        return 0
    c = s + 1
    r = 0
    while comb(c + r, c) < l:
        r += 1
    return r * l - comb(c + r, r - 1)


def dp_tables(L, S):
    C = np.zeros((L + 1, S + 1), dtype=np.int64)
    F = np.zeros((L + 1, S + 1), dtype=np.int64)
    for l in range(2, L + 1):
        C[l, 0] = F[l, 0] = l * (l - 1) // 2
    for s in range(1, S + 1):
        for l in range(2, L + 1):
            m = np.arange(1, l)
            C[l, s] = (m + C[l - m, s - 1] + C[m, s]).min()
            F[l, s] = (F[l - m, s - 1] + C[m, s]).min()
    return C, F


def f_minplus(L, S):
    """F(L, S) by S min-plus convolutions of closed-form C columns."""
    ls = np.arange(L + 1, dtype=np.int64)
    Fp = ls * (ls - 1) // 2
    Fp[:2] = 0
    for s in range(1, S + 1):
        Cs = np.array([closed_c(int(l), s) for l in ls], dtype=np.int64)
        Fn = np.zeros(L + 1, dtype=np.int64)
        lo = L if s == S else 2
        for l in range(lo, L + 1):
            m = np.arange(1, l)
            Fn[l] = (Fp[l - m] + Cs[m]).min()
        Fp = Fn
    return int(Fp[L])


def test_small_runs_match_the_recursion_and_the_closed_form():
    L, S = 60, 6
    C, F = dp_tables(L, S)
    for l in range(1, L + 1):
        for s in range(1, S + 1):
            p = plan(l, s)
            se = min(s, l)  # the engine holds at most one slot per step
            assert p["recomputed_again"] == C[l, se] == closed_c(l, se), (l, s)
            assert p["recomputed_first"] == F[l, se], (l, s)
            assert p["chain_snapshots"] == min(se, l - 1), (l, s)


@pytest.mark.parametrize("L,S", [(12000, 3), (30000, 1), (5000, 200), (100000, 40),
                                 (1000000, 20)])
def test_long_runs_beyond_the_table_reach_the_optimum(L, S):
    """l^2 s > 4e8: the split follows the closed-form rules."""
    assert L * L * S > 4e8
    p = plan(L, S)
    assert p["recomputed_again"] == closed_c(L, S)
    if L <= 30000:
        assert p["recomputed_first"] == f_minplus(L, S)
    assert p["recomputed_first"] <= p["recomputed_again"]


def test_more_snapshots_never_recompute_more():
    for L in (7, 50, 200, 1000):
        prev = None
        for s in range(1, 24):
            p = plan(L, s)
            if prev is not None:
                assert p["recomputed_first"] <= prev["recomputed_first"], (L, s)
                assert p["recomputed_again"] <= prev["recomputed_again"], (L, s)
            prev = p


def test_one_slot_per_step_stores_every_state():
    p = plan(200, 199)
    assert p == dict(recomputed_first=0, recomputed_again=199, chain_snapshots=199)
    assert plan(1, 5) == dict(recomputed_first=0, recomputed_again=0, chain_snapshots=0)


def test_bad_arguments_are_rejected():
    with pytest.raises(BoxzyError):
        plan(0, 3)
    with pytest.raises(BoxzyError):
        plan(10, 0)


@pytest.mark.parametrize("n,nsteps,snaps,entries,keep,measured", [
    # engine_device_bytes of the adjoint bench runs on a B200
    (128, 200, 15, 8, False, 3109558336),     # C4
    (128, 200, 15, 2, True, 20957310016),     # C4, stage-0 results kept
    (128, 200, 199, 2, True, 37885074496),    # C4, every state kept
    (512, 400, 11, 6, False, 152775565952)])  # C5
def test_device_bytes_match_the_engines_measured(n, nsteps, snaps, entries, keep, measured):
    hp = ic.turbulent_params(n)
    assert device_bytes(hp, nsteps, snaps, entries, keep) == measured


def test_device_bytes_grow_by_one_plane_set_per_snapshot():
    hp = ic.turbulent_params(32)
    one = 5 * hp.ngrid * 8
    assert device_bytes(hp, 50, 8) - device_bytes(hp, 50, 7) == one
    assert device_bytes(hp, 50, 8, stage0_cache=5) - device_bytes(hp, 50, 8) == 3 * one
    assert device_bytes(hp, 50, 80) == device_bytes(hp, 50, 50)  # at most one per step
    with pytest.raises(BoxzyError):
        device_bytes(hp, 50, 8, stage0_cache=1)


def test_device_bytes_refuses_the_grids_the_engine_refuses():
    import dataclasses
    hp = ic.turbulent_params(16)
    with pytest.raises(BoxzyError) as e:
        device_bytes(dataclasses.replace(hp, fluxangmom=True), 20, 4)
    assert e.value.code == 3  # BX_ERR_UNSUPPORTED: flux_ang runs on the per-phase kernels
    # a tabulated EOS: the engine has no reverse of the table lookup
    with pytest.raises(BoxzyError) as e:
        device_bytes(dataclasses.replace(hp, h2stat=1), 20, 4)
    assert e.value.code == 3
    # a reflective 3-D box is taken: its lagging corner ghosts enter only the
    # Courant maximum (the engine takes the dt sequence of the per-phase kernels)
    walls = {f"no_outflow_{w}": True for w in ("xl", "xr", "yl", "yr", "zl", "zr")}
    assert device_bytes(dataclasses.replace(hp, **walls), 20, 4) == device_bytes(hp, 20, 4)
    with pytest.raises(BoxzyError) as e:  # int32 cell indices, as bx_create
        device_bytes(dataclasses.replace(hp, nx=1300, ny=1300, nz=1300), 20, 4)
    assert e.value.code == 1
    assert device_bytes(hp, 20, 4) > 0
