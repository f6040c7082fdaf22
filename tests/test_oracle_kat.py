"""Known-answer tests of the oracle's building blocks and conservation of its
step: generalised minmod (utils.f90:696-707) and the limited slope with
theta = 1.25 (utils.f90:738-741, Makefile:20), interface_muscl (flux.f90:299-308)
with and without Courant terms, the HLL face flux (flux.f90:513-590) on equal
states (the Euler flux), on supersonic states (the upwind flux), on mirrored
states (a reflective wall: no mass or energy through it) and against a numpy
restatement of the Harten-Lax-van Leer formula with Davis's wave-speed bounds;
the conservative form of the update (interior faces cancel; totals change by
the flux through the boundary faces, whose ghost states have no slope), and
mass kept to round-off where the walls see no normal velocity; the tabulated
EOS on ideal-gas tables reproducing the fixed-gamma state."""
import numpy as np
import pytest

import oracle as O
from boxzyhydro_b200 import grid as G
from tests.helpers import small_random_box


def test_genminmod_branches():
    cases = [((1.0, 2.0, 3.0), 1.0), ((3.0, 2.0, 1.0), 1.0), ((2.0, 0.5, 3.0), 0.5),
             ((-1.0, -2.0, -3.0), -1.0), ((-3.0, -2.0, -0.25), -0.25),
             ((1.0, -2.0, 3.0), 0.0), ((-1.0, 2.0, -3.0), 0.0),
             ((0.0, 1.0, 2.0), 0.0), ((-1.0, 0.0, -2.0), 0.0), ((0.0, 0.0, 0.0), 0.0)]
    for args, want in cases:
        got = O.kat_genminmod(*args)
        assert got == want, (args, got, want)
        assert not np.signbit(got) or want < 0, args  # the zero branch returns +0


@pytest.mark.parametrize("c,want", [((0.0, 1.0, 2.0), 1.0),     # linear: the central slope
                                    ((0.0, 1.0, 3.0), 1.25),    # theta * left difference
                                    ((0.0, 2.0, 3.0), 1.25),    # theta * right difference
                                    ((3.0, 2.0, 0.0), -1.25),
                                    ((0.0, 1.0, 0.0), 0.0),     # extremum: flat
                                    ((0.0, 0.0, 1.0), 0.0)])
def test_slope_limiter_known_answers(c, want):
    assert O.kat_slope(*c) == want


def test_slope_matches_the_formula_bit_for_bit():
    rng = np.random.default_rng(1)
    c = rng.standard_normal((2000, 3))
    for c0, c1, c2 in c:
        a, b, d = 1.25 * (c1 - c0), 0.5 * (c2 - c0), 1.25 * (c2 - c1)
        want = min(a, min(b, d)) if (a > 0 and b > 0 and d > 0) else (
            max(a, max(b, d)) if (a < 0 and b < 0 and d < 0) else 0.0)
        assert O.kat_slope(c0, c1, c2) == want


def test_muscl_states():
    # no Courant terms: the cell value minus and plus half the slope, exactly
    for q, s in [(1.0, 0.3), (-2.5, 1e-3), (0.125, -0.75)]:
        assert O.kat_muscl(q, 0.0, 0.0, s) == (q - 0.5 * s, q + 0.5 * s)
    rng = np.random.default_rng(2)
    for q, lm, lp, s in rng.standard_normal((500, 4)):
        lm, lp = -abs(lm), abs(lp)  # lambda_minus <= 0 <= lambda_plus
        m, p = O.kat_muscl(q, lm, lp, s)
        assert m == q + 0.5 * (-1.0 - lm) * s and p == q + 0.5 * (1.0 - lp) * s


def euler_flux(st, idir):
    """The exact flux of a state (rho, u1, u2, u3, p, eps, gamma) through a face
    normal to idir, with E = eps + rho |u|^2 / 2 as the face uses it."""
    rho, u, p, eps = st[0], np.asarray(st[1:4]), st[4], st[5]
    E = eps + 0.5 * rho * float(u @ u)
    vn = u[idir]
    f = np.array([rho * vn, rho * u[0] * vn, rho * u[1] * vn, rho * u[2] * vn, (E + p) * vn])
    f[1 + idir] += p
    return f


def random_state(rng, mach=1.0):
    rho, p, gam = np.exp(rng.uniform(-1, 1)), np.exp(rng.uniform(-1, 1)), rng.choice([1.4, 5 / 3])
    c = np.sqrt(gam * p / rho)
    u = rng.uniform(-1, 1, 3) * mach * c
    return np.array([rho, *u, p, p / (gam - 1.0), gam])


@pytest.mark.parametrize("idir", [0, 1, 2])
def test_hll_of_equal_states_is_the_euler_flux(idir):
    rng = np.random.default_rng(10 + idir)
    for _ in range(200):
        st = random_state(rng, mach=3.0)
        f = O.kat_face_flux(st, st, idir)
        assert np.allclose(f, euler_flux(st, idir), rtol=1e-14, atol=1e-15 * np.abs(st).max())


@pytest.mark.parametrize("idir", [0, 1, 2])
def test_hll_of_supersonic_states_is_upwind(idir):
    rng = np.random.default_rng(20 + idir)
    for _ in range(100):
        L, R = random_state(rng), random_state(rng)
        for s in (L, R):
            s[1 + idir] = 1.5 * np.sqrt(s[6] * s[4] / s[0]) + rng.uniform(0, 1)
        assert np.allclose(O.kat_face_flux(L, R, idir), euler_flux(L, idir), rtol=1e-15, atol=0)
        Lm, Rm = L.copy(), R.copy()
        Lm[1 + idir] *= -1
        Rm[1 + idir] *= -1
        assert np.allclose(O.kat_face_flux(Lm, Rm, idir), euler_flux(Rm, idir), rtol=1e-15, atol=0)


@pytest.mark.parametrize("idir", [0, 1, 2])
def test_hll_at_a_mirror_passes_no_mass_or_energy(idir):
    rng = np.random.default_rng(30 + idir)
    for _ in range(200):
        L = random_state(rng, mach=2.0)
        R = L.copy()
        R[1 + idir] = -L[1 + idir]
        f = O.kat_face_flux(L, R, idir)
        assert f[0] == 0.0 and f[4] == 0.0
        for t in range(3):
            if t != idir:
                assert f[1 + t] == 0.0


def test_hll_matches_the_formula_bit_for_bit():
    """F = (a+ F_L + a- F_R - a+ a- (U_R - U_L)) / (a+ + a-), a+ = max(0, v_R + c_R,
    v_L + c_L), a- = max(0, c_R - v_R, c_L - v_L), in flux.f90's order."""
    rng = np.random.default_rng(4)
    for k in range(600):
        idir = k % 3
        L, R = random_state(rng, 2.0), random_state(rng, 2.0)
        U, F = [], []
        for s in (L, R):
            d, vx, vy, vz, p, e = s[:6]
            u = [d, d * vx, d * vy, d * vz, e + 0.5 * d * (vx * vx + vy * vy + vz * vz)]
            v = s[1 + idir]
            f = [0.0] * 5
            f[1 + idir] = p
            f = [u[0] * v, f[1] + u[1] * v, f[2] + u[2] * v, f[3] + u[3] * v, (u[4] + p) * v]
            U.append(u)
            F.append(f)
        cl = np.sqrt(L[6] * L[4] / L[0])
        cr = np.sqrt(R[6] * R[4] / R[0])
        vl, vr = L[1 + idir], R[1 + idir]
        ap = max(max(0.0, vr + cr), vl + cl)
        am = max(max(0.0, -(vr - cr)), -(vl - cl))
        want = [(ap * F[0][i] + am * F[1][i] - ap * am * (U[1][i] - U[0][i])) / (ap + am)
                for i in range(5)]
        assert list(O.kat_face_flux(L, R, idir)) == want, k


def _cell_q(c, u, p, g, small_eps):
    """Per-cell reconstruction variables (rho, u1, u2, u3, p, eps, gamma) as
    calculate_slopes/calculate_states form them (eps from the u array)."""
    eps = np.maximum(c[:, 4] - 0.5 * c[:, 0] * (u[:, 0] * u[:, 0] + u[:, 1] * u[:, 1] +
                                                u[:, 2] * u[:, 2]), small_eps)
    return np.stack([c[:, 0], u[:, 0], u[:, 1], u[:, 2], p, eps, g], axis=1)


def _face_state(q, sten, side, idir, dt, ds):
    """Face state of cell sten[1] (stencil minus, centre, plus along idir): its
    'minus' (side -1) or 'plus' (side +1) state by slope and interface_muscl."""
    qc = q[sten[1]]
    sound = np.sqrt(qc[4] * qc[6] / qc[0])
    lp = max(qc[1 + idir] + sound, 0.0) * dt / ds
    lm = min(qc[1 + idir] - sound, 0.0) * dt / ds
    out = np.empty(7)
    for v in range(7):
        sl = O.kat_slope(q[sten[0], v], qc[v], q[sten[2], v])
        out[v] = O.kat_muscl(qc[v], lm, lp, sl)[0 if side < 0 else 1]
    return out


@pytest.mark.parametrize("avg", [0, 1])
def test_flux_is_conservative_and_walls_are_first_order(avg):
    """One flux call on a 2-D box with reflective walls: the change of every
    conserved total over the interior equals the flux through the boundary faces,
    where the ghost cell's state has no slope (flux.f90:53-57 gives every ghost the
    stencil (igrid, igrid, igrid)) and the interior cell's has its limited slope.
    Interior faces cancel to round-off.  The reference therefore does not keep mass
    exactly with reflective walls: the two states of a wall face are not mirror
    images unless the slope of the wall-normal velocity vanishes there.  With
    avg = 1 (the second stage, flux.f90:209-216) the totals are half those of the
    step input, the stage input and the boundary flux."""
    st = small_random_box(nx=20, ny=12, nz=1, walls=(1,) * 6, seed=5, amp=0.3)
    hp = st.params
    inner = G.boundary_flags(hp.nx, hp.ny, hp.nz) == 0
    o = O.Oracle(hp)
    o.set_state(st.cons, st.u, st.p, np.full(hp.ngrid, hp.gammafix))
    for _ in range(2):
        o.step()  # ghosts, u and p as the loop leaves them
    dt = 1e-3
    o.set_clock(0.0, dt, 0.0, 0)
    c0, u0, p0, g0 = o.get_state()
    q = _cell_q(c0, u0, p0, g0, hp.small_eps)
    nx, ny = hp.nx, hp.ny
    idx = lambda ix, iy: iy * nx + ix  # noqa: E731 (0-based, x fastest)
    vol, ayz, axz = hp.dx * hp.dy * hp.dz, hp.dy * hp.dz, hp.dx * hp.dz
    boundary = np.zeros(5)
    for iy in range(2, ny - 2):
        for ix, ghost, side in ((2, 1, -1), (nx - 3, nx - 2, +1)):
            cell = _face_state(q, (idx(ix - 1, iy), idx(ix, iy), idx(ix + 1, iy)), side, 0, dt, hp.dx)
            g = q[idx(ghost, iy)]
            f = O.kat_face_flux(g, cell, 0) if side < 0 else O.kat_face_flux(cell, g, 0)
            boundary += side * ayz * f
    for ix in range(2, nx - 2):
        for iy, ghost, side in ((2, 1, -1), (ny - 3, ny - 2, +1)):
            cell = _face_state(q, (idx(ix, iy - 1), idx(ix, iy), idx(ix, iy + 1)), side, 1, dt, hp.dy)
            g = q[idx(ix, ghost)]
            f = O.kat_face_flux(g, cell, 1) if side < 0 else O.kat_face_flux(cell, g, 1)
            boundary += side * axz * f
    old = c0 * (1.0 + 0.01 * np.cos(np.arange(c0.size)).reshape(c0.shape))
    o.set_cons_old(old)
    o.flux(avg)
    c1 = o.get_state()[0]
    if avg == 0:
        change = (c1[inner] - c0[inner]).sum(axis=0)
        want = -boundary * dt / vol
    else:
        change = c1[inner].sum(axis=0)
        want = 0.5 * (old[inner].sum(axis=0) + c0[inner].sum(axis=0) - boundary * dt / vol)
    scale = np.abs(c0[inner]).sum(axis=0)
    assert np.all(np.abs(change - want) <= 1e-13 * scale), (change, want)
    assert abs(want[0]) > 1e-8 * scale[0]  # mass does cross the walls
    o.close()


def test_mass_kept_where_walls_see_no_normal_velocity():
    """Zero wall-normal velocity in the two cell layers by each wall: the slopes of
    that velocity vanish there, the wall faces are mirror images, and one flux call
    keeps mass and energy to round-off."""
    st = small_random_box(nx=20, ny=14, nz=1, walls=(1,) * 6, seed=6, amp=0.3)
    hp = st.params
    nx, ny = hp.nx, hp.ny
    c = st.cons.reshape(ny, nx, 5).copy()
    c[:, :4, 1] = c[:, -4:, 1] = 0.0
    c[:4, :, 2] = c[-4:, :, 2] = 0.0
    cons = c.reshape(-1, 5)
    u = cons[:, 1:4] / cons[:, :1]
    gam = hp.gammafix
    p = (gam - 1.0) * (cons[:, 4] - 0.5 * cons[:, 0] * (u * u).sum(axis=1))
    o = O.Oracle(hp)
    o.set_state(cons, u, p, np.full(hp.ngrid, gam))
    o.set_ghost_cells()
    o.velocity()  # u and p of the mirrored ghosts, as the loop leaves them
    o.state()
    o.set_clock(0.0, 1e-3, 0.0, 0)
    inner = G.boundary_flags(hp.nx, hp.ny, hp.nz) == 0
    c0 = o.get_state()[0]
    o.flux(0)
    c1 = o.get_state()[0]
    for v in (0, 4):
        m0 = c0[inner, v].sum()
        assert abs(c1[inner, v].sum() - m0) <= 1e-14 * abs(m0), v
    assert not np.array_equal(c1[inner], c0[inner])
    o.close()


def test_tabulated_state_of_an_ideal_gas_table_is_the_fixed_gamma_state():
    """Tables of an ideal gas (gamma and mu constant, T = (gamma-1) eng mu / R at
    every entry): get_gamma2's interpolation in energy and between density rows
    is linear in a linear function, so the tabulated state() (state.f90:60-79,
    eos.f90:653-699) gives the fixed-gamma pressure (state.f90:49-59) to
    rounding, and gamma and mu exactly; energies beyond the table are clamped."""
    import dataclasses
    from tests.eos_tables import synthetic_table
    st = small_random_box(nx=12, ny=11, nz=10, walls=(0,) * 6, seed=7)
    hp = st.params
    gam, mu = 5.0 / 3.0, 2.3
    tab = synthetic_table()
    eng = tab["eng_table2"]
    tab["gamma_table2"] = np.full_like(eng, gam)
    tab["muc_table2"] = np.full_like(eng, mu)
    tab["tk_table2"] = (gam - 1.0) * eng * mu / hp.rgas
    rng = np.random.default_rng(12)
    ng = hp.ngrid
    rho = np.exp(rng.uniform(np.log(0.01), np.log(10.0), ng))  # across the density rows
    u = rng.uniform(-1, 1, (ng, 3))
    e_spec = np.exp(rng.uniform(np.log(0.3), np.log(5.0), ng))  # inside every row's range
    cons = np.empty((ng, 5))
    cons[:, 0] = rho
    cons[:, 1:4] = rho[:, None] * u
    cons[:, 4] = rho * e_spec + 0.5 * rho * (u * u).sum(axis=1)
    res = {}
    for h2stat in (-1, 0):
        hq = dataclasses.replace(hp, h2stat=h2stat, gammafix=gam)
        o = O.Oracle(hq)
        if h2stat >= 0:
            o.set_eos_table(tab)
        o.set_state(cons, u, np.ones(ng), np.full(ng, gam))
        o.state()
        res[h2stat] = o.get_state()[2:], o.muc_array()
        o.close()
    (p_fix, g_fix), _ = res[-1]
    (p_tab, g_tab), mu_tab = res[0]
    assert np.allclose(p_tab, p_fix, rtol=1e-13, atol=0)
    assert np.all(g_tab == gam) and np.all(mu_tab == mu)
    # an energy above every row's table is clamped to the row's last entry
    hq = dataclasses.replace(hp, h2stat=0, gammafix=gam)
    o = O.Oracle(hq)
    o.set_eos_table(tab)
    hot = cons.copy()
    hot[:, 4] = rho * 1e4 + 0.5 * rho * (u * u).sum(axis=1)
    o.set_state(hot, u, np.ones(ng), np.full(ng, gam))
    o.state()
    p_hot = o.get_state()[2]
    o.close()
    assert np.all(p_hot < (gam - 1.0) * rho * eng.max() * (1 + 1e-12))
