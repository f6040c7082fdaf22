"""The synthetic workloads against their specification (the bench configs): the
turbulent box (lognormal density with sigma_ln = 0.5 from a unit-variance k^-2
Gaussian field, p = 1, solenoidal k^-2 velocity at RMS Mach 1 against
sqrt(gamma p / <rho>), gamma = 5/3 given to full precision, outflow walls, CFL
0.4), the x-split Sod tube of 512x4x4 cells, the Sod state with a 5 % Gaussian
density blob of the adjoint runs, and the seeded Riemann ensemble (sides from
{32, 48, 64, 96}, rho and p log-uniform in [0.1, 10], v in [-1, 1], gamma 1.4 or
5/3, random split axis)."""
import numpy as np
import pytest

from boxzyhydro_b200 import grid as G
from boxzyhydro_b200 import ic


def interior(st, q):
    hp = st.params
    zs, ys, xs = G.active_slices(hp.nx, hp.ny, hp.nz)
    return q.reshape(hp.nz, hp.ny, hp.nx)[zs, ys, xs]


def shell_slope(field):
    """Least-squares slope of log shell-averaged power against log k (k from 2 to
    a third of the grid, where shells hold many modes)."""
    n = field.shape[0]
    p = np.abs(np.fft.fftn(field)) ** 2
    k1 = np.fft.fftfreq(n) * n
    kz, ky, kx = np.meshgrid(k1, k1, k1, indexing="ij")
    k = np.sqrt(kx * kx + ky * ky + kz * kz)
    ks = np.arange(2, n // 3)
    pw = np.array([p[(k >= s - 0.5) & (k < s + 0.5)].mean() for s in ks])
    return np.polyfit(np.log(ks), np.log(pw), 1)[0]


@pytest.fixture(scope="module")
def turb():
    return ic.turbulent_box(n=48, seed=1234)


def test_turbulent_box_parameters(turb):
    hp = turb.params
    assert hp.gammafix == 1.6666666666666667  # not the default 1.66666666667
    assert (hp.nx, hp.ny, hp.nz) == (52, 52, 52) and hp.dx == hp.dy == hp.dz == 1.0 / 48
    assert hp.cfl == 0.4 and hp.h2stat == -1
    assert not any([hp.no_outflow_xl, hp.no_outflow_xr, hp.no_outflow_yl, hp.no_outflow_yr,
                    hp.no_outflow_zl, hp.no_outflow_zr])


def test_turbulent_density_is_lognormal_with_sigma_half(turb):
    rho = interior(turb, turb.cons[:, 0])
    lr = np.log(rho)
    assert abs(lr.std() - 0.5) < 1e-12
    assert abs(lr.mean() + 0.125) < 1e-12  # -sigma^2/2
    assert -2.4 < shell_slope(lr) < -1.6   # P(k) ~ k^-2


def test_turbulent_velocity_is_solenoidal_at_mach_one(turb):
    hp = turb.params
    u = [interior(turb, turb.u[:, d]) for d in range(3)]
    rho = interior(turb, turb.cons[:, 0])
    assert np.all(interior(turb, turb.p) == 1.0)
    vrms = np.sqrt(np.mean(u[0] ** 2 + u[1] ** 2 + u[2] ** 2))
    cs = np.sqrt(hp.gammafix / rho.mean())
    assert abs(vrms / cs - 1.0) < 1e-12
    n = rho.shape[0]
    k1 = np.fft.fftfreq(n) * n
    kz, ky, kx = np.meshgrid(k1, k1, k1, indexing="ij")
    uh = [np.fft.fftn(c) for c in u]  # (z, y, x) axes: u[0] is vx along the last axis
    div = kx * uh[0] + ky * uh[1] + kz * uh[2]
    k = np.sqrt(kx * kx + ky * ky + kz * kz)
    scale = np.sqrt(sum(np.abs(c) ** 2 for c in uh)) * k
    assert np.abs(div).max() < 1e-12 * scale.max()
    assert -2.4 < shell_slope(u[0]) < -1.6


def test_turbulent_ghosts_copy_the_nearest_interior_cell(turb):
    hp = turb.params
    c = turb.cons.reshape(hp.nz, hp.ny, hp.nx, 5)
    assert np.array_equal(c[:, :, 0], c[:, :, 2]) and np.array_equal(c[:, :, 1], c[:, :, 2])
    assert np.array_equal(c[:, -1], c[:, -3]) and np.array_equal(c[0], c[2])


def test_sod_tube_512x4x4():
    st = ic.sod_x()
    hp = st.params
    assert (hp.nx, hp.ny, hp.nz) == (516, 8, 4) and hp.dx == 1.0 / 512
    assert hp.gammafix == 1.4 and hp.cfl == 0.1 and hp.endtime == 0.2
    rho = st.cons.reshape(hp.nz, hp.ny, hp.nx, 5)[:, 2:-2, 2:-2, 0]
    assert np.all(rho[..., :256] == 1.0) and np.all(rho[..., 256:] == 0.125)
    p = st.p.reshape(hp.nz, hp.ny, hp.nx)[:, 2:-2, 2:-2]
    assert np.all(p[..., :256] == 1.0) and np.all(p[..., 256:] == 0.1)
    assert np.all(st.u == 0.0)


def test_adjoint_state_has_a_five_percent_blob():
    a = ic.sod_blob_box(n=32, seed=4)
    b = ic.sod_blob_box(n=32, seed=4, blob=False)
    ra, rb = interior(a, a.cons[:, 0]), interior(b, b.cons[:, 0])
    rel = ra / rb - 1.0
    assert 0.045 < rel.max() <= 0.05 and rel.min() >= 0.0
    assert np.array_equal(interior(a, a.p), interior(b, b.p))
    assert a.params.gammafix == 1.6666666666666667


def test_riemann_ensemble_draws():
    spec = ic.riemann_ensemble_spec(4096, seed=2024)
    assert spec == ic.riemann_ensemble_spec(4096, seed=2024)  # seeded
    assert len(spec) == 4096
    sides = np.array([s["side"] for s in spec])
    assert set(sides) == {32, 48, 64, 96}
    mean_cells = (sides.astype(float) ** 3).mean()
    assert abs(mean_cells / 322560.0 - 1.0) < 0.05  # E[s^3] over the four sides
    assert {s["gamma"] for s in spec} == {1.4, 1.6666666666666667}
    assert {s["axis"] for s in spec} == {0, 1, 2}
    for s in spec:
        for rho, v, p in (s["left"], s["right"]):
            assert 0.1 <= rho <= 10.0 and 0.1 <= p <= 10.0 and -1.0 <= v <= 1.0
