"""Tangent-linear model of the fused hydro step (numpy, value + tangent pairs).

TEST INFRASTRUCTURE ONLY: the checker for the GPU adjoint (bx_adj_backward).
It advances the same map the fused stage kernels compute (and bx_adj
differentiates) -- sources, stage 0, stage 1 of the reference step
(main.f90:289-515, flux.f90, state.f90, velocity.f90, source.f90) with the face
ghosts read through the donor rule -- carrying a directional derivative along
with every value, with the dt sequence given and every max/min/limiter branch
taken where the values put it.  Values are evaluated in the reference's order,
so they reproduce the GPU forward; the tangent is the exact (up to rounding)
Jacobian-vector product, which makes the dot-product test
<lamT, J v> = <J^T lamT, v> hold to rounding error.
"""
from __future__ import annotations

import numpy as np

HALF = 0.5
THETA = 1.25


class D:
    """A value array with its tangent."""
    __slots__ = ("v", "t")

    def __init__(self, v, t):
        self.v = v
        self.t = t

    def __add__(self, o):
        if isinstance(o, D):
            return D(self.v + o.v, self.t + o.t)
        return D(self.v + o, self.t)

    def __radd__(self, o):
        return D(o + self.v, self.t)

    def __sub__(self, o):
        if isinstance(o, D):
            return D(self.v - o.v, self.t - o.t)
        return D(self.v - o, self.t)

    def __rsub__(self, o):
        return D(o - self.v, -self.t)

    def __mul__(self, o):
        if isinstance(o, D):
            return D(self.v * o.v, self.t * o.v + self.v * o.t)
        return D(self.v * o, self.t * o)

    def __rmul__(self, o):
        return D(o * self.v, o * self.t)

    def __truediv__(self, o):
        if isinstance(o, D):
            q = self.v / o.v
            return D(q, (self.t - q * o.t) / o.v)
        return D(self.v / o, self.t / o)

    def __neg__(self):
        return D(-self.v, -self.t)

    def __getitem__(self, k):
        return D(self.v[k], self.t[k])


def dsqrt(a):
    s = np.sqrt(a.v)
    with np.errstate(divide="ignore", invalid="ignore"):
        t = np.where(s > 0, a.t / (2.0 * np.where(s > 0, s, 1.0)), 0.0)
    return D(s, t)


def dabs(a):
    sg = np.where(a.v < 0, -1.0, 1.0)
    return D(np.abs(a.v), sg * a.t)


def pick(cond, a, b):
    """cond ? a : b elementwise (a, b dual or scalar)."""
    av, at = (a.v, a.t) if isinstance(a, D) else (a, 0.0)
    bv, bt = (b.v, b.t) if isinstance(b, D) else (b, 0.0)
    return D(np.where(cond, av, bv), np.where(cond, at, bt))


def maxd(a, b):
    """max(a, b) taking a only where a > b (the forward's branch rule)."""
    av = a.v if isinstance(a, D) else a
    bv = b.v if isinstance(b, D) else b
    return pick(av > bv, a, b)


def mind(a, b):
    av = a.v if isinstance(a, D) else a
    bv = b.v if isinstance(b, D) else b
    return pick(av < bv, a, b)


def slope(c0, c1, c2):
    """genminmod slope (utils.f90:696-741) and its tangent (selected argument)."""
    d1, d2, d3 = c1 - c0, c2 - c0, c2 - c1
    x1, x2, x3 = THETA * d1, HALF * d2, THETA * d3
    a1, a2, a3 = np.abs(x1.v), np.abs(x2.v), np.abs(x3.v)
    pos = (d1.v > 0) & (d3.v > 0)
    neg = (d1.v < 0) & (d3.v < 0)
    m23 = np.fmin(a2, a3)
    s1 = a1 <= m23
    s2 = (~s1) & (a2 <= a3)
    val = pick(s1, x1, pick(s2, x2, x3))
    on = pos | neg
    return D(np.where(on, val.v, 0.0), np.where(on, val.t, 0.0))


class Grid:
    def __init__(self, hp):
        self.hp = hp
        self.nx, self.ny, self.nz = hp.nx, hp.ny, hp.nz
        self.threed = hp.nz >= 6
        self.a0 = (2, 2, 2 if self.threed else 0)
        self.a1 = (hp.nx - 2, hp.ny - 2, hp.nz - 2 if self.threed else hp.nz)
        w = hp.no_outflow
        self.walls = w
        self.maps = []
        for ax, n in enumerate((hp.nx, hp.ny, hp.nz)):
            idx = np.arange(n)
            flip = np.zeros(n, bool)
            if ax < 2 or self.threed:
                a0, a1 = self.a0[ax], self.a1[ax]
                wl, wr = w[2 * ax], w[2 * ax + 1]
                for c in range(n):
                    if c < a0:
                        idx[c], flip[c] = (2 * a0 - 1 - c, True) if wl else (a0, False)
                    elif c >= a1:
                        idx[c], flip[c] = (2 * a1 - 1 - c, True) if wr else (a1 - 1, False)
            self.maps.append((idx, flip))
        self.interior = np.zeros((self.nz, self.ny, self.nx), bool)
        self.interior[self.a0[2]:self.a1[2], self.a0[1]:self.a1[1], self.a0[0]:self.a1[0]] = True
        self.dx, self.dy, self.dz = hp.dx, hp.dy, hp.dz
        self.pow2 = all(_is_pow2(v) for v in (hp.dx, hp.dy, hp.dz))

    def fill(self, c):
        """Full grid from the interior through the donor rule (5 dual fields)."""
        (ix, fx), (iy, fy), (iz, fz) = self.maps
        out = []
        for q in range(5):
            v = c[q].v[np.ix_(iz, iy, ix)]
            t = c[q].t[np.ix_(iz, iy, ix)]
            sg = None
            if q == 1:
                sg = np.where(fx, -1.0, 1.0)[None, None, :]
            elif q == 2:
                sg = np.where(fy, -1.0, 1.0)[None, :, None]
            elif q == 3:
                sg = np.where(fz, -1.0, 1.0)[:, None, None]
            if sg is not None:
                v = v * sg
                t = t * sg
            out.append(D(v, t))
        return out


def _is_pow2(x):
    m, e = np.frexp(x)
    return m == 0.5


def src(c, nsrc, eps):
    d, m1, m2, m3, E = c
    for _ in range(nsrc):
        ek = (HALF * (m1 * m1 + m2 * m2 + m3 * m3)) / d
        E = maxd(E - ek, eps) + ek
    return [d, m1, m2, m3, E]


def prims(G, stage, A, B):
    hp = G.hp
    gm1 = hp.gammafix - 1.0
    d = A[0]
    u = [A[1] / d, A[2] / d, A[3] / d]
    e = maxd(A[4] - (HALF * d) * (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]), hp.small_eps)
    if stage == 0:
        p = e * gm1
    else:
        s = [B[1] / B[0], B[2] / B[0], B[3] / B[0]]
        p = maxd(A[4] - (d * HALF) * (s[0] * s[0] + s[1] * s[1] + s[2] * s[2]), hp.small_eps) * gm1
    c = dsqrt((p * hp.gammafix) / d)
    return [d, u[0], u[1], u[2], p, e], c


def _shift(a, ax, k):
    """a shifted by k cells along axis ax (numpy axis 2-ax), edges replicated."""
    return D(np.roll(a.v, -k, axis=2 - ax), np.roll(a.t, -k, axis=2 - ax))


def states(G, Q, c, ax, dt):
    """minus/plus face states along axis ax for every cell (ghosts: cell values)."""
    ds = (G.dx, G.dy, G.dz)[ax]
    ud = Q[1 + ax]
    lp = maxd(ud + c, 0.0) * dt
    lm = mind(ud - c, 0.0) * dt
    if G.pow2:
        lp = lp * (1.0 / ds)
        lm = lm * (1.0 / ds)
    else:
        lp = lp / ds
        lm = lm / ds
    hm = HALF * (-1.0 - lm)
    hp_ = HALF * (1.0 - lp)
    mi, pl = [], []
    for q in range(6):
        s = slope(_shift(Q[q], ax, -1), Q[q], _shift(Q[q], ax, 1))
        s = D(np.where(G.interior, s.v, 0.0), np.where(G.interior, s.t, 0.0))
        mi.append(Q[q] + hm * s)
        pl.append(Q[q] + hp_ * s)
    return mi, pl


def hll(L, R, gam, ax):
    dl, u1l, u2l, u3l, pl, el = L
    dr, u1r, u2r, u3r, pr, er = R
    ul, ur = [u1l, u2l, u3l], [u1r, u2r, u3r]
    vl, vr = ul[ax], ur[ax]
    sl = [dl, dl * u1l, dl * u2l, dl * u3l, el + (HALF * dl) * (u1l * u1l + u2l * u2l + u3l * u3l)]
    sr = [dr, dr * u1r, dr * u2r, dr * u3r, er + (HALF * dr) * (u1r * u1r + u2r * u2r + u3r * u3r)]
    fl = [sl[0] * vl] + [(pl + sl[1 + j] * vl) if j == ax else sl[1 + j] * vl for j in range(3)]
    fr = [sr[0] * vr] + [(pr + sr[1 + j] * vr) if j == ax else sr[1 + j] * vr for j in range(3)]
    fl.append((sl[4] + pl) * vl)
    fr.append((sr[4] + pr) * vr)
    cr = dsqrt((gam * pr) / dr)
    cl = dsqrt((gam * pl) / dl)
    ap = maxd(vl + cl, maxd(vr + cr, 0.0))
    am = maxd(-(vl - cl), maxd(-(vr - cr), 0.0))
    apam = ap * am
    den = ap + am
    return [(ap * fl[k] + am * fr[k] - apam * (sr[k] - sl[k])) / den for k in range(5)]


def flux_update(G, Q, c, dt):
    """L(C) on interior cells: -(dt/vol) sum_d A_d (F_{i+1/2} - F_{i-1/2})."""
    hp = G.hp
    nax = 3 if G.threed else 2
    areas = (hp.dy * hp.dz, hp.dx * hp.dz, hp.dy * hp.dx)
    terms = []
    for ax in range(nax):
        mi, pl = states(G, Q, c, ax, dt)
        Lst = [_shift(pl[q], ax, -1) for q in range(6)]  # plus state of the low neighbour
        F = hll(Lst, mi, hp.gammafix, ax)                 # flux through the low face
        dF = [_shift(F[k], ax, 1) - F[k] for k in range(5)]
        terms.append([areas[ax] * dF[k] for k in range(5)])
    out = []
    vol = hp.dx * hp.dy * hp.dz
    for k in range(5):
        s = terms[0][k] + terms[1][k]
        if nax == 3:
            s = s + terms[2][k]
        x = (-s) * dt
        out.append(x * (1.0 / vol) if G.pow2 else x / vol)
    return out


def step(G, X, nsrc, dt):
    """One step of the fused map: X (interior meaningful) -> C2 (interior)."""
    hp = G.hp
    Xf = G.fill(X)
    C0 = src(Xf, nsrc, hp.small_eps)
    Q, c = prims(G, 0, C0, C0)
    L0 = flux_update(G, Q, c, dt)
    C1 = [C0[k] + L0[k] for k in range(5)]
    C1f = G.fill(C1)
    Q1, c1 = prims(G, 1, C1f, C0)
    L1 = flux_update(G, Q1, c1, dt)
    return [HALF * ((C0[k] + C1f[k]) + L1[k]) for k in range(5)]


def run(hp, cons0, dcons0, dts):
    """Forward run with tangents.  cons0, dcons0: (ngrid,5) reference layout.
    Returns (consT, dconsT) (ngrid,5): consT = src(C2_T) filled to the ghosts."""
    G = Grid(hp)
    shp = (hp.nz, hp.ny, hp.nx)
    X = [D(cons0[:, q].reshape(shp).copy(), dcons0[:, q].reshape(shp).copy()) for q in range(5)]
    nsrc = 1
    for dt in dts:
        X = step(G, X, nsrc, float(dt))
        nsrc = 2
    Xf = G.fill(src(X, 1, hp.small_eps))
    cons = np.stack([Xf[q].v.ravel() for q in range(5)], 1)
    dcons = np.stack([Xf[q].t.ravel() for q in range(5)], 1)
    return cons, dcons
