"""Exact solution of the 1-D Riemann problem for an ideal gas.

The reference checks its Sod run against the exact solution it ships as
analysis/sod.ana (gamma=1.4, t=0.4, diaphragm at 0, x in [-1,1]).  This module
computes that solution for any gamma and pair of states (the iterative
pressure solver and sampling of Toro, "Riemann Solvers and Numerical Methods
for Fluid Dynamics", ch. 4), so every Sod-like and batched Riemann box can be
compared with the exact answer.
"""
from __future__ import annotations

import math

import numpy as np


def _f_and_df(p, rho_k, p_k, c_k, g):
    if p > p_k:  # shock
        a = 2.0 / ((g + 1.0) * rho_k)
        b = (g - 1.0) / (g + 1.0) * p_k
        sq = math.sqrt(a / (p + b))
        f = (p - p_k) * sq
        df = sq * (1.0 - 0.5 * (p - p_k) / (b + p))
    else:        # rarefaction
        pr = p / p_k
        f = 2.0 * c_k / (g - 1.0) * (pr ** ((g - 1.0) / (2.0 * g)) - 1.0)
        df = 1.0 / (rho_k * c_k) * pr ** (-(g + 1.0) / (2.0 * g))
    return f, df


def star_state(rl, ul, pl, rr, ur, pr, g, tol=1e-14, maxit=200):
    """(p*, u*) of the Riemann problem; raises if a vacuum forms."""
    cl = math.sqrt(g * pl / rl)
    cr = math.sqrt(g * pr / rr)
    if 2.0 * (cl + cr) / (g - 1.0) <= ur - ul:
        raise ValueError("vacuum is generated")
    # two-rarefaction guess, then Newton iterations
    z = (g - 1.0) / (2.0 * g)
    p = ((cl + cr - 0.5 * (g - 1.0) * (ur - ul)) /
         (cl / pl ** z + cr / pr ** z)) ** (1.0 / z)
    p = max(p, 1e-12 * min(pl, pr))
    for _ in range(maxit):
        fl, dfl = _f_and_df(p, rl, pl, cl, g)
        fr, dfr = _f_and_df(p, rr, pr, cr, g)
        pn = p - (fl + fr + ur - ul) / (dfl + dfr)
        if pn <= 0:
            pn = 0.5 * p
        if abs(pn - p) <= tol * 0.5 * (pn + p):
            p = pn
            break
        p = pn
    fl, _ = _f_and_df(p, rl, pl, cl, g)
    fr, _ = _f_and_df(p, rr, pr, cr, g)
    u = 0.5 * (ul + ur) + 0.5 * (fr - fl)
    return p, u


def sample(xi, rl, ul, pl, rr, ur, pr, g):
    """(rho, u, p) at similarity coordinates xi = (x - x0)/t (array)."""
    xi = np.asarray(xi, dtype=np.float64)
    ps, us = star_state(rl, ul, pl, rr, ur, pr, g)
    cl = math.sqrt(g * pl / rl)
    cr = math.sqrt(g * pr / rr)
    gm = (g - 1.0) / (g + 1.0)
    rho = np.empty_like(xi)
    u = np.empty_like(xi)
    p = np.empty_like(xi)
    left = xi <= us
    # ---- left of contact
    if ps > pl:  # left shock
        rsl = rl * ((ps / pl + gm) / (ps / pl * gm + 1.0))
        sl = ul - cl * math.sqrt((g + 1.0) / (2.0 * g) * ps / pl + (g - 1.0) / (2.0 * g))
        m = left & (xi < sl)
        rho[m], u[m], p[m] = rl, ul, pl
        m = left & (xi >= sl)
        rho[m], u[m], p[m] = rsl, us, ps
    else:        # left rarefaction
        rsl = rl * (ps / pl) ** (1.0 / g)
        csl = cl * (ps / pl) ** ((g - 1.0) / (2.0 * g))
        shl, stl = ul - cl, us - csl
        m = left & (xi < shl)
        rho[m], u[m], p[m] = rl, ul, pl
        m = left & (xi >= shl) & (xi < stl)
        c = 2.0 / (g + 1.0) * (cl + (g - 1.0) / 2.0 * (ul - xi[m]))
        u[m] = 2.0 / (g + 1.0) * (cl + (g - 1.0) / 2.0 * ul + xi[m])
        rho[m] = rl * (c / cl) ** (2.0 / (g - 1.0))
        p[m] = pl * (c / cl) ** (2.0 * g / (g - 1.0))
        m = left & (xi >= stl)
        rho[m], u[m], p[m] = rsl, us, ps
    right = ~left
    if ps > pr:  # right shock
        rsr = rr * ((ps / pr + gm) / (ps / pr * gm + 1.0))
        sr = ur + cr * math.sqrt((g + 1.0) / (2.0 * g) * ps / pr + (g - 1.0) / (2.0 * g))
        m = right & (xi > sr)
        rho[m], u[m], p[m] = rr, ur, pr
        m = right & (xi <= sr)
        rho[m], u[m], p[m] = rsr, us, ps
    else:        # right rarefaction
        rsr = rr * (ps / pr) ** (1.0 / g)
        csr = cr * (ps / pr) ** ((g - 1.0) / (2.0 * g))
        shr, str_ = ur + cr, us + csr
        m = right & (xi > shr)
        rho[m], u[m], p[m] = rr, ur, pr
        m = right & (xi <= shr) & (xi > str_)
        c = 2.0 / (g + 1.0) * (cr - (g - 1.0) / 2.0 * (ur - xi[m]))
        u[m] = 2.0 / (g + 1.0) * (-cr + (g - 1.0) / 2.0 * ur + xi[m])
        rho[m] = rr * (c / cr) ** (2.0 / (g - 1.0))
        p[m] = pr * (c / cr) ** (2.0 * g / (g - 1.0))
        m = right & (xi <= str_)
        rho[m], u[m], p[m] = rsr, us, ps
    return rho, u, p


def sod_profile(x, t, x0=0.0, g=1.4, left=(1.0, 0.0, 1.0), right=(0.125, 0.0, 0.1)):
    """Exact Sod profile (rho, u, p) at positions x and time t > 0."""
    xi = (np.asarray(x, dtype=np.float64) - x0) / t
    return sample(xi, left[0], left[1], left[2], right[0], right[1], right[2], g)
