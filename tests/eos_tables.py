"""Synthetic tables in the layout of the reference's eos module (eos.f90:30-51),
for exercising the tabulated state() path (H2STAT >= 0) without the reference's
calc_eos_table, whose physics (hydrogen partition functions, dissociation and
ionisation) the host keeps.  The tables are physically consistent at their
points: T = (gamma - 1) eng mu / R, so p = rho T R / mu = (gamma - 1) rho eng."""
from __future__ import annotations

import numpy as np

from boxzyhydro_b200 import celldump as CD


def synthetic_table(neos: int = 40, neos_rho: int = 9, seed: int = 0) -> dict:
    """log-spaced specific energies per density row, smooth gamma and mu; code
    densities covered: about 0.0017 to 17 (the dict Hydro.set_eos_table takes)."""
    rng = np.random.default_rng(seed)
    u = CD.units()
    D = float(u[CD.UNIT_NAMES.index("density")])
    R = float(u[CD.UNIT_NAMES.index("rgas")])
    log_low, drho = -9.0, 0.5
    j = np.arange(1, neos_rho + 1)
    i = np.arange(1, neos + 1)[:, None]
    rho_table = 10.0 ** (log_low + (j - 1) * drho) / D
    deng = 0.05 + 0.002 * j
    e0 = 0.1 * (1.0 + 0.1 * j) * rng.uniform(0.9, 1.1, neos_rho)
    eng = e0[None, :] * 10.0 ** ((i - 1) * deng[None, :])
    gam = 1.35 + 0.25 * np.sin(0.2 * i + j[None, :])
    muc = 2.3 - 0.5 * i / neos + 0.01 * j[None, :]
    tk = (gam - 1.0) * eng * muc / R
    return dict(neos=neos, neos_rho=neos_rho, log_rho_eos_low=log_low, drho_eos=drho,
                density_unit=D, tk_bgrnd=1e-6, eng_table2=eng, gamma_table2=gam,
                muc_table2=muc, tk_table2=tk, rho_table=rho_table, deng_eos_array=deng)


__all__ = ["synthetic_table"]
