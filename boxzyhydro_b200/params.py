"""Run parameters of the hydro step, mirroring the reference's namelists.

The reference reads six namelist groups from the file named on its command
line (input.f90:7-36) into module variables whose defaults live in
parameters.f90:26-96.  `HydroParams` holds the fields the hydrodynamic step
reads, with the same names and defaults; `read_namelist` parses an `in.nml`
(the same text format, so the reference's ICFILES work unchanged).
"""
from __future__ import annotations

import dataclasses
import re
from typing import Dict, List, Tuple

PI = 3.1415926535897931          # parameters.f90:11
RGAS_CGS = 8.254e7               # parameters.f90:9


def rgas_code_units() -> float:
    """scale%rgas of get_units (units.f90:10-17), same operation order."""
    length = 1.496e13
    time = (3600.0 * 365.25 * 24.0) / (2.0 * PI)
    vel = length / time
    kelvin = 1.0
    return RGAS_CGS / ((vel * vel) / kelvin)


def muc_from_abundances(xabun=0.73, yabun=0.27, zabun=0.0, mu_z=16.78) -> float:
    """Mean molecular weight muc of calc_eos_table (eos.f90:144)."""
    return 1.0 / (xabun * 0.5 + yabun * 0.25 + zabun / mu_z)


@dataclasses.dataclass
class HydroParams:
    """Fields of grid_params, hydro and eos_input used by the hydro step."""
    nx: int = 50
    ny: int = 50
    nz: int = 50
    dx: float = 0.25
    dy: float = 0.25
    dz: float = 0.25
    yoffset: float = 0.0
    fluxangmom: bool = False
    no_outflow_xl: bool = True
    no_outflow_xr: bool = True
    no_outflow_yl: bool = True
    no_outflow_yr: bool = True
    no_outflow_zl: bool = True
    no_outflow_zr: bool = True
    small_rho: float = 1e-10
    small_eps: float = 1e-40
    vlimit: float = 1e1
    starttime: float = 0.0
    endtime: float = 0.0
    dtout: float = 10.0
    cfl: float = 0.1
    irestart: int = 0
    avmagx: float = 0.0
    avmagy: float = 0.0
    avmagz: float = 0.0
    gammafix: float = 1.66666666667
    h2stat: int = 0
    xabun: float = 0.73
    yabun: float = 0.27
    zabun: float = 0.0
    mu_z: float = 16.78
    tk_bgrnd: float = 1e-6
    write_ascii: bool = True

    @property
    def muc(self) -> float:
        return muc_from_abundances(self.xabun, self.yabun, self.zabun, self.mu_z)

    @property
    def rgas(self) -> float:
        return rgas_code_units()

    @property
    def no_outflow(self) -> Tuple[bool, bool, bool, bool, bool, bool]:
        """Wall flags as the grid sees them: z walls are off when nz<6
        (init_grid.f90:76-79)."""
        zl = self.no_outflow_zl and self.nz >= 6
        zr = self.no_outflow_zr and self.nz >= 6
        return (self.no_outflow_xl, self.no_outflow_xr, self.no_outflow_yl,
                self.no_outflow_yr, zl, zr)

    @property
    def ngrid(self) -> int:
        return self.nx * self.ny * self.nz

    def n_active(self) -> int:
        ax = max(self.nx - 4, 0)
        ay = max(self.ny - 4, 0)
        az = self.nz if self.nz < 6 else max(self.nz - 4, 0)
        return ax * ay * az

    def validate(self) -> None:
        if self.h2stat < -1:
            raise ValueError("H2STAT must be -1 (fixed gamma) or >= 0 (tabulated EOS)")
        if self.nx < 5 or self.ny < 5:
            raise ValueError("nx and ny must be >= 5 (two ghost layers per side)")
        if self.nz >= 6 and self.nz < 5:
            raise ValueError("bad nz")
        if not (self.dx > 0 and self.dy > 0 and self.dz > 0):
            raise ValueError("cell sizes must be positive")
        if not (self.gammafix > 1.0):
            raise ValueError("gammafix must exceed 1")


_FIELD_ALIASES: Dict[str, str] = {"h2stat": "h2stat"}


def _parse_value(tok: str):
    t = tok.strip().strip(",")
    tl = t.lower()
    if tl in (".true.", "t", ".t.", "true"):
        return True
    if tl in (".false.", "f", ".f.", "false"):
        return False
    if (t.startswith("'") and t.endswith("'")) or (t.startswith('"') and t.endswith('"')):
        return t[1:-1]
    num = tl.replace("d", "e")
    try:
        if re.fullmatch(r"[+-]?\d+", num):
            return int(num)
        return float(num)
    except ValueError:
        return t


def parse_namelist_text(text: str) -> Dict[str, Dict[str, object]]:
    """Parse Fortran namelist groups: {'grid_params': {'nx': 8, ...}, ...}."""
    groups: Dict[str, Dict[str, object]] = {}
    cur = None
    for raw in text.splitlines():
        line = raw.split("!")[0].strip()
        if not line:
            continue
        if line.startswith("&"):
            cur = line[1:].strip().lower()
            groups.setdefault(cur, {})
            continue
        if line.startswith("/"):
            cur = None
            continue
        if cur is None:
            continue
        for part in re.split(r",(?=\s*[A-Za-z_]\w*\s*=)", line):
            if "=" not in part:
                continue
            k, v = part.split("=", 1)
            groups[cur][k.strip().lower()] = _parse_value(v)
    return groups


def read_namelist(path: str) -> HydroParams:
    """Read an in.nml the way read_params does (input.f90:21-36)."""
    with open(path) as f:
        groups = parse_namelist_text(f.read())
    return params_from_groups(groups)


def params_from_groups(groups: Dict[str, Dict[str, object]]) -> HydroParams:
    hp = HydroParams()
    fields = {f.name for f in dataclasses.fields(HydroParams)}
    for g in ("io_control", "grid_params", "hydro", "eos_input"):
        for k, v in groups.get(g, {}).items():
            name = _FIELD_ALIASES.get(k, k)
            if name in fields:
                cur = getattr(hp, name)
                if isinstance(cur, bool):
                    v = bool(v)
                elif isinstance(cur, int) and not isinstance(cur, bool):
                    v = int(v)
                elif isinstance(cur, float):
                    v = float(v)
                setattr(hp, name, v)
    return hp
