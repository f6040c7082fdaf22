"""Host-side logic that needs no GPU: the C ABI library loads and exports every
symbol of include/boxzy_gpu.h, its ghost-fill plans reproduce the oracle's
set_ghost_cells sweeps exactly, namelist parsing, and grid geometry."""
import ctypes
import os
import re

import numpy as np
import pytest

import oracle as O
from boxzyhydro_b200 import _lib
from boxzyhydro_b200 import grid as G
from boxzyhydro_b200.hydro import apply_ghost_plan, ghost_plan
from boxzyhydro_b200.params import (HydroParams, muc_from_abundances, parse_namelist_text,
                                    params_from_groups, rgas_code_units)

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    names = []
    for hdr in ("boxzy_gpu.h", "boxzy_diag.h"):
        text = open(os.path.join(ROOT, "include", hdr)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(bx_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    L = ctypes.CDLL(_lib.LIB_PATH)
    names = header_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_library_version_string():
    assert b"sm_100a" in _lib.lib().bx_version()


def test_bx_params_layout_matches_header():
    # 4 int32, 10 doubles, 6+2 int32 -> 16 + 80 + 32 bytes, no padding
    assert ctypes.sizeof(_lib.BxParams) == 136
    assert _lib.BxParams.no_outflow.offset == 96 and _lib.BxParams.flags.offset == 124


WALLS = [(1, 1, 1, 1, 1, 1), (0, 0, 0, 0, 0, 0), (1, 0, 1, 0, 1, 0), (0, 1, 1, 0, 0, 1)]
DIMS = [(8, 200, 1), (12, 10, 8), (9, 9, 6), (10, 11, 7), (516, 8, 4), (13, 9, 3), (11, 7, 12)]


@pytest.mark.parametrize("dims", DIMS)
@pytest.mark.parametrize("walls", WALLS)
def test_ghost_plan_reproduces_sequential_fill(dims, walls):
    hp = HydroParams(nx=dims[0], ny=dims[1], nz=dims[2], dx=0.1, dy=0.1, dz=0.1, h2stat=-1,
                     gammafix=1.4, no_outflow_xl=bool(walls[0]), no_outflow_xr=bool(walls[1]),
                     no_outflow_yl=bool(walls[2]), no_outflow_yr=bool(walls[3]),
                     no_outflow_zl=bool(walls[4]), no_outflow_zr=bool(walls[5]))
    rng = np.random.default_rng(hash(dims) % 1000)
    c = rng.standard_normal((hp.ngrid, 5))
    o = O.Oracle(hp)
    o.set_state(c, np.zeros((hp.ngrid, 3)), np.ones(hp.ngrid), np.full(hp.ngrid, 1.4))
    o.set_ghost_cells()
    c1 = o.get_state()[0]
    o.set_ghost_cells()
    c2 = o.get_state()[0]
    pl = ghost_plan(hp)
    assert np.array_equal(apply_ghost_plan(c, pl["src1"], pl["sgn1"], pl["dst"]), c1)
    assert np.array_equal(apply_ghost_plan(c, pl["src2"], pl["sgn2"], pl["dst"]), c2)
    b = G.boundary_flags(*dims)
    assert np.array_equal(np.sort(pl["dst"]), np.nonzero(b)[0])
    o.close()


def test_fused_eligibility():
    def ok(dims, walls):
        hp = HydroParams(nx=dims[0], ny=dims[1], nz=dims[2], dx=0.1, dy=0.1, dz=0.1,
                         h2stat=-1, gammafix=1.4,
                         no_outflow_xl=bool(walls[0]), no_outflow_xr=bool(walls[1]),
                         no_outflow_yl=bool(walls[2]), no_outflow_yr=bool(walls[3]),
                         no_outflow_zl=bool(walls[4]), no_outflow_zr=bool(walls[5]))
        return ghost_plan(hp)["fused_ok"]
    assert ok((260, 260, 260), (0,) * 6)          # outflow box
    assert ok((516, 8, 4), (1,) * 6)              # reflective tube, nz<6
    assert not ok((20, 20, 20), (1,) * 6)         # reflective 3-D: corner ghosts lag
    assert not ghost_plan(HydroParams(nx=20, ny=20, nz=20, h2stat=-1, gammafix=1.4,
                                      no_outflow_xl=False, no_outflow_xr=False,
                                      no_outflow_yl=False, no_outflow_yr=False,
                                      no_outflow_zl=False, no_outflow_zr=False),
                          phase_only=True)["fused_ok"]


def test_grid_flags_match_oracle():
    for dims in DIMS:
        hp = HydroParams(nx=dims[0], ny=dims[1], nz=dims[2], h2stat=-1, gammafix=1.4)
        o = O.Oracle(hp)
        b, nb = o.grid_info()
        assert np.array_equal(b, G.boundary_flags(*dims))
        o.close()


NML = """
&io_control
write_ascii=.false.
/
&grid_params
dx=0.01d0, dy=0.01d0
dz=0.01d0
nx=8
ny=200
nz=1
fluxangmom=.false.
no_outflow_xl=.true.
no_outflow_zr=.false.
/
&hydro
endtime=0.4
small_rho=1d-12
small_eps=1d-40
vlimit=10.
/
&eos_input
H2STAT=-1
gammafix=1.4d0
/
"""


def test_namelist_parsing():
    hp = params_from_groups(parse_namelist_text(NML))
    assert (hp.nx, hp.ny, hp.nz) == (8, 200, 1)
    assert hp.dx == 0.01 and hp.dy == 0.01 and hp.dz == 0.01
    assert hp.small_rho == 1e-12 and hp.small_eps == 1e-40 and hp.vlimit == 10.0
    assert hp.h2stat == -1 and hp.gammafix == 1.4 and hp.endtime == 0.4
    assert hp.no_outflow_xl is True and hp.no_outflow_zr is False
    assert hp.cfl == 0.1  # parameters.f90:74 default
    hp.validate()


def test_units_and_muc_match_oracle():
    assert rgas_code_units() == O.rgas_code_units()
    assert muc_from_abundances() == O.muc()
    assert abs(muc_from_abundances() - 1.0 / 0.4325) < 1e-15


# C types of the headers -> (kind, size) of the value passed
_C_SCALARS = {"int": ("i", 4), "int32_t": ("i", 4), "int64_t": ("i", 8), "uint32_t": ("u", 4),
              "uint8_t": ("u", 1), "unsigned long long": ("u", 8), "double": ("f", 8),
              "char": ("i", 1), "void": ("v", 0)}
_C_STRUCTS = {"bx_params": 136, "bx_eos_table": None}  # sizes checked elsewhere
_C_OPAQUE = ("bx_handle", "bx_batch", "bx_adj")


def header_prototypes():
    """(name, return type, [(base type, pointer depth)]) of every prototype."""
    out = []
    for hdr in ("boxzy_gpu.h", "boxzy_diag.h"):
        text = open(os.path.join(ROOT, "include", hdr)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"^\s*#.*$", "", text, flags=re.M)
        for m in re.finditer(r"([\w\s]+?)\s*(\**)\s*(bx_\w+)\s*\(([^)]*)\)\s*;", text):
            ret = (" ".join(m.group(1).replace("const", " ").split()), len(m.group(2)))
            params = []
            for p in m.group(4).split(","):
                p = " ".join(p.replace("const", " ").split())
                if p in ("", "void"):
                    continue
                depth = p.count("*")
                toks = p.replace("*", " ").split()
                params.append((" ".join(toks[:-1]), depth))
            out.append((m.group(3), ret, params))
    return out


def _ctype_matches(c_type, ct):
    base, depth = c_type
    if depth == 0:
        kind, size = _C_SCALARS[base]
        if kind == "f":
            return ct in (ctypes.c_double,)
        return (ct is not None and issubclass(ct, ctypes._SimpleCData) and ct not in
                (ctypes.c_double, ctypes.c_float, ctypes.c_void_p, ctypes.c_char_p) and
                ctypes.sizeof(ct) == size)
    if base in _C_OPAQUE and depth == 1:
        return ct is ctypes.c_void_p
    if ct is ctypes.c_void_p:
        return True  # any pointer may be passed as an address
    if base == "char" and depth == 1:
        return ct is ctypes.c_char_p
    if not (isinstance(ct, type) and issubclass(ct, ctypes._Pointer)):
        return False
    inner = ct._type_
    if depth > 1 or base in _C_OPAQUE:
        return inner is ctypes.c_void_p if depth == 2 or base in _C_OPAQUE else False
    if base in _C_STRUCTS:
        return inner.__name__.lower().replace("_", "") == base.replace("_", "")
    return _ctype_matches((base, 0), inner)


def test_ctypes_signatures_match_the_header():
    """Every prototype of include/*.h has argtypes and restype in the Python layer
    whose widths and kinds match the C declaration (an int32/int64 slip would
    pass garbage through the ABI without an error)."""
    L = _lib.lib()
    protos = header_prototypes()
    assert len(protos) == len(header_functions())
    bad = []
    for name, ret, params in protos:
        f = getattr(L, name)
        if f.argtypes is None:
            bad.append(f"{name}: no argtypes")
            continue
        if len(f.argtypes) != len(params):
            bad.append(f"{name}: {len(f.argtypes)} argtypes for {len(params)} parameters")
            continue
        for k, (p, ct) in enumerate(zip(params, f.argtypes)):
            if not _ctype_matches(p, ct):
                bad.append(f"{name} arg {k}: C {p} vs ctypes {ct}")
        want_ret = ctypes.c_char_p if ret == ("char", 1) else ctypes.c_int
        if f.restype is not want_ret:
            bad.append(f"{name}: restype {f.restype} for C {ret}")
    assert not bad, bad
