"""Host-side logic that needs no GPU: the C ABI library loads and exports every
symbol of include/boxzy_gpu.h, the ctypes layer and the Fortran interface module
(include/boxzy_gpu.f90) bind those prototypes with matching argument types, its
ghost-fill plans reproduce the oracle's set_ghost_cells sweeps exactly (and grids
beyond int32 cell indices are refused), namelist parsing, and grid geometry."""
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


def _split_top(s):
    """Split on commas outside parentheses."""
    out, depth, cur = [], 0, ""
    for ch in s:
        depth += ch == "("
        depth -= ch == ")"
        if ch == "," and depth == 0:
            out.append(cur.strip())
            cur = ""
        else:
            cur += ch
    if cur.strip():
        out.append(cur.strip())
    return out


def _fortran_source(name):
    text = open(os.path.join(ROOT, "include", name)).read()
    src = re.sub(r"!.*", "", text)
    return re.sub(r"&\s*\n\s*", " ", src)


def fortran_module():
    """The interface module (include/boxzy_gpu.f90) up to its `contains`."""
    src = _fortran_source("boxzy_gpu.f90")
    assert src.count("module boxzy_gpu") == 2
    return src.split("\ncontains\n")[0]


def _fortran_decls(body):
    decls = {}
    for stmt in re.split(r"[;\n]", body):
        stmt = stmt.strip()
        if "::" not in stmt:
            continue
        left, names = stmt.split("::")
        parts = _split_top(left)
        spec, attrs = parts[0].replace(" ", ""), [a.replace(" ", "") for a in parts[1:]]
        for n in _split_top(names):
            m = re.match(r"(\w+)\s*(\((.*)\))?", n)
            decls[m.group(1)] = (spec, "value" in attrs, m.group(3))
    return decls


def _header_structs():
    out = {}
    for hdr in ("boxzy_gpu.h",):
        text = open(os.path.join(ROOT, "include", hdr)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"typedef struct (\w+) \{(.*?)\} \1;", text, flags=re.S):
            fields = []
            for decl in m.group(2).split(";"):
                decl = " ".join(decl.replace("const", " ").split())
                if not decl:
                    continue
                base = decl.split()[0]
                for n in decl[len(base):].split(","):
                    n = n.strip()
                    ptr = n.startswith("*")
                    mm = re.match(r"\*?\s*(\w+)(\[(\d+)\])?", n)
                    kind = ("ptr", 8) if ptr else (_C_SCALARS[base][0], _C_SCALARS[base][1])
                    fields += [(mm.group(1), kind)] * int(mm.group(3) or 1)
            out[m.group(1)] = fields
    return out


_F_KINDS = {"real(c_double)": ("f", 8), "integer(c_int64_t)": ("i", 8),
            "integer(c_int32_t)": ("i", 4), "integer(c_int)": ("i", 4), "type(c_ptr)": ("ptr", 8)}


def _fortran_matches(decl, c_param):
    spec, value, dims = decl
    base, depth = c_param
    if spec == "type(c_ptr)":
        return depth >= 1 if value else depth == 2
    if spec.startswith("type("):  # a bind(c) derived type, passed by reference
        return not value and depth == 1 and base == spec[5:-1]
    if spec == "character(kind=c_char)":
        return base == "char" and depth == 1 and dims == "*"
    kind, size = _F_KINDS[spec]
    if value != (depth == 0) or (value and dims):
        return False
    ck, cs = _C_SCALARS[base]
    return cs == size and (ck == kind or (kind == "i" and ck == "u"))


def test_fortran_interfaces_match_the_header():
    """The ISO_C_BINDING module include/boxzy_gpu.f90 (what a maintainer adds to
    the reference) against include/boxzy_gpu.h: every interface binds an exported
    C name with the right argument count, kinds, widths and passing (value or
    reference), its bind(c) types lay out the C structs field by field, and every
    bx_ call of its procedures and of the main loop (include/boxzy_gpu_loop.f90)
    has an interface."""
    src = fortran_module()
    protos = {n: (r, p) for n, r, p in header_prototypes()}
    bad, fnames = [], set()
    funcs = re.finditer(r"(integer\(c_int\)|type\(c_ptr\))\s+function\s+(\w+)\s*\(([^)]*)\)\s*"
                        r"bind\(c,\s*name=\"(\w+)\"\)(.*?)end function", src, flags=re.S)
    for m in funcs:
        res, fname, args, cname, body = m.groups()
        fnames.add(fname)
        if cname not in protos:
            bad.append(f"{fname}: {cname} is not declared in the header")
            continue
        ret, params = protos[cname]
        want = ("int", 0) if res == "integer(c_int)" else None
        if (want and ret != want) or (not want and ret[1] == 0):
            bad.append(f"{fname}: result {res} for C {ret}")
        names = [a.strip() for a in args.split(",") if a.strip()]
        if len(names) != len(params):
            bad.append(f"{fname}: {len(names)} dummies for {len(params)} C parameters")
            continue
        decls = _fortran_decls(body)
        for k, (n, p) in enumerate(zip(names, params)):
            if n not in decls or not _fortran_matches(decls[n], p):
                bad.append(f"{fname} dummy {k} ({n}): {decls.get(n)} vs C {p}")
    assert len(fnames) >= 25, sorted(fnames)
    # bind(c) derived types against the C structs
    structs = _header_structs()
    for m in re.finditer(r"type, bind\(c\) :: (\w+)(.*?)end type", src, flags=re.S):
        name, body = m.groups()
        fields = []
        for stmt in body.strip().split("\n"):
            left, names = stmt.split("::")
            for n in _split_top(names):
                mm = re.match(r"(\w+)(\((\d+)\))?", n)
                fields += [(mm.group(1), _F_KINDS[left.strip()])] * int(mm.group(3) or 1)
        if fields != structs.get(name):
            bad.append(f"type {name}: {fields} vs C {structs.get(name)}")
    # calls in the module's own procedures and in the main loop
    helpers = _fortran_source("boxzy_gpu.f90").split("\ncontains\n")[1]
    own = set(re.findall(r"function\s+(bx_\w+)\s*\(", helpers))
    assert {"bx_message", "bx_advance_to"} <= own
    loop = _fortran_source("boxzy_gpu_loop.f90")
    assert "subroutine bx_main_loop" in loop
    called = set()
    for body in (helpers, loop):
        called |= set(re.findall(r"\b(bx_\w+)\s*\(", body))
    types = {"bx_params", "bx_eos_table"}
    missing = sorted(called - fnames - types - own - {"bx_main_loop"})
    assert not missing, missing
    assert {"bx_run", "bx_step", "bx_download", "bx_advance_to"} <= called
    assert not bad, bad


def test_ghost_plan_rejects_grids_beyond_int32_indices():
    """The plan stores int32 cell indices: 1300^3 cells (> 2^31) is refused before
    any table is built, like bx_create refuses it."""
    hp = HydroParams(nx=1300, ny=1300, nz=1300, dx=0.1, dy=0.1, dz=0.1, h2stat=-1,
                     gammafix=1.4)
    with pytest.raises(_lib.BoxzyError, match="2\\^31"):
        ghost_plan(hp)


def test_batch_refuses_a_box_beyond_int32_indices():
    """Each box's ghost plan holds int32 cell indices: a 1300^3 box is refused
    while the parameters are checked, before any device work."""
    from boxzyhydro_b200.batch import Batch
    hp = HydroParams(nx=1300, ny=1300, nz=1300, dx=0.1, dy=0.1, dz=0.1, h2stat=-1,
                     gammafix=1.4, no_outflow_xl=False, no_outflow_xr=False,
                     no_outflow_yl=False, no_outflow_yr=False, no_outflow_zl=False,
                     no_outflow_zr=False)
    with pytest.raises(_lib.BoxzyError, match="box 0"):
        Batch([hp])


@pytest.mark.parametrize("field,value,msg", [
    ("nx", 4, "too small"), ("ny", 3, "too small"), ("nz", 0, "too small"),
    ("h2stat", -2, "H2STAT"), ("dx", 0.0, ">0"), ("dy", float("nan"), ">0"),
    ("gammafix", 1.0, "gammafix"), ("cfl", 0.0, ">0"), ("dz", 1e-50, "1e-40"),
    ("nx", 1300, "2\\^31")])
def test_create_refuses_invalid_parameters(field, value, msg):
    """bx_create checks its parameters before any device work, so a refusal
    needs no GPU: status BX_ERR_ARG and the message of bx_last_error(NULL)."""
    hp = HydroParams(nx=12, ny=10, nz=8, dx=0.1, dy=0.1, dz=0.1, h2stat=-1, gammafix=1.4)
    p = _lib.make_params(hp)
    if field == "nx" and value == 1300:
        p.nx = p.ny = p.nz = 1300
    else:
        setattr(p, field, value)
    h = ctypes.c_void_p()
    L = _lib.lib()
    assert L.bx_create(ctypes.byref(p), ctypes.byref(h)) == 1  # BX_ERR_ARG
    assert not h.value
    assert re.search(msg, L.bx_last_error(None).decode())


def test_noalloc_sweep_refusals_need_no_device():
    """bx_ghost_fill_noalloc checks its sizes and pointers before any device
    call: negative or oversized counts and null pointers are refused with
    BX_ERR_ARG and a message, an empty sweep is a no-op."""
    L = _lib.lib()
    msg = lambda: L.bx_noalloc_last_error().decode()  # noqa: E731
    vp = ctypes.c_void_p
    assert L.bx_ghost_fill_noalloc(None, 100, None, None, None, 0, None) == 0
    assert L.bx_ghost_fill_noalloc(None, 100, None, None, None, -1, None) == 1
    assert "nghost >= 0" in msg()
    assert L.bx_ghost_fill_noalloc(None, 0, None, None, None, 5, None) == 1
    assert L.bx_ghost_fill_noalloc(None, 1 << 30, None, None, None, (1 << 20) + 1, None) == 1
    assert "1048576" in msg()
    assert L.bx_ghost_fill_noalloc(vp(16), 100, None, vp(16), vp(16), 5, None) == 1
    assert "null device pointer" in msg()


@pytest.mark.parametrize("change,msg", [
    (dict(fluxangmom=True), "unsupported"),
    (dict(h2stat=0), "unsupported"),
    (dict(no_outflow_xl=True, no_outflow_xr=True, no_outflow_yl=True, no_outflow_yr=True,
          no_outflow_zl=True, no_outflow_zr=True), "")])
def test_batch_refuses_boxes_off_the_fused_path(change, msg):
    """A box the fused stages do not run (angular-momentum fluxing, tabulated EOS,
    a ghost fill that two sweeps do not resolve) is refused as unsupported while
    the parameters are checked, before any device work."""
    import dataclasses
    from boxzyhydro_b200.batch import Batch
    base = HydroParams(nx=20, ny=20, nz=20, dx=0.05, dy=0.05, dz=0.05, h2stat=-1,
                       gammafix=1.4, no_outflow_xl=False, no_outflow_xr=False,
                       no_outflow_yl=False, no_outflow_yr=False, no_outflow_zl=False,
                       no_outflow_zr=False)
    hp = dataclasses.replace(base, **change)
    with pytest.raises(_lib.BoxzyError, match="UNSUPPORTED") as e:
        Batch([hp])
    assert msg in str(e.value)
