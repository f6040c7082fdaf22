"""ctypes binding of libboxzy_gpu.so (the C ABI declared in include/boxzy_gpu.h).

The library is built in-tree (boxzyhydro_b200/Makefile) and loaded from this
package directory.  There is no fallback: if the shared library is missing or a
call fails, a BoxzyError is raised.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libboxzy_gpu.so")

BX_OK = 0
ERR_NAMES = {1: "BX_ERR_ARG", 2: "BX_ERR_CUDA", 3: "BX_ERR_UNSUPPORTED", 4: "BX_ERR_STATE",
             5: "BX_ERR_NOMEM"}
STATUS_VLIMIT, STATUS_LOWRHO, STATUS_NONFINITE, STATUS_ZEROWAVE = 1, 2, 4, 8
FLAG_PHASE_ONLY = 1


class BoxzyError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERR_NAMES.get(code, code)}: {msg}")
        self.code = code


class BxParams(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("h2stat", C.c_int32),
        ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
        ("cfl", C.c_double), ("small_rho", C.c_double), ("small_eps", C.c_double),
        ("vlimit", C.c_double), ("gammafix", C.c_double), ("muc", C.c_double),
        ("rgas", C.c_double), ("no_outflow", C.c_int32 * 6), ("fluxangmom", C.c_int32),
        ("flags", C.c_int32), ("yoffset", C.c_double),
    ]


class BxEosTable(C.Structure):
    _fields_ = [
        ("neos", C.c_int32), ("neos_rho", C.c_int32),
        ("log_rho_eos_low", C.c_double), ("drho_eos", C.c_double),
        ("density_unit", C.c_double), ("tk_bgrnd", C.c_double),
        ("eng_table2", C.c_void_p), ("gamma_table2", C.c_void_p),
        ("muc_table2", C.c_void_p), ("tk_table2", C.c_void_p),
        ("rho_table", C.c_void_p), ("deng_eos_array", C.c_void_p),
    ]


_lib = None


def lib():
    """Load the library (raises BoxzyError when it is not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise BoxzyError(-1, f"{LIB_PATH} is not built; run `make -C {_HERE}` "
                             "or __graft_entry__.build()")
    L = C.CDLL(LIB_PATH)
    H = C.c_void_p
    dp = C.POINTER(C.c_double)
    i64p = C.POINTER(C.c_int64)
    i32p = C.POINTER(C.c_int32)
    vp = C.c_void_p
    sig = {
        "bx_version": (C.c_char_p, []),
        "bx_last_error": (C.c_char_p, [H]),
        "bx_create": (C.c_int, [C.POINTER(BxParams), C.POINTER(H)]),
        "bx_destroy": (C.c_int, [H]),
        "bx_set_stream": (C.c_int, [H, vp]),
        "bx_upload": (C.c_int, [H, vp, vp, vp]),
        "bx_download": (C.c_int, [H, vp, vp, vp]),
        "bx_upload_conserved": (C.c_int, [H, vp]),
        "bx_set_clock": (C.c_int, [H, C.c_double, C.c_double, C.c_int64]),
        "bx_get_clock": (C.c_int, [H, dp, dp, dp, i64p]),
        "bx_step": (C.c_int, [H, C.c_double, i32p]),
        "bx_step_host": (C.c_int, [H, vp, vp, C.c_double, i32p]),
        "bx_run": (C.c_int, [H, C.c_double, C.c_int64, i64p]),
        "bx_write_celldump": (C.c_int, [H, C.c_char_p, vp]),
        "bx_read_celldump": (C.c_int, [H, C.c_char_p, vp, dp, i64p]),
        "bx_state": (C.c_int, [H]),
        "bx_velocity": (C.c_int, [H]),
        "bx_courant": (C.c_int, [H, dp]),
        "bx_source": (C.c_int, [H, C.c_int32]),
        "bx_ghost": (C.c_int, [H]),
        "bx_flux": (C.c_int, [H, C.c_int32]),
        "bx_avisc": (C.c_int, [H]),
        "bx_set_avmag": (C.c_int, [H, C.c_double, C.c_double, C.c_double]),
        "bx_download_qq": (C.c_int, [H, C.c_void_p]),
        "bx_save_cons_old": (C.c_int, [H]),
        "bx_set_dt": (C.c_int, [H, C.c_double]),
        "bx_set_gforce": (C.c_int, [H, vp]),
        "bx_set_phi": (C.c_int, [H, vp]),
        "bx_set_eos_table": (C.c_int, [H, C.POINTER(BxEosTable)]),
        "bx_status": (C.c_int, [H, C.POINTER(C.c_uint32), i32p]),
        "bx_device_cons": (C.c_int, [H, C.POINTER(C.c_void_p), i64p]),
        "bx_ghost_plan": (C.c_int, [C.POINTER(BxParams), i64p, vp, vp, vp, vp, vp, i32p]),
        "bx_profile": (C.c_int, [H, C.c_int32]),
        "bx_profile_read": (C.c_int, [H, dp, dp, i64p, i64p]),
        "bx_step_host_profile": (C.c_int, [H, C.c_int32]),
        "bx_step_host_timeline": (C.c_int, [H, C.POINTER(C.c_int32), dp]),
        "bx_fp64_peak": (C.c_int, [dp, dp]),
        "bx_check_shared_division": (C.c_int, [C.c_ulonglong, C.c_ulonglong, C.c_int,
                                               C.POINTER(C.c_ulonglong), dp, dp]),
        "bx_ghost_fill_noalloc": (C.c_int, [vp, C.c_int64, vp, vp, vp, C.c_int64, vp]),
        "bx_noalloc_last_error": (C.c_char_p, []),
        "bx_batch_create": (C.c_int, [C.c_int32, C.POINTER(BxParams), C.POINTER(H)]),
        "bx_batch_destroy": (C.c_int, [H]),
        "bx_batch_set_stream": (C.c_int, [H, vp]),
        "bx_batch_upload": (C.c_int, [H, C.c_int32, vp]),
        "bx_batch_set_clock": (C.c_int, [H, C.c_int32, C.c_double, C.c_double, C.c_int64]),
        "bx_batch_get_clock": (C.c_int, [H, C.c_int32, dp, dp, dp, i64p]),
        "bx_batch_run": (C.c_int, [H, C.c_int64, C.c_double, C.c_int32]),
        "bx_batch_autotune": (C.c_int, [H, C.c_int32, i32p, dp]),
        "bx_batch_set_persistent": (C.c_int, [H, C.c_int32]),
        "bx_batch_set_tile_shape": (C.c_int, [H, C.c_int32]),
        "bx_batch_get_tile_shape": (C.c_int, [H, i32p, i32p, i32p, i32p]),
        "bx_batch_get_persistent": (C.c_int, [H, i32p]),
        "bx_batch_wait_selftest": (C.c_int, [C.c_int64, i32p, dp]),
        "bx_batch_download": (C.c_int, [H, C.c_int32, vp, vp, vp]),
        "bx_batch_info": (C.c_int, [H, dp, i64p, i32p, i64p]),
        "bx_batch_last_error": (C.c_char_p, [H]),
        "bx_adj_create": (C.c_int, [C.POINTER(BxParams), C.c_int64, C.c_int32, C.POINTER(H)]),
        "bx_adj_destroy": (C.c_int, [H]),
        "bx_adj_set_stream": (C.c_int, [H, vp]),
        "bx_adj_keep_stage0": (C.c_int, [H, C.c_int32]),
        "bx_adj_stage0_cache": (C.c_int, [H, C.c_int32]),
        "bx_adj_host_level": (C.c_int, [H, C.c_int64, C.POINTER(C.c_int64)]),
        "bx_adj_forward": (C.c_int, [H, vp, vp, C.c_int32]),
        "bx_adj_forward_branches": (C.c_int, [H, vp, vp, vp, vp]),
        "bx_adj_backward": (C.c_int, [H, vp, vp]),
        "bx_adj_stats": (C.c_int, [H, dp, dp, i64p, i64p]),
        "bx_adj_dts": (C.c_int, [H, dp]),
        "bx_adj_plan": (C.c_int, [C.c_int64, C.c_int32, i64p, i64p, i32p]),
        "bx_adj_device_bytes": (C.c_int, [C.POINTER(BxParams), C.c_int64, C.c_int32, C.c_int32,
                                          C.c_int32, i64p]),
        "bx_adj_last_error": (C.c_char_p, [H]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def check(rc, h=None):
    if rc != BX_OK:
        msg = lib().bx_last_error(h)
        raise BoxzyError(rc, msg.decode() if msg else "")


def make_params(hp, flags=0) -> BxParams:
    """bx_params from a HydroParams (namelist fields)."""
    p = BxParams()
    p.nx, p.ny, p.nz = int(hp.nx), int(hp.ny), int(hp.nz)
    p.h2stat = int(hp.h2stat)
    p.dx, p.dy, p.dz = float(hp.dx), float(hp.dy), float(hp.dz)
    p.cfl = float(hp.cfl)
    p.small_rho = float(hp.small_rho)
    p.small_eps = float(hp.small_eps)
    p.vlimit = float(hp.vlimit)
    p.gammafix = float(hp.gammafix)
    p.muc = float(hp.muc)
    p.rgas = float(hp.rgas)
    walls = (hp.no_outflow_xl, hp.no_outflow_xr, hp.no_outflow_yl, hp.no_outflow_yr,
             hp.no_outflow_zl, hp.no_outflow_zr)
    for k, w in enumerate(walls):
        p.no_outflow[k] = 1 if w else 0
    p.fluxangmom = 1 if hp.fluxangmom else 0
    p.flags = int(flags)
    p.yoffset = float(hp.yoffset)
    return p
