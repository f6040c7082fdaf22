"""ctypes binding of the CPU oracle (oracle/bx_oracle.c).

TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and bench.py's
cpu_baseline leg use this module as the checker.  The product never imports it.

Parity status: per-step parity of the restatement is unpinned by a reference
binary (no Fortran compiler in this image); end states are pinned by
tests/test_oracle_golden.py against the reference's analysis/sod.ana and
analysis/sodtest.dat.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libbx_oracle.so")
_lib = None


class OxParams(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("h2stat", C.c_int32),
        ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
        ("cfl", C.c_double), ("small_rho", C.c_double), ("small_eps", C.c_double),
        ("vlimit", C.c_double), ("gammafix", C.c_double),
        ("muc", C.c_double), ("rgas", C.c_double),
        ("no_outflow", C.c_int32 * 6), ("racy_ghosts", C.c_int32), ("pad", C.c_int32),
        ("fluxangmom", C.c_int32), ("pad2", C.c_int32), ("yoffset", C.c_double),
    ]


def build():
    """Compile the oracle library with its Makefile (gcc, -ffp-contract=off)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        P = C.c_void_p
        dp = C.POINTER(C.c_double)
        L.ox_create.restype = P
        L.ox_create.argtypes = [C.POINTER(OxParams)]
        L.ox_destroy.argtypes = [P]
        L.ox_ngrid.restype = C.c_int64
        L.ox_ngrid.argtypes = [P]
        L.ox_nghost.restype = C.c_int64
        L.ox_nghost.argtypes = [P]
        L.ox_grid_info.argtypes = [P, C.c_void_p, C.c_void_p]
        L.ox_ghost_list.argtypes = [P, C.c_void_p]
        L.ox_set_state.argtypes = [P, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.ox_get_state.argtypes = [P, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.ox_set_gforce.argtypes = [P, C.c_void_p]
        L.ox_get_cons_old.argtypes = [P, C.c_void_p]
        L.ox_set_cons_old.argtypes = [P, C.c_void_p]
        L.ox_set_clock.argtypes = [P, C.c_double, C.c_double, C.c_double, C.c_int64]
        L.ox_get_clock.argtypes = [P, dp, dp, dp, C.POINTER(C.c_int64), dp]
        for fn in ("ox_state", "ox_velocity", "ox_courant", "ox_set_ghost_cells",
                   "ox_save_cons_old"):
            getattr(L, fn).argtypes = [P]
        L.ox_source.argtypes = [P, C.c_int]
        L.ox_avisc.argtypes = [P, C.c_double, C.c_double, C.c_double, C.c_void_p]
        L.ox_flux.argtypes = [P, C.c_int]
        L.ox_flux_ang.argtypes = [P, C.c_int]
        L.ox_step.argtypes = [P, C.c_double]
        L.ox_step.restype = C.c_int
        L.ox_step_dt.argtypes = [P, C.c_double]
        L.ox_run.argtypes = [P, C.c_double, C.c_int64]
        L.ox_run.restype = C.c_int64
        L.ox_set_threads.argtypes = [C.c_int]
        L.ox_rgas_code_units.restype = C.c_double
        L.ox_set_eos_table.argtypes = [P, C.c_void_p]
        L.ox_get_muc.argtypes = [P, C.c_void_p]
        L.ox_muc.restype = C.c_double
        L.ox_muc.argtypes = [C.c_double] * 4
        for fn in ("ox_kat_genminmod", "ox_kat_slope"):
            getattr(L, fn).restype = C.c_double
            getattr(L, fn).argtypes = [C.c_double] * 3
        L.ox_kat_muscl.argtypes = [C.c_double] * 4 + [dp, dp]
        L.ox_kat_face_flux.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class OxEosTable(C.Structure):
    _fields_ = [
        ("neos", C.c_int32), ("neos_rho", C.c_int32),
        ("log_rho_eos_low", C.c_double), ("drho_eos", C.c_double),
        ("density_unit", C.c_double), ("tk_bgrnd", C.c_double),
        ("eng_table2", C.c_void_p), ("gamma_table2", C.c_void_p),
        ("muc_table2", C.c_void_p), ("tk_table2", C.c_void_p),
        ("rho_table", C.c_void_p), ("deng_eos_array", C.c_void_p),
    ]


class Oracle:
    """One reference grid held on the CPU, with the reference's global arrays.

    Arrays use the reference layout: cons (ng,5), u (ng,3), p (ng,), adindx (ng,),
    cell index = ix + iy*nx + iz*nx*ny (0-based), x fastest.
    """

    def __init__(self, params, racy_ghosts=False):
        L = lib()
        op = OxParams()
        op.nx, op.ny, op.nz = int(params.nx), int(params.ny), int(params.nz)
        op.h2stat = int(params.h2stat)
        op.dx, op.dy, op.dz = float(params.dx), float(params.dy), float(params.dz)
        op.cfl = float(params.cfl)
        op.small_rho = float(params.small_rho)
        op.small_eps = float(params.small_eps)
        op.vlimit = float(params.vlimit)
        op.gammafix = float(params.gammafix)
        op.muc = float(params.muc)
        op.rgas = float(params.rgas)
        for k, w in enumerate(params.no_outflow):
            op.no_outflow[k] = 1 if w else 0
        op.racy_ghosts = 1 if racy_ghosts else 0
        op.fluxangmom = 1 if getattr(params, "fluxangmom", False) else 0
        op.yoffset = float(getattr(params, "yoffset", 0.0))
        self._h = L.ox_create(C.byref(op))
        self.ng = int(L.ox_ngrid(self._h))
        self.params = params

    def close(self):
        if self._h:
            lib().ox_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- arrays
    def set_state(self, cons, u=None, p=None, adindx=None):
        f = lambda a, n: None if a is None else np.ascontiguousarray(a, dtype=np.float64).reshape(self.ng * n)
        c, uu, pp, gg = f(cons, 5), f(u, 3), f(p, 1), f(adindx, 1)
        lib().ox_set_state(self._h, _ptr(c), _ptr(uu), _ptr(pp), _ptr(gg))

    def get_state(self):
        c = np.empty((self.ng, 5))
        u = np.empty((self.ng, 3))
        p = np.empty(self.ng)
        g = np.empty(self.ng)
        lib().ox_get_state(self._h, _ptr(c), _ptr(u), _ptr(p), _ptr(g))
        return c, u, p, g

    def set_gforce(self, g3):
        g = None if g3 is None else np.ascontiguousarray(g3, dtype=np.float64)
        lib().ox_set_gforce(self._h, _ptr(g))

    def calc_gforce(self, phi):
        """utils.f90:549-571 (calc_gforce): gforce = -(phi(b+) - phi(b-))/(2 d) on
        interior cells through the neighbour table (b(3)/b(4) x, b(1)/b(2) y,
        b(5)/b(6) z); ghost rows zero."""
        b, nb = self.grid_info()
        m = b == 0
        P = self.params
        phi = np.asarray(phi, dtype=np.float64)
        g = np.zeros((self.ng, 3))
        g[m, 0] = -(phi[nb[m, 2]] - phi[nb[m, 3]]) / (2.0 * P.dx)
        g[m, 1] = -(phi[nb[m, 0]] - phi[nb[m, 1]]) / (2.0 * P.dy)
        g[m, 2] = -(phi[nb[m, 4]] - phi[nb[m, 5]]) / (2.0 * P.dz)
        return g

    def set_eos_table(self, tab):
        """tab: dict of the eos module's tables (see boxzyhydro_b200.eos_table)."""
        keep = {k: np.asfortranarray(tab[k], dtype=np.float64)
                for k in ("eng_table2", "gamma_table2", "muc_table2", "tk_table2",
                          "rho_table", "deng_eos_array")}
        t = OxEosTable()
        t.neos, t.neos_rho = int(tab["neos"]), int(tab["neos_rho"])
        t.log_rho_eos_low = float(tab["log_rho_eos_low"])
        t.drho_eos = float(tab["drho_eos"])
        t.density_unit = float(tab["density_unit"])
        t.tk_bgrnd = float(tab["tk_bgrnd"])
        for k, a in keep.items():
            setattr(t, k, a.ctypes.data)
        lib().ox_set_eos_table(self._h, C.byref(t))

    def muc_array(self):
        m = np.empty(self.ng)
        lib().ox_get_muc(self._h, _ptr(m))
        return m

    def get_cons_old(self):
        c = np.empty((self.ng, 5))
        lib().ox_get_cons_old(self._h, _ptr(c))
        return c

    def set_cons_old(self, c):
        c = np.ascontiguousarray(c, dtype=np.float64)
        lib().ox_set_cons_old(self._h, _ptr(c))

    def grid_info(self):
        b = np.empty(self.ng, dtype=np.int32)
        nb = np.empty((self.ng, 6), dtype=np.int32)
        lib().ox_grid_info(self._h, _ptr(b), _ptr(nb))
        return b, nb

    def ghost_list(self):
        n = int(lib().ox_nghost(self._h))
        idx = np.empty(n, dtype=np.int64)
        lib().ox_ghost_list(self._h, _ptr(idx))
        return idx

    # ---- clock
    def set_clock(self, time=0.0, dt=0.0, dtold=0.0, step=0):
        lib().ox_set_clock(self._h, time, dt, dtold, step)

    def clock(self):
        t, dt, dto, r = C.c_double(), C.c_double(), C.c_double(), C.c_double()
        st = C.c_int64()
        lib().ox_get_clock(self._h, C.byref(t), C.byref(dt), C.byref(dto), C.byref(st), C.byref(r))
        return dict(time=t.value, dt=dt.value, dtold=dto.value, step=st.value, dtrate=r.value)

    # ---- phases
    def state(self):
        lib().ox_state(self._h)

    def velocity(self):
        lib().ox_velocity(self._h)

    def courant(self):
        lib().ox_courant(self._h)

    def source(self, siter):
        lib().ox_source(self._h, int(siter))

    def set_ghost_cells(self):
        lib().ox_set_ghost_cells(self._h)

    def flux(self, avg):
        """flux(avg), or flux_ang(avg) when fluxangmom is set (main.f90:343-346)."""
        if getattr(self.params, "fluxangmom", False):
            lib().ox_flux_ang(self._h, int(avg))
        else:
            lib().ox_flux(self._h, int(avg))

    def save_cons_old(self):
        lib().ox_save_cons_old(self._h)

    def avisc(self, avmagx=0.0, avmagy=0.0, avmagz=0.0):
        """qq(3, ngrid) of avisc.f90:4-26 from the current velocity array, (ngrid, 3)."""
        qq = np.empty((self.ng, 3))
        lib().ox_avisc(self._h, float(avmagx), float(avmagy), float(avmagz), qq.ctypes.data)
        return qq

    def step(self, endtime=1e300):
        return lib().ox_step(self._h, float(endtime)) == 0

    def step_dt(self, dt_full):
        lib().ox_step_dt(self._h, float(dt_full))

    def run(self, endtime=1e300, nsteps=1 << 62):
        return int(lib().ox_run(self._h, float(endtime), int(nsteps)))


def set_threads(n):
    lib().ox_set_threads(int(n))


def rgas_code_units():
    return lib().ox_rgas_code_units()


def muc(xabun=0.73, yabun=0.27, zabun=0.0, mu_z=16.78):
    return lib().ox_muc(xabun, yabun, zabun, mu_z)


# known-answer probes of the restatement's building blocks (its own tests)
def kat_genminmod(x1, x2, x3):
    return lib().ox_kat_genminmod(float(x1), float(x2), float(x3))


def kat_slope(c0, c1, c2):
    return lib().ox_kat_slope(float(c0), float(c1), float(c2))


def kat_muscl(q, lm, lp, sl):
    """(minus, plus) face states of interface_muscl."""
    m, p = C.c_double(), C.c_double()
    lib().ox_kat_muscl(float(q), float(lm), float(lp), float(sl), C.byref(m), C.byref(p))
    return m.value, p.value


def kat_face_flux(left, right, idir):
    """HLL flux (5,) of one face; left/right = (rho, u1, u2, u3, p, eps, gamma)."""
    L = np.ascontiguousarray(left, dtype=np.float64)
    R = np.ascontiguousarray(right, dtype=np.float64)
    assert L.shape == (7,) and R.shape == (7,) and idir in (0, 1, 2)
    f = np.empty(5)
    lib().ox_kat_face_flux(_ptr(L), _ptr(R), int(idir), _ptr(f))
    return f
