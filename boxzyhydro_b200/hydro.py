"""Host-side mirror of the reference's hydro-step interface, over the C ABI.

`Hydro` holds one grid on the GPU.  Its methods carry the names of the
reference's subroutines (state, velocity, courant, source, set_ghost_cells,
flux, avisc) and act on the handle's device copies of the module arrays
exactly as those subroutines act on grid_commons; `step` is one iteration of
the main loop (main.f90:212-545) and `run` the loop itself.  Arrays cross the
boundary in the reference layout: cons (ng,5), u (ng,3), p (ng,).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _lib
from ._lib import BoxzyError, check, lib, make_params
from .params import HydroParams


def _arr(a, n, k):
    if a is None:
        return None
    a = np.ascontiguousarray(a, dtype=np.float64)
    if a.size != n * k:
        raise ValueError(f"expected {n}x{k} doubles, got shape {a.shape}")
    return a


class Hydro:
    """One BOXZYHYDRO grid advanced by the sm_100a kernels."""

    def __init__(self, params: HydroParams, phase_only: bool = False):
        params.validate()
        self.params = params
        self.ng = params.ngrid
        self._p = make_params(params, _lib.FLAG_PHASE_ONLY if phase_only else 0)
        h = C.c_void_p()
        check(lib().bx_create(C.byref(self._p), C.byref(h)), None)
        self._h = h

    # ---- lifetime
    def close(self):
        if getattr(self, "_h", None):
            lib().bx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _c(self, rc):
        check(rc, self._h)

    # ---- arrays
    def upload(self, cons, u=None, p=None):
        c = _arr(cons, self.ng, 5)
        uu = _arr(u, self.ng, 3)
        pp = _arr(p, self.ng, 1)
        ptr = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)
        self._c(lib().bx_upload(self._h, ptr(c), ptr(uu), ptr(pp)))

    def upload_conserved(self, cons):
        """State at a step boundary from cons alone (u = m/rho, p from state())."""
        c = _arr(cons, self.ng, 5)
        self._c(lib().bx_upload_conserved(self._h, c.ctypes.data_as(C.c_void_p)))

    def upload_state(self, st):
        self.upload(st.cons, st.u, st.p)

    def download(self):
        c = np.empty((self.ng, 5))
        u = np.empty((self.ng, 3))
        p = np.empty(self.ng)
        self._c(lib().bx_download(self._h, c.ctypes.data_as(C.c_void_p),
                                  u.ctypes.data_as(C.c_void_p), p.ctypes.data_as(C.c_void_p)))
        return c, u, p

    def set_gforce(self, g3):
        g = _arr(g3, self.ng, 3)
        self._c(lib().bx_set_gforce(self._h, None if g is None else g.ctypes.data_as(C.c_void_p)))

    def set_eos_table(self, tab):
        """Tables of the eos module for H2STAT >= 0 (dict with neos, neos_rho,
        log_rho_eos_low, drho_eos, density_unit, tk_bgrnd and the arrays
        eng_table2, gamma_table2, muc_table2, tk_table2 of shape (neos, neos_rho)
        and rho_table, deng_eos_array of neos_rho)."""
        keep = {k: np.asfortranarray(tab[k], dtype=np.float64)
                for k in ("eng_table2", "gamma_table2", "muc_table2", "tk_table2",
                          "rho_table", "deng_eos_array")}
        t = _lib.BxEosTable()
        t.neos, t.neos_rho = int(tab["neos"]), int(tab["neos_rho"])
        t.log_rho_eos_low = float(tab["log_rho_eos_low"])
        t.drho_eos = float(tab["drho_eos"])
        t.density_unit = float(tab["density_unit"])
        t.tk_bgrnd = float(tab["tk_bgrnd"])
        for k, a in keep.items():
            setattr(t, k, a.ctypes.data)
        self._c(lib().bx_set_eos_table(self._h, C.byref(t)))

    def set_phi(self, phi):
        """Gravitational potential from the host's solver: gforce by calc_gforce."""
        ph = _arr(phi, self.ng, 1)
        self._c(lib().bx_set_phi(self._h, None if ph is None else ph.ctypes.data_as(C.c_void_p)))

    def set_stream(self, stream_ptr):
        self._c(lib().bx_set_stream(self._h, C.c_void_p(stream_ptr) if stream_ptr else None))

    def device_cons(self):
        """(device pointer, ngrid) of the reference cons planes (SoA, 5 x ngrid)."""
        ptr = C.c_void_p()
        n = C.c_int64()
        self._c(lib().bx_device_cons(self._h, C.byref(ptr), C.byref(n)))
        return ptr.value, n.value

    # ---- clock (main.f90 time, dt, dtold, step)
    def set_clock(self, time=0.0, dtold=0.0, step=0):
        self._c(lib().bx_set_clock(self._h, float(time), float(dtold), int(step)))

    def clock(self):
        t, dt, dto = C.c_double(), C.c_double(), C.c_double()
        st = C.c_int64()
        self._c(lib().bx_get_clock(self._h, C.byref(t), C.byref(dt), C.byref(dto), C.byref(st)))
        return dict(time=t.value, dt=dt.value, dtold=dto.value, step=st.value)

    def set_dt(self, dt):
        self._c(lib().bx_set_dt(self._h, float(dt)))

    # ---- celldump files (write_files.f90:55-63, read_hydro.f90:122-187)
    def write_celldump(self, path, phi=None):
        """state() on the arrays, then the celldump of the handle's state."""
        ph = _arr(phi, self.ng, 1)
        self._c(lib().bx_write_celldump(self._h, os.fsencode(path),
                                        None if ph is None else ph.ctypes.data_as(C.c_void_p)))

    def read_celldump(self, path, want_phi=False):
        """Restart from a celldump: returns (time, step[, phi])."""
        ph = np.empty(self.ng) if want_phi else None
        t = C.c_double()
        st = C.c_int64()
        self._c(lib().bx_read_celldump(self._h, os.fsencode(path),
                                       None if ph is None else ph.ctypes.data_as(C.c_void_p),
                                       C.byref(t), C.byref(st)))
        return (t.value, st.value, ph) if want_phi else (t.value, st.value)

    # ---- the reference's subroutines
    def state(self):
        self._c(lib().bx_state(self._h))

    def velocity(self):
        self._c(lib().bx_velocity(self._h))

    def courant(self):
        dt = C.c_double()
        self._c(lib().bx_courant(self._h, C.byref(dt)))
        return dt.value

    def source(self, siter):
        self._c(lib().bx_source(self._h, int(siter)))

    def set_ghost_cells(self):
        self._c(lib().bx_ghost(self._h))

    def flux(self, avg):
        self._c(lib().bx_flux(self._h, int(avg)))

    def avisc(self):
        """avisc.f90:4-26 on the device: the qq array from the velocity array."""
        self._c(lib().bx_avisc(self._h))

    def set_avmag(self, avmagx=0.0, avmagy=0.0, avmagz=0.0):
        """The hydro namelist's avmagx/y/z (parameters.f90:77) that avisc reads."""
        self._c(lib().bx_set_avmag(self._h, float(avmagx), float(avmagy), float(avmagz)))

    def qq(self):
        """The artificial-viscosity array qq(3, ngrid), as (ngrid, 3)."""
        out = np.empty((self.params.ngrid, 3))
        self._c(lib().bx_download_qq(self._h, out.ctypes.data))
        return out

    def save_cons_old(self):
        self._c(lib().bx_save_cons_old(self._h))

    # ---- main loop
    def step(self, endtime=1e300):
        ran = C.c_int32()
        self._c(lib().bx_step(self._h, float(endtime), C.byref(ran)))
        return bool(ran.value)

    def step_host(self, cons_in, cons_out=None, endtime=1e300):
        """One step of a state held on the host: upload_conserved(cons_in), step(),
        download of cons into cons_out (cons_in itself when None), with the copies
        overlapped with the step (bx_step_host).  Arrays (ngrid, 5) float64,
        C-contiguous; page-locked memory lets the copies run asynchronously."""
        if cons_out is None:
            cons_out = cons_in
        for a in (cons_in, cons_out):
            if (not isinstance(a, np.ndarray) or a.dtype != np.float64 or a.shape != (self.ng, 5)
                    or not a.flags.c_contiguous):
                raise ValueError("cons arrays must be C-contiguous float64 of shape (ngrid, 5)")
        if not cons_out.flags.writeable:
            raise ValueError("cons_out must be writeable")
        ran = C.c_int32()
        self._c(lib().bx_step_host(self._h, cons_in.ctypes.data_as(C.c_void_p),
                                   cons_out.ctypes.data_as(C.c_void_p), float(endtime),
                                   C.byref(ran)))
        return bool(ran.value)

    def run(self, endtime=1e300, nsteps=(1 << 62)):
        n = C.c_int64()
        self._c(lib().bx_run(self._h, float(endtime), int(nsteps), C.byref(n)))
        return n.value

    def profile(self, enable=True):
        """Start (or stop) CUDA-event timing of the fused stage kernels."""
        self._c(lib().bx_profile(self._h, 1 if enable else 0))

    def profile_read(self):
        a, b = C.c_double(), C.c_double()
        n, k = C.c_int64(), C.c_int64()
        self._c(lib().bx_profile_read(self._h, C.byref(a), C.byref(b), C.byref(n), C.byref(k)))
        return dict(ms_stage0=a.value, ms_stage1=b.value, fused_steps=n.value, launches=k.value)

    def step_host_profile(self, enable=True):
        """Record CUDA events per slab in the following step_host calls."""
        self._c(lib().bx_step_host_profile(self._h, 1 if enable else 0))

    def step_host_timeline(self):
        """The last profiled step_host call, per slab (rows): milliseconds from
        its start to upload start, upload end, stage 0 enqueued after that
        upload, stage 1 end, conversion end, download start, download end."""
        ns = C.c_int32()
        self._c(lib().bx_step_host_timeline(self._h, C.byref(ns), None))
        ms = np.empty((ns.value, 7), dtype=np.float64)
        self._c(lib().bx_step_host_timeline(self._h, C.byref(ns),
                                            ms.ctypes.data_as(C.POINTER(C.c_double))))
        return ms

    def status(self):
        bits = C.c_uint32()
        path = C.c_int32()
        self._c(lib().bx_status(self._h, C.byref(bits), C.byref(path)))
        return bits.value, path.value


def ghost_plan(params: HydroParams, phase_only=False):
    """The ghost-fill plan of a grid (host only, no GPU): dict of arrays."""
    p = make_params(params, _lib.FLAG_PHASE_ONLY if phase_only else 0)
    n = C.c_int64(0)
    ok = C.c_int32(0)
    check(lib().bx_ghost_plan(C.byref(p), C.byref(n), None, None, None, None, None,
                              C.byref(ok)))
    k = n.value
    out = dict(dst=np.empty(k, np.int32), src1=np.empty(k, np.int32), sgn1=np.empty(k, np.uint8),
               src2=np.empty(k, np.int32), sgn2=np.empty(k, np.uint8))
    vp = lambda a: a.ctypes.data_as(C.c_void_p)
    check(lib().bx_ghost_plan(C.byref(p), C.byref(n), vp(out["dst"]), vp(out["src1"]),
                              vp(out["sgn1"]), vp(out["src2"]), vp(out["sgn2"]), C.byref(ok)))
    out["fused_ok"] = bool(ok.value)
    return out


def apply_ghost_plan(cons, src, sgn, dst):
    """Apply a plan to a (ng,5) array on the host (gather then scatter)."""
    vals = cons[src].copy()
    for b, k in ((1, 1), (2, 2), (4, 3)):
        m = (sgn & b) != 0
        vals[m, k] = -vals[m, k]
    out = cons.copy()
    out[dst] = vals
    return out


def fp64_peak():
    """Measured FP64 FMA throughput of the current device (TFLOP/s)."""
    t, ms = C.c_double(), C.c_double()
    check(lib().bx_fp64_peak(C.byref(t), C.byref(ms)))
    return t.value


__all__ = ["Hydro", "BoxzyError", "ghost_plan", "apply_ghost_plan", "fp64_peak"]
