"""Batched ensembles of independent boxes (bx_batch_* of the C ABI).

The reference advances one grid per process.  `Batch` advances many grids at
once -- each with its own size, gamma, CFL number, dt and clock -- with the same
stage kernels as `Hydro`, so every box evolves exactly as it would alone; a run
of n steps is one CUDA graph launch (four kernels per step, or one persistent
kernel for the whole run).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import BoxzyError, lib, make_params
from .params import HydroParams


class Batch:
    def __init__(self, params_list):
        self.params = list(params_list)
        n = len(self.params)
        for hp in self.params:
            hp.validate()
        arr = (type(make_params(self.params[0])) * n)(*[make_params(hp) for hp in self.params])
        h = C.c_void_p()
        rc = lib().bx_batch_create(n, arr, C.byref(h))
        if rc:
            raise BoxzyError(rc, lib().bx_batch_last_error(None).decode())
        self._h = h
        self.nbox = n

    def _c(self, rc):
        if rc:
            raise BoxzyError(rc, lib().bx_batch_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None):
            lib().bx_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr):
        self._c(lib().bx_batch_set_stream(self._h, C.c_void_p(stream_ptr) if stream_ptr else None))

    def upload(self, box, cons):
        hp = self.params[box]
        c = np.ascontiguousarray(cons, dtype=np.float64)
        if c.size != hp.ngrid * 5:
            raise ValueError("cons must be (ngrid,5)")
        self._c(lib().bx_batch_upload(self._h, int(box), c.ctypes.data_as(C.c_void_p)))

    def set_clock(self, box, time=0.0, dtold=0.0, step=0):
        self._c(lib().bx_batch_set_clock(self._h, int(box), float(time), float(dtold), int(step)))

    def clock(self, box):
        t, dt, dto = C.c_double(), C.c_double(), C.c_double()
        st = C.c_int64()
        self._c(lib().bx_batch_get_clock(self._h, int(box), C.byref(t), C.byref(dt),
                                         C.byref(dto), C.byref(st)))
        return dict(time=t.value, dt=dt.value, dtold=dto.value, step=st.value)

    def run(self, nsteps, endtime=1e300, graph=True):
        self._c(lib().bx_batch_run(self._h, int(nsteps), float(endtime), 1 if graph else 0))

    def set_persistent(self, enable=True):
        """One launch per run (a queue of step/stage/tile items) instead of four
        launches per step; the same results."""
        self._c(lib().bx_batch_set_persistent(self._h, 1 if enable else 0))

    def set_tile_shape(self, shape):
        """0: 32 x 8 column tiles, 1: 16 x 16 (the same results)."""
        self._c(lib().bx_batch_set_tile_shape(self._h, int(shape)))

    @property
    def tile_shape(self):
        """(shape index, tx, ty, depth) of the stage kernels' tiles."""
        v = [C.c_int32() for _ in range(4)]
        self._c(lib().bx_batch_get_tile_shape(self._h, *[C.byref(x) for x in v]))
        return tuple(x.value for x in v)

    @property
    def persistent(self):
        e = C.c_int32()
        self._c(lib().bx_batch_get_persistent(self._h, C.byref(e)))
        return bool(e.value)

    def autotune(self, reps=2):
        """Pick the ensemble's tile shape and depth, then the launch form (four
        launches per step or one persistent launch), by timing trial steps from the
        current states (left unchanged): returns (depth, ms per step); depth 0 is
        the default rule, >= 2**30 whole box depths; `tile_shape` and `persistent`
        tell the rest."""
        zc = C.c_int32()
        ms = C.c_double()
        self._c(lib().bx_batch_autotune(self._h, int(reps), C.byref(zc), C.byref(ms)))
        return zc.value, ms.value

    def download(self, box):
        n = self.params[box].ngrid
        c = np.empty((n, 5))
        u = np.empty((n, 3))
        p = np.empty(n)
        self._c(lib().bx_batch_download(self._h, int(box), c.ctypes.data_as(C.c_void_p),
                                        u.ctypes.data_as(C.c_void_p),
                                        p.ctypes.data_as(C.c_void_p)))
        return c, u, p

    def info(self):
        ms = C.c_double()
        nl = C.c_int64()
        ns = C.c_int32()
        cells = C.c_int64()
        self._c(lib().bx_batch_info(self._h, C.byref(ms), C.byref(nl), C.byref(ns),
                                    C.byref(cells)))
        return dict(last_run_ms=ms.value, launches=nl.value, solo_boxes=ns.value,
                    pool_cells=cells.value)


def wait_selftest(poll_limit: int):
    """The persistent launch's bounded wait on a counter nothing advances: returns
    (gave_up, ms)."""
    g = C.c_int32()
    ms = C.c_double()
    rc = lib().bx_batch_wait_selftest(int(poll_limit), C.byref(g), C.byref(ms))
    if rc:
        raise BoxzyError(rc, lib().bx_batch_last_error(None).decode())
    return bool(g.value), ms.value


def pool_bytes(params_list) -> int:
    """Device bytes a Batch of these boxes allocates (three plane sets)."""
    return sum(3 * 5 * 8 * hp.ngrid for hp in params_list)


__all__ = ["Batch", "pool_bytes", "wait_selftest"]
