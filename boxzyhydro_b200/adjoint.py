"""Discrete adjoint of a run of the hydro step, as a torch.autograd.Function.

`AdjointRun` wraps the bx_adj_* entry points: `forward` advances the reference
cons (a CUDA tensor of shape (5, ngrid), SoA planes rho, m1, m2, m3, E) through
nsteps steps of the fused stage kernels, recording the dt sequence; `backward`
returns the vector-Jacobian product for a given adjoint of the final state,
with that dt sequence and every limiter branch held fixed.  Snapshots follow a
binomial schedule in `snapshots` plane sets.  This module is the only place the
package touches PyTorch.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import BoxzyError, lib, make_params
from .params import HydroParams


class AdjointEngine:
    def __init__(self, params: HydroParams, nsteps: int, snapshots: int):
        params.validate()
        self.params = params
        self.nsteps = int(nsteps)
        p = make_params(params)
        h = C.c_void_p()
        rc = lib().bx_adj_create(C.byref(p), self.nsteps, int(snapshots), C.byref(h))
        if rc:
            raise BoxzyError(rc, lib().bx_adj_last_error(None).decode())
        self._h = h

    def _c(self, rc):
        if rc:
            raise BoxzyError(rc, lib().bx_adj_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None):
            lib().bx_adj_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def keep_stage0(self, enable=True):
        """Keep every step's stage-0 result from the next forward (memory for
        speed: the backward then skips recomputing stage 0)."""
        self._c(lib().bx_adj_keep_stage0(self._h, 1 if enable else 0))

    def stage0_cache(self, entries):
        """Entries of the backward pass's cache of stage-0 results (>= 2)."""
        self._c(lib().bx_adj_stage0_cache(self._h, int(entries)))

    def host_level(self, stride):
        """Copy every stride-th state of the next forward run to pinned host
        memory and reverse the segments between them one by one (0: off).
        Returns the pinned bytes."""
        hb = C.c_int64()
        self._c(lib().bx_adj_host_level(self._h, int(stride), C.byref(hb)))
        return hb.value

    def set_stream(self, ptr):
        self._c(lib().bx_adj_set_stream(self._h, C.c_void_p(ptr) if ptr else None))

    def forward_ptr(self, cons0_ptr, consT_ptr, frozen=False):
        self._c(lib().bx_adj_forward(self._h, C.c_void_p(cons0_ptr), C.c_void_p(consT_ptr),
                                     1 if frozen else 0))

    def forward_branches_ptr(self, base_ptr, pert_ptr, baseT_ptr, pertT_ptr):
        """The last unfrozen forward run from a base and a perturbed initial state,
        the perturbed run taking every branch the base run takes (dt sequence
        held too): a smooth map whose central differences check the backward."""
        self._c(lib().bx_adj_forward_branches(self._h, C.c_void_p(base_ptr), C.c_void_p(pert_ptr),
                                              C.c_void_p(baseT_ptr), C.c_void_p(pertT_ptr)))

    def backward_ptr(self, lamT_ptr, lam0_ptr):
        self._c(lib().bx_adj_backward(self._h, C.c_void_p(lamT_ptr), C.c_void_p(lam0_ptr)))

    def stats(self):
        f, b = C.c_double(), C.c_double()
        r, nb = C.c_int64(), C.c_int64()
        self._c(lib().bx_adj_stats(self._h, C.byref(f), C.byref(b), C.byref(r), C.byref(nb)))
        return dict(ms_forward=f.value, ms_backward=b.value, recomputed_steps=r.value,
                    device_bytes=nb.value)

    def dts(self):
        out = np.empty(self.nsteps)
        self._c(lib().bx_adj_dts(self._h, out.ctypes.data_as(C.POINTER(C.c_double))))
        return out


def plan(nsteps: int, snapshots: int) -> dict:
    """The checkpoint schedule of an nsteps run with `snapshots` plane sets,
    computed on the host (no device): forward steps recomputed by the first
    backward after a forward (`recomputed_first`, what `stats()` reports) and by
    a further backward of the same run (`recomputed_again`), and the snapshots
    the forward run stores on its way (`chain_snapshots`)."""
    first, again = C.c_int64(), C.c_int64()
    chain = C.c_int32()
    rc = lib().bx_adj_plan(int(nsteps), int(snapshots), C.byref(first), C.byref(again),
                           C.byref(chain))
    if rc:
        raise BoxzyError(rc, lib().bx_adj_last_error(None).decode())
    return dict(recomputed_first=first.value, recomputed_again=again.value,
                chain_snapshots=chain.value)


def device_bytes(params: HydroParams, nsteps: int, snapshots: int, stage0_cache: int = 2,
                 keep_stage0: bool = False) -> int:
    """Device bytes of an engine for this grid (what `stats()` reports), computed
    on the host, to size a run to the device before allocating."""
    out = C.c_int64()
    p = make_params(params)
    rc = lib().bx_adj_device_bytes(C.byref(p), int(nsteps), int(snapshots), int(stage0_cache),
                                   1 if keep_stage0 else 0, C.byref(out))
    if rc:
        raise BoxzyError(rc, lib().bx_adj_last_error(None).decode())
    return out.value


def _torch():
    import torch
    return torch


class AdjointRun:
    """cons_T = AdjointRun.apply(cons0, engine): differentiable w.r.t. cons0."""

    @staticmethod
    def apply(cons0, engine):
        return _Fn.apply(cons0, engine)


def _make_fn():
    torch = _torch()

    class Fn(torch.autograd.Function):
        @staticmethod
        def forward(ctx, cons0, engine):
            c0 = cons0.detach().contiguous()
            out = torch.empty_like(c0)
            torch.cuda.synchronize(c0.device)
            engine.forward_ptr(c0.data_ptr(), out.data_ptr(), frozen=False)
            ctx.engine = engine
            return out

        @staticmethod
        def backward(ctx, gT):
            g = gT.detach().contiguous()
            out = torch.empty_like(g)
            torch.cuda.synchronize(g.device)
            ctx.engine.backward_ptr(g.data_ptr(), out.data_ptr())
            return out, None

    return Fn


class _Lazy:
    _fn = None

    def apply(self, *a):
        if _Lazy._fn is None:
            _Lazy._fn = _make_fn()
        return _Lazy._fn.apply(*a)


_Fn = _Lazy()

__all__ = ["AdjointEngine", "AdjointRun"]
