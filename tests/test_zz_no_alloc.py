"""The ghost sweep that allocates nothing (bx_ghost_fill_noalloc) against bx_ghost.

Callers that cannot allocate device memory -- a host program that has reserved
the device's memory for its own pool, or a runtime held to a fixed memory
budget -- use bx_ghost_fill_noalloc, which keeps its gather scratch in a static
device array inside the library.  This test gives it device memory owned by
the test (torch tensors), calls it twice in a row through the C ABI, and
requires after each call exactly the planes that the handle-based bx_ghost
produces after the same number of sweeps (the suite's tolerance is zero).  The
grid has reflective walls on five sides and nz >= 6, so some ghosts read other
ghosts' values from before the sweep and the gather/scatter order matters.

The file name sorts last so that a run stopping at the first failure has run
every other test before this one.
"""
import ctypes as C

import numpy as np
import pytest

from boxzyhydro_b200 import _lib
from boxzyhydro_b200.hydro import Hydro, ghost_plan
from tests.helpers import small_random_box

pytestmark = pytest.mark.gpu


def _soa(cons):
    return np.ascontiguousarray(cons.T)


def test_noalloc_ghost_sweep_matches_bx_ghost_twice():
    import torch

    st = small_random_box(nx=37, ny=21, nz=13, walls=(1, 1, 1, 0, 1, 1), seed=21)
    hp = st.params
    ng = hp.ngrid

    # expected: the handle-based sweep, once and twice
    g = Hydro(hp)
    g.upload(st.cons, st.u, st.p)
    g.set_ghost_cells()
    want1 = g.download()[0]
    g.set_ghost_cells()
    want2 = g.download()[0]
    g.close()
    assert not np.array_equal(want1, st.cons)

    plan = ghost_plan(hp)
    nghost = len(plan["dst"])
    assert nghost <= 1048576
    dev = torch.device("cuda", 0)
    cons = torch.from_numpy(_soa(st.cons)).to(dev)
    dst = torch.from_numpy(plan["dst"]).to(dev)
    src = torch.from_numpy(plan["src1"]).to(dev)
    sgn = torch.from_numpy(plan["sgn1"]).to(dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    torch.cuda.synchronize(dev)

    L = _lib.lib()
    for want in (want1, want2):
        rc = L.bx_ghost_fill_noalloc(C.c_void_p(cons.data_ptr()), ng, C.c_void_p(dst.data_ptr()),
                                     C.c_void_p(src.data_ptr()), C.c_void_p(sgn.data_ptr()),
                                     nghost, C.c_void_p(stream))
        assert rc == 0, L.bx_noalloc_last_error()
        torch.cuda.synchronize(dev)
        got = cons.cpu().numpy().T
        assert np.array_equal(got, want)


def test_noalloc_rejects_too_many_ghosts():
    L = _lib.lib()
    rc = L.bx_ghost_fill_noalloc(None, 10, None, None, None, 1048577, None)
    assert rc == 1
    assert b"BX_NOALLOC_MAX_GHOSTS" in L.bx_noalloc_last_error()
