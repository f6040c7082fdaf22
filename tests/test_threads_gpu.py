"""Handles made and stepped from two host threads at once.

The stage kernels need a dynamic shared-memory limit above the default, an
attribute the CUDA runtime holds per device; the library sets it once per
kernel and device under a lock.  This test runs in a fresh process, so the
two threads are the first to launch those kernels: both must get the same
result as the oracle, bit for bit."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import sys, threading
sys.path[:0] = [ROOT, ROOT + "/oracle"]
import numpy as np
import oracle as O
from boxzyhydro_b200.hydro import Hydro
from tests.helpers import small_random_box

st = small_random_box(nx=40, ny=20, nz=18, walls=(0,) * 6, seed=21)
out, errs = {}, []
go = threading.Barrier(2)

def work(k):
    try:
        g = Hydro(st.params)
        g.upload(st.cons, st.u, st.p)
        go.wait()
        for _ in range(5):
            assert g.step()
        out[k] = (g.download(), g.status()[1])
        g.close()
    except Exception as e:
        errs.append(repr(e))

ts = [threading.Thread(target=work, args=(k,)) for k in range(2)]
for t in ts: t.start()
for t in ts: t.join()
assert not errs, errs
o = O.Oracle(st.params)
o.set_state(st.cons, st.u, st.p, st.adindx)
for _ in range(5):
    assert o.step()
c0, u0, p0, _ = o.get_state()
for k in range(2):
    (c, u, p), path = out[k]
    assert path == 1, "expected the fused stage kernels"
    assert np.array_equal(c, c0) and np.array_equal(u, u0) and np.array_equal(p, p0), k
print("threads ok")
"""


def test_two_host_threads_create_and_step_handles():
    code = CHILD.replace("ROOT", repr(ROOT))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                       timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "threads ok" in r.stdout
