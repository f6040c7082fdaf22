"""The reciprocal-based divisions of the stage kernels equal IEEE division bit for bit.

Each HLL face divides five flux numerators by the same wave-speed sum, and the
lambdas, the update and the Courant rate divide by the cell sizes and volume;
the kernels compute one correctly rounded reciprocal (on the device for the
wave-speed sum, on the host for the grid constants) and correct each quotient
with an FMA residual.  This checks the device implementation against the device's
IEEE double division on random operands (random mantissas and exponents inside
and far outside the window where the short form is used, exact multiples and
near-ties)."""
import ctypes as C

import pytest

from boxzyhydro_b200 import _lib

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("exp_range,seed", [(60, 1), (200, 2), (449, 3), (1000, 4)])
def test_shared_division_is_ieee(exp_range, seed):
    bad = C.c_ulonglong()
    a, d = C.c_double(), C.c_double()
    rc = _lib.lib().bx_check_shared_division(50_000_000, seed, exp_range, C.byref(bad),
                                             C.byref(a), C.byref(d))
    assert rc == 0
    assert bad.value == 0, f"{bad.value} mismatches, e.g. {a.value!r} / {d.value!r}"
