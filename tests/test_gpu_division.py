"""The stencils' division (Newton-Raphson refinement of a reciprocal
estimate) against IEEE binary64 division: within 1 ulp over random operands
spanning the magnitudes the kernels divide by, and IEEE results for the
special denominators it hands to the hardware division."""
import ctypes as C

import numpy as np
import pytest

from orctm_b200 import _lib

pytestmark = pytest.mark.gpu
_D = C.POINTER(C.c_double)


def _div(a, b):
    lib = _lib.load()
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    q = np.empty_like(a)
    _lib.check(lib.orctm_check_division(0, a.ctypes.data_as(_D), b.ctypes.data_as(_D),
                                        q.ctypes.data_as(_D), a.size))
    return q


def test_within_one_ulp_of_ieee():
    g = np.random.Generator(np.random.PCG64(20261203))
    n = 1 << 20
    a = g.standard_normal(n) * 10.0 ** g.uniform(-30, 30, n)
    b = np.abs(g.standard_normal(n)) * 10.0 ** g.uniform(-25, 25, n) + 1e-20
    b[: n // 4] *= -1.0
    q = _div(a, b)
    ref = a / b
    ulp = np.abs(np.spacing(ref))
    err = np.abs(q - ref) / ulp
    assert err.max() <= 1.0, err.max()
    # almost always correctly rounded
    assert (q == ref).mean() > 0.99


def test_special_denominators_take_ieee_division():
    a = np.array([1.0, -2.0, 0.0, 3.0, 1.0, 5.0])
    b = np.array([0.0, 0.0, 0.0, np.inf, 1e-310, np.nan])
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        ref = a / b
    q = _div(a, b)
    assert np.array_equal(np.isnan(q), np.isnan(ref))
    m = ~np.isnan(ref)
    assert np.array_equal(q[m], ref[m])
