"""Elementary functions of the tracking maps (stb_crmath.cuh).

The reference calls the host C library's asin/exp/sin/cos/pow.  The kernels
use correctly rounded double-double evaluations instead; these tests check
(CPU) that they sit within 1 ulp of the C library and agree with it on all
but a small fraction of arguments (the C library itself misrounds those,
e.g. exp(-38.706775399911955) is off by 0.50015 ulp in glibc), and (GPU) that
the device build returns the host build's values bit for bit.
"""
import math
from ctypes import POINTER, c_double

import numpy as np
import pytest


def ev(native_lib, fn, x, device):
    x = np.ascontiguousarray(x, dtype=np.float64)
    n = x.size // (2 if fn in (4, 5, 14, 15) else 1)
    out = np.empty(n)
    rc = native_lib.stb_math_eval(fn, x.ctypes.data_as(POINTER(c_double)), out.ctypes.data_as(POINTER(c_double)),
                                  n, device)
    assert rc == 0
    return out


def samples(kind, n, seed=0):
    rng = np.random.default_rng(seed)
    if kind == "asin":  # trajectory slopes inside an aperture
        return (rng.random(n) * 2 - 1) * rng.choice([3e-6, 3e-5, 3e-4, 3e-3, 3e-2], n)
    if kind == "exp":  # beam-beam Gaussian factors: non-positive arguments
        return -rng.random(n) * rng.choice([1e-4, 1e-2, 1.0, 20.0, 300.0], n)
    return (rng.random(n) * 2 - 1) * rng.choice([1e-3, 0.3, 3.3, 40.0], n)  # RF / crab phases


CASES = [("asin", 0, math.asin), ("exp", 1, math.exp), ("sin", 2, math.sin), ("cos", 3, math.cos)]


@pytest.mark.parametrize("name,fn,ref", CASES)
def test_within_one_ulp_of_libm(native_lib, name, fn, ref):
    x = samples(name, 50000)
    y = ev(native_lib, fn, x, -1)
    r = np.array([ref(v) for v in x])
    ulp = np.array([math.ulp(v) for v in r])
    assert np.all(np.abs(y - r) <= ulp)
    assert np.mean(y != r) < 0.005


def test_asin_small_slopes_match_libm(native_lib):
    x = samples("asin", 100000, seed=1)
    x = x[np.abs(x) < 1e-3]
    y = ev(native_lib, 0, x, -1)
    r = np.array([math.asin(v) for v in x])
    assert np.mean(y != r) < 2e-4


def test_integer_power(native_lib):
    rng = np.random.default_rng(2)
    h = rng.random(5000) * 3 + 0.05
    m = -rng.integers(6, 30, 5000).astype(np.float64)
    y = ev(native_lib, 4, np.stack([h, m], 1).ravel(), -1)
    r = np.array([math.pow(a, b) for a, b in zip(h, m)])
    assert np.max(np.abs(y - r) / np.abs(r)) <= 2.3e-16


@pytest.mark.gpu
@pytest.mark.parametrize("name,fn,ref", CASES)
def test_device_equals_host(native_lib, name, fn, ref):
    x = samples(name, 200000, seed=5)
    assert np.array_equal(ev(native_lib, fn, x, 0), ev(native_lib, fn, x, -1))


@pytest.mark.gpu
def test_device_power_equals_host(native_lib):
    rng = np.random.default_rng(3)
    hm = np.stack([rng.random(20000) * 3 + 0.05, -rng.integers(6, 30, 20000).astype(np.float64)], 1).ravel()
    assert np.array_equal(ev(native_lib, 4, hm, 0), ev(native_lib, 4, hm, -1))


@pytest.mark.gpu
def test_shared_reciprocal_quotient_equals_ieee_division(native_lib):
    """qdiv(a, b, RN(1/b)) (Markstein correction) against the IEEE quotient,
    over random operands spanning many binades and significands near 1 and 2."""
    rng = np.random.default_rng(11)
    n = 2_000_000
    a = rng.standard_normal(n) * 10.0 ** rng.integers(-12, 6, n)
    b = (1.0 + rng.random(n)) * 2.0 ** rng.integers(-40, 20, n)
    b[: n // 8] = np.nextafter(2.0, 0.0) * 2.0 ** rng.integers(-10, 10, n // 8)  # significand 1.11..1
    a[n // 8: n // 4] = np.nextafter(1.0, 2.0) * rng.integers(1, 1000, n // 8)
    ab = np.stack([a, b], 1).ravel()
    q = ev(native_lib, 5, ab, 0)
    assert np.array_equal(q, a / b)
    assert np.array_equal(ev(native_lib, 15, ab, 0), a / b)
