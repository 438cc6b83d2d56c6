"""Elementary functions of the tracking maps (stb_crmath.cuh).

The reference calls the host C library's asin/exp/sin/cos/pow.  The kernels
use correctly rounded double-double evaluations instead; these tests check
(CPU) that they are exactly the correctly rounded values, against mpmath at 60
significant digits, on the sampled argument ranges of the maps and on
near-midpoint arguments found by an extended-precision search; that they sit
within 1 ulp of the C library and agree with it on all but a small fraction
of arguments (the C library itself misrounds those, e.g.
exp(-38.706775399911955) is off by 0.50015 ulp in glibc); that the oracle's
independent correctly rounded shim (oracle/crlibm_shim.cpp: x87 extended and
binary128 evaluations, no code shared with the tracker) passes the same
mpmath check; and (GPU) that the device build returns the host build's values
bit for bit.
"""
import ctypes
import math
from ctypes import POINTER, c_double

import mpmath
import numpy as np
import pytest

import oracle_bridge


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
MP_FN = {0: mpmath.asin, 1: mpmath.exp, 2: mpmath.sin, 3: mpmath.cos}
NP_FN = {0: np.arcsin, 1: np.exp, 2: np.sin, 3: np.cos}


def mp_rounded(fn, x, m=None, digits=60):
    """The correctly rounded (nearest, ties to even) double of f(x), or of
    x**m for fn 4, from a `digits`-digit mpmath evaluation."""
    with mpmath.workdps(digits):
        v = mpmath.mpf(float(x)) ** int(m) if fn == 4 else MP_FN[fn](mpmath.mpf(float(x)))
    with mpmath.workprec(53):
        return float(+v)


def near_midpoint(fn, x, keep, m=None):
    """The `keep` arguments of x whose value lies closest to a rounding
    midpoint between two doubles, by an x87 extended-precision evaluation
    (hard cases for a correctly rounded implementation)."""
    xl = x.astype(np.longdouble)
    v = xl ** m.astype(np.longdouble) if fn == 4 else NP_FN[fn](xl)
    d = v.astype(np.float64)
    u = np.spacing(np.abs(d)).astype(np.longdouble)
    frac = (v - d.astype(np.longdouble)) / u
    dist = np.abs(np.abs(frac) - 0.5)
    idx = np.argsort(dist.astype(np.float64))[:keep]
    return idx


def hard_and_sampled(name, fn, seed):
    x = samples(name, 2000, seed=seed)
    pool = samples(name, 400000, seed=seed + 100)
    return np.concatenate([x, pool[near_midpoint(fn, pool, 64)]])


def pown_cases(seed):
    rng = np.random.default_rng(seed)
    h = np.concatenate([rng.random(1500) * 3 + 0.05, 1.0 / (3.2 * rng.random(1500) + 1e-3)])
    m = -rng.integers(6, 30, h.size).astype(np.float64)
    ph = rng.random(400000) * 3 + 0.05
    pm = -rng.integers(6, 30, ph.size).astype(np.float64)
    k = near_midpoint(4, ph, 64, pm)
    return np.concatenate([h, ph[k]]), np.concatenate([m, pm[k]])


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


@pytest.mark.parametrize("name,fn,ref", CASES)
def test_correctly_rounded_vs_mpmath(native_lib, name, fn, ref):
    """The tracker's functions (host build of the device code) are the
    correctly rounded values."""
    x = hard_and_sampled(name, fn, seed=21)
    y = ev(native_lib, fn, x, -1)
    r = np.array([mp_rounded(fn, v) for v in x])
    bad = np.flatnonzero(y != r)
    assert bad.size == 0, f"{name}: {bad.size} misrounded, e.g. x={x[bad[0]]!r}"


def test_pown_correctly_rounded_vs_mpmath(native_lib):
    h, m = pown_cases(22)
    y = ev(native_lib, 4, np.stack([h, m], 1).ravel(), -1)
    r = np.array([mp_rounded(4, a, b) for a, b in zip(h, m)])
    assert np.array_equal(y, r)


def _crshim():
    if not oracle_bridge.ref_available(cr=True):
        pytest.skip("compiled reference oracle with correctly rounded libm (oracle/_ref) not built here")
    lib = ctypes.CDLL(str(oracle_bridge.REF_CR_SO))
    lib.stb_crshim_eval.restype = ctypes.c_double
    lib.stb_crshim_eval.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double]
    lib.stb_crshim_unresolved.restype = ctypes.c_long
    return lib


@pytest.mark.parametrize("name,fn,ref", CASES)
def test_oracle_shim_correctly_rounded_vs_mpmath(name, fn, ref):
    """The correctly rounded oracle's own functions, which share no code with
    the tracker, are the correctly rounded values too."""
    lib = _crshim()
    x = hard_and_sampled(name, fn, seed=31)
    y = np.array([lib.stb_crshim_eval(fn, float(v), 0.0) for v in x])
    r = np.array([mp_rounded(fn, v) for v in x])
    assert np.array_equal(y, r)
    h, m = pown_cases(32)
    y = np.array([lib.stb_crshim_eval(4, float(a), float(b)) for a, b in zip(h, m)])
    assert np.array_equal(y, np.array([mp_rounded(4, a, b) for a, b in zip(h, m)]))
    assert lib.stb_crshim_unresolved() == 0


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


def _drift_check(native_lib, n, seed, device):
    from ctypes import c_ulonglong
    bad = (c_ulonglong * 4)()
    assert native_lib.stb_check_drift_quotients(n, seed, device, bad) == 0
    return list(bad)


def test_drift_quotients_equal_ieee_on_the_host(native_lib):
    """The drift's seeded square root and reciprocal and its quotients
    (stb_physics.cuh drift_quotients), built for the host, against IEEE sqrt
    and division on 4e6 random drift arguments."""
    assert _drift_check(native_lib, 4_000_000, 2024, -1) == [0, 0, 0, 0]


@pytest.mark.gpu
def test_drift_quotients_equal_ieee_on_the_gpu(native_lib):
    """The same on the GPU over 2e9 random drift arguments (device code,
    -fmad=false unit)."""
    for seed in (1, 2):
        assert _drift_check(native_lib, 1_000_000_000, seed, 0) == [0, 0, 0, 0]


def _sincos_check(native_lib, n, seed, device):
    from ctypes import c_ulonglong
    cnt = (c_ulonglong * 4)()
    assert native_lib.stb_check_sincos(n, seed, device, cnt) == 0
    return list(cnt)


def test_sincos_fast_path_equals_series_on_the_host(native_lib):
    """The table-driven fast path of sin/cos (rounding decided by a proven
    error bound) returns the double-double series' values whenever it
    answers, and leaves few arguments to the series (host build)."""
    n = 2_000_000
    ds, dc, slow, slow_near = _sincos_check(native_lib, n, 7, -1)
    assert (ds, dc) == (0, 0)
    assert slow < 1e-3 * n  # expected about 2^-15 of the generic arguments
    assert slow_near < 0.1 * n  # offsets below 2^-34 from k pi/128 always take the series


def test_sincos_table_header_is_current():
    """stb_sincos_table.cuh is what its generator writes (mpmath constants)."""
    import importlib.util
    from pathlib import Path
    csrc = Path(__file__).resolve().parents[1] / "simtrack_b200" / "csrc"
    spec = importlib.util.spec_from_file_location("gen_sincos_table", csrc / "gen_sincos_table.py")
    gen = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gen)
    assert (csrc / "stb_sincos_table.cuh").read_text() == gen.text()


@pytest.mark.gpu
def test_sincos_fast_path_equals_series_on_the_gpu(native_lib):
    """The same on the GPU over 1e9 arguments (device code, -fmad=false unit)."""
    n = 500_000_000
    for seed in (1, 2):
        ds, dc, slow, slow_near = _sincos_check(native_lib, n, seed, 0)
        assert (ds, dc) == (0, 0)
        assert slow < 1e-3 * n
