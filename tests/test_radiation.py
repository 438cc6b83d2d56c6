"""Quantum-excitation deviate stream of the radiating bends (stb_rng.cuh), CPU.

The reference draws radiate1's normal deviates (simtrack.cpp:4275) from GSL,
which is absent here; tracker and oracle both use a per-particle
counter-based stream instead (Philox4x32-10 + Box-Muller).  These tests pin
the generator to the published Philox known-answer vectors, check that the
tracker's host build and the oracle's independent restatement
(oracle/ref_harness.cpp) give the same deviates bit for bit, and check the
first moments and tail fraction of the distribution.
"""
import ctypes

import numpy as np
import pytest

import oracle_bridge

# Philox4x32-10 known-answer vectors (Random123 kat_vectors): counter, key, output.
KAT = [
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


def normals(native_lib, seed, pid, k0, n, device=-1):
    out = np.empty(n)
    rc = native_lib.stb_rad_normals(seed, pid, k0, n, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), device)
    assert rc == 0
    return out


@pytest.mark.parametrize("ctr,key,want", KAT)
def test_philox_known_answers(native_lib, ctr, key, want):
    c = (ctypes.c_uint * 4)(*ctr)
    k = (ctypes.c_uint * 2)(*key)
    o = (ctypes.c_uint * 4)()
    assert native_lib.stb_philox4x32_10(c, k, o) == 0
    assert tuple(o) == want


def test_stream_equals_oracle_restatement(native_lib):
    """The tracker's deviates equal the oracle harness's own restatement of
    the stream (correctly rounded cos in libsimtrack_ref_cr)."""
    if not oracle_bridge.ref_available(cr=True):
        pytest.skip("compiled reference oracle (oracle/_ref) not built here")
    ref = oracle_bridge.RefOracle(cr=True)
    for seed, pid, k0 in ((1324, 0, 0), (1324, 77, 1000), (2**40 + 5, 2**33 + 1, 2**35)):
        ours = normals(native_lib, seed, pid, k0, 4000)
        theirs = np.array([ref.L.ref_rng_stream(seed, pid, k0 + k) for k in range(4000)])
        assert np.array_equal(ours, theirs)


def test_stream_moments(native_lib):
    n = 1_000_000
    g = np.concatenate([normals(native_lib, 1324, pid, 0, n // 4) for pid in range(4)])
    assert np.all(np.isfinite(g))
    assert abs(g.mean()) < 4.0 / np.sqrt(n)
    assert abs(g.var() - 1.0) < 6.0 * np.sqrt(2.0 / n)
    tail = np.mean(np.abs(g) > 3.0)
    assert abs(tail - 0.0026998) < 5.0 * np.sqrt(0.0027 / n)
    # different particles and different draws are uncorrelated
    a, b = normals(native_lib, 1324, 5, 0, 100000), normals(native_lib, 1324, 6, 0, 100000)
    assert abs(np.corrcoef(a, b)[0, 1]) < 0.02
    assert abs(np.corrcoef(a[:-1], a[1:])[0, 1]) < 0.02


@pytest.mark.parametrize("gsbend", [False, True])
@pytest.mark.parametrize("track_form", [0, 1])
def test_srloss_u0rad_vs_reference(native_lib, gsbend, track_form):
    """Cal_SRLoss_U0rad / Cal_SRLoss_U0rad_Track (simtrack.cpp:20691-20766):
    the reference particle's radiation loss per turn, host computation,
    against the reference's own functions on the electron ring (sector
    dipoles or GSBENDs; the bends' paths on the stored orbit, zero here)."""
    from ctypes import byref, c_double
    from simtrack_b200 import api
    from simtrack_b200 import lattices as lt
    if not oracle_bridge.ref_available():
        pytest.skip("compiled reference oracle (oracle/_ref) not built here")
    lat = lt.electron_ring(gsbend=gsbend)
    try:
        line = lt.build_line(lat)
        u = c_double()
        assert native_lib.stb_cal_srloss_u0rad(line._h, track_form, byref(u)) == 0
        ref = oracle_bridge.RefOracle()
        ref.build(lat)
        assert u.value == ref.L.ref_cal_srloss(ref.line, track_form)
        assert u.value > 0.1  # MeV per turn for 3 GeV electrons in a 276 m ring
        api.Set_Radiation(False)
        assert native_lib.stb_cal_srloss_u0rad(line._h, track_form, byref(u)) == 0 and u.value == 0.0
    finally:
        api.Set_Radiation(False)
        oracle_bridge.reference_radiation_off()
