"""Track_Radial (simtrack.cpp:21641-21680) on the GPU against the reference's
own Track_Radial (needs a B200 and the compiled reference).  Tolerance as
in test_gpu_parity: 1e-12 relative with the per-coordinate rms floor, exact
loss turn and element."""
import numpy as np
import pytest

from simtrack_b200 import lattices as lt
from simtrack_b200.api import Table, Track_Radial

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def assert_close(g, o, what):
    floor = np.maximum(np.sqrt(np.mean(o * o, axis=0)), 1e-300)
    bad = np.abs(g - o) > RTOL * np.maximum(np.abs(o), floor)
    if bad.any():
        i, k = np.argwhere(bad)[0]
        raise AssertionError(f"{what}: particle {i} coord {k}: gpu {g[i, k]!r} reference {o[i, k]!r}")


@pytest.mark.parametrize("ring,nturn", [("fodo", 400), ("rhic", 60)])
def test_radial_matches_reference(ring, nturn, native_lib, ref_oracle):
    lat = lt.fodo_ring() if ring == "fodo" else lt.rhic_like_ring(seed=1)
    # offset quadrupoles steer the on-momentum reference particle off the
    # design path, so that its per-element path length (x04) is not zero
    for e in lat.elements[3::97]:
        if e.type in ("QUAD", "MULT"):
            e.misalign = (2e-4, -1e-4, 0.0, 0.0, 0.0, 0.0)
    tab = Table(lt.build_line(lat))
    ref_oracle.build(lat)
    rng = np.random.default_rng(7)
    n = 12
    X = np.zeros((n, 6))
    scale = 2e-3 if ring == "fodo" else 6 * lat.meta["sigma_ip"]
    X[:, 0] = rng.uniform(-1, 1, n) * scale
    X[:, 2] = rng.uniform(-1, 1, n) * scale
    X[:, 4] = rng.uniform(-0.05, 0.05, n)
    X[:, 5] = rng.uniform(-8e-4, 8e-4, n)
    X[-1, 0] = 0.15  # rejected by the entry check
    xg, st, ltn, lp = tab.track_radial_host(X.copy(), nturn)
    xo, so, lo, po = ref_oracle.track_radial(X.copy(), nturn)
    assert np.array_equal(st, so) and np.array_equal(ltn, lo) and np.array_equal(lp, po)
    assert_close(xg[st == 1], xo[so == 1], f"{ring} radial")
    # the radial correction is not a no-op here: plain tracking ends elsewhere in z
    xp, _, _, _ = tab.track_host(X.copy(), nturn)
    assert not np.array_equal(xp[st == 1, 4], xg[st == 1, 4])


def test_track_radial_drop_in(native_lib, ref_oracle):
    lat = lt.fodo_ring()
    line = lt.build_line(lat)
    ref_oracle.build(lat)
    x = [1e-3, 0.0, -5e-4, 0.0, 0.01, 3e-4]
    xs = list(x)
    st, ltn, lp = Track_Radial(line, xs, 100)
    xo, so, lo, po = ref_oracle.track_radial(np.array([x]), 100)
    assert (st, ltn, lp) == (so[0], lo[0], po[0])
    assert_close(np.array([xs]), xo, "drop-in")


def test_track_da_reproduces_reference_file(tmp_path, native_lib, ref_oracle):
    """Track_DA's output file (10 angles, twin-particle bisection) equals the
    reference's, byte for byte."""
    from simtrack_b200.api import Track_DA
    lat = lt.rhic_like_ring(seed=1)
    line = lt.build_line(lat)
    ref_oracle.build(lat)
    ours, theirs = tmp_path / "da_gpu.dat", tmp_path / "da_ref.dat"
    sig = lat.meta["sigma_ip"]
    ang, s = Track_DA(line, 64, 5e-4, sig, sig, ours)
    ref_oracle.track_da(64, 5e-4, sig, sig, theirs)
    assert ours.read_text() == theirs.read_text()
    # the bisections end inside the interval, at different amplitudes per angle
    assert np.all(s > 1) and np.all(s < 49) and len(set(s.tolist())) > 3


def test_onmom_dz0_and_tracking_wrt_it(native_lib, ref_oracle):
    """Cal_dz0_OnMomentumPart and Track_wrt_OnMomentumPart (simtrack.cpp:20929,
    20942) on the RHIC-like ring with offset quadrupoles, started from its
    closed orbit: dz0 and the pass's end point equal the reference's, and
    tracking with that dz0 gives the reference's coordinates and losses."""
    from ctypes import POINTER, c_double, c_int
    from simtrack_b200.api import Cal_dz0_OnMomentumPart, Cal_Orbit_Num, Track_wrt_OnMomentumPart
    lat = lt.rhic_like_ring(seed=3)
    rng = np.random.default_rng(11)
    for e in lat.elements:
        if e.type == "QUAD" and rng.random() < 0.1:
            e.misalign = (rng.normal(0, 1e-4), rng.normal(0, 1e-4), 0.0, 0.0, 0.0, 0.0)
    line = lt.build_line(lat)
    x0 = np.zeros(6)
    x0[:4] = Cal_Orbit_Num(line, 0.0)[-1][:4]
    xe, dz0 = Cal_dz0_OnMomentumPart(line, x0)
    ref_oracle.build(lat)
    xr = x0.copy()
    dr = np.empty(len(lat.elements))
    ref_oracle.L.ref_cal_dz0(ref_oracle.line, xr.ctypes.data_as(POINTER(c_double)),
                             dr.ctypes.data_as(POINTER(c_double)))
    assert np.max(np.abs(dz0)) > 0
    assert_close(dz0.reshape(-1, 1), dr.reshape(-1, 1), "dz0")
    assert_close(xe.reshape(1, 6), xr.reshape(1, 6), "end of the pass")
    sig = lat.meta["sigma_ip"]
    X = np.array([[a * sig, 0, 0.6 * a * sig, 0, 0.01, 3e-4] for a in (0.5, 3.0, 8.0, 20.0)])
    nt = 40
    xg, sg, lg, pg = Track_wrt_OnMomentumPart(line, X, dz0, nt)
    xo = X.copy()
    so = np.ones(len(X), dtype=np.int32)
    lo = np.zeros(len(X), dtype=np.int32)
    po = np.zeros(len(X), dtype=np.int32)
    P = lambda a, t: a.ctypes.data_as(POINTER(t))
    ref_oracle.L.ref_track_wrt_onmom(ref_oracle.line, P(xo, c_double), len(X), P(dz0, c_double), nt, P(so, c_int),
                                     P(lo, c_int), P(po, c_int))
    assert np.array_equal(sg, so) and np.array_equal(lg, lo) and np.array_equal(pg, po)
    assert_close(xg, xo, "tracked with dz0")
