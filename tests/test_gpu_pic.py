"""Strong-strong beam-beam by particle-in-cell, 4D (needs a B200).

BeamBeam4D_PIC (simtrack.cpp:23286-23378) on the GPU (`stb_bb4d_pic_*`,
stb_pic.cu) against the reference's own function called through the oracle
harness, on the same two macro-particle beams: round and flat beams, offset
centroids, unequal populations and charges (bbscale), halo particles outside
the 29-cell cut, and a two-particle beam.  The charge sums keep the
reference's per-cell order of additions, the FFTs its butterflies and
twiddles, and the Green function its C-library atan and log, so the kicked
beams are expected bit for bit against the reference as compiled here.
"""
from ctypes import POINTER, c_double

import numpy as np
import pytest

import oracle_bridge
from simtrack_b200 import api
from simtrack_b200._native import SimTrackError
from test_gpu_strong_strong import GAMMA, _beam

pytestmark = pytest.mark.gpu

CASES = [
    # (n1, sx1, sy1, n2, sx2, sy2, offset, Np1, Np2, bbscale1, bbscale2)
    (4000, 1.2e-4, 1.2e-4, 5000, 1.2e-4, 1.2e-4, (0.0, 0.0), 2e11, 2.2e11, 1.0, 1.0),
    (3000, 1.2e-4, 1.2e-4, 3000, 1.1e-4, 1.3e-4, (2e-5, -1e-5), 2e11, 2e11, 1.0, 1.0),
    (2500, 9.5e-5, 8.5e-6, 4000, 9.5e-5, 8.5e-6, (1e-6, 3e-7), 1.7e11, 1.1e11, -1.0, -1.0),
    (2, 1.0e-4, 1.0e-4, 2000, 1.0e-4, 5.0e-5, (0.0, 0.0), 1e11, 1e11, 1.0, 0.5),
    (200_000, 1.0e-4, 6.0e-5, 150_000, 1.1e-4, 5.5e-5, (3e-6, -2e-6), 1.5e11, 1.3e11, 1.0, 1.0),
]


def _need_ref():
    if not oracle_bridge.ref_available():
        pytest.skip("compiled reference oracle (oracle/_ref) not built here")


def _theirs(b1, b2, Np1, Np2, s1, s2):
    b1, b2 = b1.copy(), b2.copy()
    P = lambda a: a.ctypes.data_as(POINTER(c_double))
    ref = oracle_bridge.RefOracle()
    ref.L.ref_bb4d_pic(Np1, len(b1), P(b1), Np2, len(b2), P(b2), GAMMA, GAMMA, s1, s2)
    return b1, b2


@pytest.mark.parametrize("case", CASES)
def test_pic_4d_vs_reference(case):
    _need_ref()
    n1, sx1, sy1, n2, sx2, sy2, (dx, dy), Np1, Np2, s1, s2 = case
    b1 = _beam(n1, sx1, sy1, 0.0, 0.0, 1)
    b2 = _beam(n2, sx2, sy2, dx, dy, 2)
    if n1 > 100:
        b1[7, 0] += 40 * sx1  # halo particles: outside the cut, neither deposit nor get kicked
        b2[11, 2] -= 40 * sy2
    o1, o2 = b1.copy(), b2.copy()
    api.BeamBeam4D_PIC(Np1, o1, Np2, o2, GAMMA, GAMMA, s1, s2)
    r1, r2 = _theirs(b1, b2, Np1, Np2, s1, s2)
    assert np.array_equal(o1, r1) and np.array_equal(o2, r2)
    if n1 > 100:  # (a two-particle beam sets a narrow grid: most of the other beam is outside the cut)
        moved = (o1[:, 1] != b1[:, 1]).sum() + (o2[:, 1] != b2[:, 1]).sum()
        assert moved > 0.9 * (n1 + n2)
        assert o1[7, 1] == b1[7, 1] and o2[11, 3] == b2[11, 3]
    for k in (0, 2, 4, 5):  # only px and py change
        assert np.array_equal(o1[:, k], b1[:, k]) and np.array_equal(o2[:, k], b2[:, k])


def test_repeated_device_collisions_vs_reference(native_lib):
    """Three collisions in a row on device-resident beams (the _device form)."""
    import torch
    _need_ref()
    b1 = _beam(20_000, 1.0e-4, 1.0e-4, 0.0, 0.0, 5)
    b2 = _beam(30_000, 1.1e-4, 0.9e-4, 1e-5, 0.0, 6)
    d1 = torch.tensor(b1, device="cuda:0")
    d2 = torch.tensor(b2, device="cuda:0")
    r1, r2 = b1.copy(), b2.copy()
    for _ in range(3):
        assert native_lib.stb_bb4d_pic_device(2e11, len(b1), d1.data_ptr(), 2e11, len(b2), d2.data_ptr(), GAMMA,
                                              GAMMA, 1.0, 1.0, 0, None) == 0
        r1, r2 = _theirs(r1, r2, 2e11, 2e11, 1.0, 1.0)
    torch.cuda.synchronize()
    assert np.array_equal(d1.cpu().numpy(), r1) and np.array_equal(d2.cpu().numpy(), r2)


def test_rejected_inputs():
    b1 = _beam(100, 1e-4, 1e-4, 0, 0, 1)
    b2 = _beam(100, 1e-4, 1e-4, 0, 0, 2)
    with pytest.raises(SimTrackError):
        api.BeamBeam4D_PIC(1e11, b1[:1].copy(), 1e11, b2, GAMMA, GAMMA, 1.0, 1.0)
    with pytest.raises(SimTrackError):
        api.BeamBeam4D_PIC(1e11, b1, 1e11, b2, -1.0, GAMMA, 1.0, 1.0)
    # a NaN coordinate makes the grid spacing NaN: every cut test fails, so
    # no particle deposits or moves, as in the reference
    bad, o2 = b1.copy(), b2.copy()
    bad[3, 0] = np.nan
    o1 = bad.copy()
    api.BeamBeam4D_PIC(1e11, o1, 1e11, o2, GAMMA, GAMMA, 1.0, 1.0)
    assert np.array_equal(o1, bad, equal_nan=True) and np.array_equal(o2, b2)


LUMI_CASES = [
    # (n1, sx1, sy1, n2, sx2, sy2, offset, Ncoll)
    (4000, 1.2e-4, 1.2e-4, 5000, 1.2e-4, 1.2e-4, (0.0, 0.0), 1),
    (3000, 9.5e-5, 8.5e-6, 3500, 9.5e-5, 8.5e-6, (2e-5, 1e-6), 2),
    (1, 1.0e-4, 1.0e-4, 2000, 1.0e-4, 5.0e-5, (0.0, 0.0), 1),
    (150_000, 1.0e-4, 6.0e-5, 200_000, 1.1e-4, 5.5e-5, (3e-6, -2e-6), 3),
]


@pytest.mark.parametrize("case", LUMI_CASES)
def test_lumi_pic_4d_vs_reference(case):
    """Lumi_Cal_PIC_4D (simtrack.cpp:23617-23701): the charge overlap on the
    beams' joint grid, bit for bit (halo particles widen the grid)."""
    _need_ref()
    n1, sx1, sy1, n2, sx2, sy2, (dx, dy), ncoll = case
    b1 = _beam(n1, sx1, sy1, 0.0, 0.0, 3)
    b2 = _beam(n2, sx2, sy2, dx, dy, 4)
    if n2 > 100:
        b2[5, 0] += 12 * sx2
    P = lambda a: a.ctypes.data_as(POINTER(c_double))
    ours = api.Lumi_Cal_PIC_4D(1.1e11, b1, 1.2e11, b2, ncoll, 78196.0)
    ref = oracle_bridge.RefOracle()
    theirs = ref.L.ref_lumi_pic_4d(1.1e11, n1, 1.2e11, n2, P(b1.copy()), P(b2.copy()), ncoll, 78196.0)
    assert ours == theirs and ours > 0


def test_lumi_rejected_inputs():
    b = _beam(100, 1e-4, 1e-4, 0, 0, 1)
    flat = b.copy()
    flat[:, 2] = 0.0
    with pytest.raises(SimTrackError):  # no extent in y
        api.Lumi_Cal_PIC_4D(1e11, flat, 1e11, flat.copy(), 1, 1e4)
    bad = b.copy()
    bad[4, 2] = np.inf
    with pytest.raises(SimTrackError):
        api.Lumi_Cal_PIC_4D(1e11, bad, 1e11, b, 1, 1e4)


def _green(nx, hx, hy, xoff=0.0, yoff=0.0, ours=True):
    gr, gi = np.empty(4 * nx * nx), np.empty(4 * nx * nx)
    P = lambda a: a.ctypes.data_as(POINTER(c_double))
    if ours:
        from simtrack_b200._native import lib
        assert lib().stb_pic_green_function(xoff, yoff, nx, nx, hx, hy, P(gr), P(gi), 0) == 0
    else:
        oracle_bridge.RefOracle().L.ref_green_function(xoff, yoff, nx, nx, hx, hy, P(gr), P(gi))
    return gr, gi


@pytest.mark.parametrize("nx,xoff,yoff", [(8, 0.0, 0.0), (32, 1e-5, -2e-5), (64, 0.0, 0.0), (128, -3e-6, 4e-6)])
def test_green_function_vs_reference(nx, xoff, yoff):
    """Cal_Effective_Green_Function (simtrack.cpp:2881-2921): the host table
    and the GPU transform equal the reference's, bit for bit."""
    _need_ref()
    hx, hy = 15 * 1e-4 / nx, 15 * 6e-5 / nx
    ours = _green(nx, hx, hy, xoff, yoff)
    theirs = _green(nx, hx, hy, xoff, yoff, ours=False)
    assert np.array_equal(ours[0], theirs[0]) and np.array_equal(ours[1], theirs[1])


@pytest.mark.parametrize("nx,n1,n2", [(64, 4000, 5000), (128, 30_000, 20_000), (32, 2, 3000)])
def test_pic_nonoffset_vs_reference(nx, n1, n2):
    """BeamBeam4D_PIC_NonOffset (simtrack.cpp:24226-24280) with the
    reference's own Green spectrum on the caller's grid, bit for bit."""
    _need_ref()
    hx, hy = 15 * 1e-4 / nx, 15 * 6e-5 / nx
    gr, gi = _green(nx, hx, hy, ours=False)
    b1 = _beam(n1, 1e-4, 6e-5, 0.0, 0.0, 7)
    b2 = _beam(n2, 1.1e-4, 5.5e-5, 2e-6, -1e-6, 8)
    if n2 > 100:
        b2[9, 0] = 0.6 * nx * hx  # outside the cut
    P = lambda a: a.ctypes.data_as(POINTER(c_double))
    o1, o2 = b1.copy(), b2.copy()
    from simtrack_b200._native import lib
    assert lib().stb_bb4d_pic_nonoffset_host(1.5e11, n1, P(o1), 1.3e11, n2, P(o2), GAMMA, GAMMA, 1.0, -1.0, nx, nx,
                                             hx, hy, P(gr), P(gi), 0) == 0
    r1, r2 = b1.copy(), b2.copy()
    oracle_bridge.RefOracle().L.ref_bb4d_pic_nonoffset(1.5e11, n1, P(r1), 1.3e11, n2, P(r2), GAMMA, GAMMA, 1.0, -1.0,
                                                       nx, nx, hx, hy, P(gr), P(gi))
    assert np.array_equal(o1, r1) and np.array_equal(o2, r2)
    assert (o2[:, 1] != b2[:, 1]).sum() > 0.9 * n2
    if n2 > 100:
        assert o2[9, 1] == b2[9, 1]


def test_pic_grid_rejections():
    from simtrack_b200._native import lib
    gr, gi = np.empty(4 * 48 * 48), np.empty(4 * 48 * 48)
    P = lambda a: a.ctypes.data_as(POINTER(c_double))
    assert lib().stb_pic_green_function(0.0, 0.0, 48, 48, 1e-5, 1e-5, P(gr), P(gi), 0) != 0  # not a power of two
    assert lib().stb_pic_green_function(0.0, 0.0, 32, 64, 1e-5, 1e-5, P(gr), P(gi), 0) != 0  # not square
    assert lib().stb_pic_green_function(0.0, 0.0, 1024, 1024, 1e-5, 1e-5, P(gr), P(gi), 0) != 0  # above 512


@pytest.mark.parametrize("case", [(3000, 2600, 4, 3, 1.0, 1.0), (2001, 2003, 3, 3, -1.0, 0.5)])
def test_pic_6d_vs_reference(case, tmp_path, monkeypatch):
    """BeamBeam6D_PIC (simtrack.cpp:23380-23615): z sort, slices, collision
    order, drift, 4D PIC per slice pair, drift back; bit for bit (bunch
    sizes that leave uncollided remainders in the second case)."""
    _need_ref()
    monkeypatch.chdir(tmp_path)  # the reference writes its bunches and slices to ./bunch*.dat
    Mp1, Mp2, ns1, ns2, s1, s2 = case
    b1 = _beam(Mp1, 1.2e-4, 1.0e-4, 0.0, 0.0, 11)
    b2 = _beam(Mp2, 1.1e-4, 1.1e-4, 1e-5, -5e-6, 12)
    o1, o2 = b1.copy(), b2.copy()
    api.BeamBeam6D_PIC(2e11, o1, 1.8e11, o2, GAMMA, GAMMA, s1, s2, ns1, ns2)
    P = lambda a: a.ctypes.data_as(POINTER(c_double))
    r1, r2 = b1.copy(), b2.copy()
    oracle_bridge.RefOracle().L.ref_bb6d_pic(2e11, Mp1, P(r1), 1.8e11, Mp2, P(r2), GAMMA, GAMMA, s1, s2, ns1, ns2)
    assert np.array_equal(o1, r1) and np.array_equal(o2, r2)
    assert (np.sort(o1[:, 4]) == np.sort(b1[:, 4])).all() and (o1[:-1, 4] >= o1[1:, 4]).all()


@pytest.mark.parametrize("case", [(3000, 2600, 4, 3, 1.0, 1.0, 2), (2001, 2003, 3, 3, -1.0, 0.5, 1)])
def test_lumi_pic_6d_vs_reference(case, tmp_path, monkeypatch):
    """Lumi_Cal_PIC_6D (simtrack.cpp:23703-23944): the summed slice-pair
    luminosities and the bunches after the soft-Gaussian passes, bit for bit."""
    _need_ref()
    monkeypatch.chdir(tmp_path)  # the reference writes ./collide_order.dat
    Mp1, Mp2, ns1, ns2, s1, s2, ncoll = case
    b1 = _beam(Mp1, 1.2e-4, 1.0e-4, 0.0, 0.0, 13)
    b2 = _beam(Mp2, 1.1e-4, 1.1e-4, 1e-5, -5e-6, 14)
    o1, o2 = b1.copy(), b2.copy()
    ours = api.Lumi_Cal_PIC_6D(2e11, o1, 1.8e11, o2, ns1, ns2, GAMMA, GAMMA, s1, s2, ncoll, 78196.0)
    P = lambda a: a.ctypes.data_as(POINTER(c_double))
    r1, r2 = b1.copy(), b2.copy()
    theirs = oracle_bridge.RefOracle(cr=True).L.ref_lumi_pic_6d(2e11, Mp1, 1.8e11, Mp2, ns1, ns2, P(r1), P(r2),
                                                                GAMMA, GAMMA, s1, s2, ncoll, 78196.0)
    assert ours == theirs and ours > 0
    assert np.array_equal(o1, r1) and np.array_equal(o2, r2)


def test_pic_6d_nonoffset_vs_reference():
    """BeamBeam6D_PIC_NonOffset (simtrack.cpp:24282-24432): slices by
    boundary, particles in place, each slice pair colliding as the 4D
    non-offset PIC with N scaled by the slice's share; bit for bit, with the
    reference's own Green spectrum."""
    _need_ref()
    Mp1, Mp2, ns, nx = 4000, 3600, 5, 64
    b1 = _beam(Mp1, 1.2e-4, 1.0e-4, 0.0, 0.0, 21)
    b2 = _beam(Mp2, 1.1e-4, 1.1e-4, 1e-5, -5e-6, 22)
    zb1 = np.array([1.0, 0.1, 0.03, -0.03, -0.1, -1.0])
    zb2 = np.array([1.0, 0.12, 0.02, -0.04, -0.11, -1.0])
    hx, hy = 15 * 1.1e-4 / nx, 15 * 1.0e-4 / nx
    gr, gi = _green(nx, hx, hy, ours=False)
    P = lambda a: a.ctypes.data_as(POINTER(c_double))
    from simtrack_b200._native import lib
    o1, o2 = b1.copy(), b2.copy()
    assert lib().stb_bb6d_pic_nonoffset_host(2e11, Mp1, P(o1), 1.8e11, Mp2, P(o2), GAMMA, GAMMA, 1.0, 1.0, ns, ns,
                                             P(zb1), P(zb2), nx, nx, hx, hy, P(gr), P(gi), 0) == 0
    r1, r2 = b1.copy(), b2.copy()
    oracle_bridge.RefOracle().L.ref_bb6d_pic_nonoffset(2e11, Mp1, P(r1), 1.8e11, Mp2, P(r2), GAMMA, GAMMA, 1.0, 1.0,
                                                       ns, ns, P(zb1.copy()), P(zb2.copy()), nx, nx, hx, hy, P(gr),
                                                       P(gi))
    assert np.array_equal(o1, r1) and np.array_equal(o2, r2)
    assert np.array_equal(o1[:, 4], b1[:, 4])  # particles stay in place
    assert (o1[:, 1] != b1[:, 1]).sum() > 0.9 * Mp1


@pytest.mark.parametrize("theta", [0.0, 0.0125])
def test_lumi_pic_6d_angle_vs_reference(theta, tmp_path, monkeypatch):
    """Lumi_Cal_PIC_6D_Angle (simtrack.cpp:23946-24224): the Lorentz boost
    of both bunches to the head-on frame, then the sliced luminosity; the
    luminosity and the (boosted) bunches bit for bit."""
    _need_ref()
    monkeypatch.chdir(tmp_path)  # the reference writes its bunches, slices and collision order
    Mp1, Mp2, ns1, ns2 = 2400, 2000, 3, 4
    b1 = _beam(Mp1, 1.2e-4, 1.0e-4, 0.0, 0.0, 31)
    b2 = _beam(Mp2, 1.1e-4, 1.1e-4, 1e-5, -5e-6, 32)
    P = lambda a: a.ctypes.data_as(POINTER(c_double))
    from ctypes import byref
    from simtrack_b200._native import lib
    o1, o2 = b1.copy(), b2.copy()
    lumi = c_double()
    assert lib().stb_lumi_pic_6d_angle_host(2e11, Mp1, 1.8e11, Mp2, theta, ns1, ns2, P(o1), P(o2), GAMMA, GAMMA, 1.0,
                                            1.0, 1, 78196.0, 0, byref(lumi)) == 0
    r1, r2 = b1.copy(), b2.copy()
    theirs = oracle_bridge.RefOracle(cr=True).L.ref_lumi_pic_6d_angle(2e11, Mp1, 1.8e11, Mp2, theta, ns1, ns2, P(r1),
                                                                      P(r2), GAMMA, GAMMA, 1.0, 1.0, 1, 78196.0)
    assert lumi.value == theirs and theirs > 0
    assert np.array_equal(o1, r1) and np.array_equal(o2, r2)


def test_pic_6d_interpolation_vs_reference():
    """BeamBeam6D_PIC_Interpolation (simtrack.cpp:24434-24700): per slice
    pair, two potentials at the front and back of the other slice, the field
    interpolated in s at each particle's own collision point; bit for bit with
    the reference's own Green spectrum."""
    _need_ref()
    Mp1, Mp2, ns, nx = 4000, 3600, 5, 64
    b1 = _beam(Mp1, 1.2e-4, 1.0e-4, 0.0, 0.0, 41)
    b2 = _beam(Mp2, 1.1e-4, 1.1e-4, 1e-5, -5e-6, 42)
    zb1 = np.array([1.0, 0.1, 0.03, -0.03, -0.1, -1.0])
    zb2 = np.array([1.0, 0.12, 0.02, -0.04, -0.11, -1.0])
    hx, hy = 15 * 1.1e-4 / nx, 15 * 1.0e-4 / nx
    gr, gi = _green(nx, hx, hy, ours=False)
    P = lambda a: a.ctypes.data_as(POINTER(c_double))
    from simtrack_b200._native import lib
    o1, o2 = b1.copy(), b2.copy()
    assert lib().stb_bb6d_pic_interpolation_host(2e11, Mp1, P(o1), 1.8e11, Mp2, P(o2), GAMMA, GAMMA, 1.0, 1.0, ns,
                                                 ns, P(zb1), P(zb2), nx, nx, hx, hy, P(gr), P(gi), 0) == 0
    r1, r2 = b1.copy(), b2.copy()
    oracle_bridge.RefOracle().L.ref_bb6d_pic_interpolation(2e11, Mp1, P(r1), 1.8e11, Mp2, P(r2), GAMMA, GAMMA, 1.0,
                                                           1.0, ns, ns, P(zb1.copy()), P(zb2.copy()), nx, nx, hx, hy,
                                                           P(gr), P(gi))
    assert np.array_equal(o1, r1) and np.array_equal(o2, r2)
    assert (o1[:, 1] != b1[:, 1]).sum() > 0.9 * Mp1
