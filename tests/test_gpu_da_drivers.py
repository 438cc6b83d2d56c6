"""The reference's other dynamic-aperture drivers and Cal_Tunes_Track on the
GPU (needs a B200), against the compiled reference on the RHIC-like ring:

* Track_DA1, Track_DA2, Track_DA3, Track_DA_Radial (simtrack.cpp:21443-21734):
  the output files byte for byte (the reference's own drivers write theirs);
* Track_DA_Uniform, Track_DA_Radial_Uniform (21574, 21736): the file written
  up to the first loss equals the lines the reference's Track() /
  Track_Radial() outcomes give (the reference's sweep ends the process at
  that loss, so it is restated here rather than called);
* Cal_Tunes_Track (20971-21025): tunes within 1e-9 of the reference's
  FineTuneFinder on the reference's own turn-by-turn record."""
import math

import numpy as np
import pytest

from simtrack_b200 import api
from simtrack_b200 import lattices as lt

pytestmark = pytest.mark.gpu

NTURN = 64
DELTAP = 5e-4


@pytest.fixture(scope="module")
def ring():
    lat = lt.rhic_like_ring(seed=1)
    return lat, lt.build_line(lat)


@pytest.mark.parametrize("name,which", [("Track_DA1", 1), ("Track_DA2", 2), ("Track_DA3", 3),
                                        ("Track_DA_Radial", 4)])
def test_bisection_driver_file(name, which, ring, tmp_path, native_lib, ref_oracle):
    lat, line = ring
    lat.set_reference()
    ref_oracle.build(lat)
    s = lat.meta["sigma_ip"]
    ours, theirs = tmp_path / "gpu.dat", tmp_path / "ref.dat"
    ang, sig = api.Track_DA_driver(name, line, NTURN, DELTAP, s, s, filename=ours)
    ref_oracle.L.ref_track_da_driver(ref_oracle.line, which, NTURN, DELTAP, s, s, str(theirs).encode())
    assert ours.read_text() == theirs.read_text()
    assert len(ang) == (5 if which in (1, 3) else 10)
    assert len(set(sig.tolist())) > 2  # the bisections end at different amplitudes


@pytest.mark.parametrize("name,radial", [("Track_DA_Uniform", False), ("Track_DA_Radial_Uniform", True)])
def test_uniform_driver_file(name, radial, ring, tmp_path, native_lib, ref_oracle):
    lat, line = ring
    lat.set_reference()
    ref_oracle.build(lat)
    s, angle = lat.meta["sigma_ip"], 0.7
    path = tmp_path / "gpu.dat"
    flags, sig = api.Track_DA_driver(name, line, NTURN, DELTAP, s, s, angle=angle, filename=path)
    amps = [1. + i * 0.2 for i in range(150)]
    X = np.array([[a * math.cos(angle) * s, 0., a * math.sin(angle) * s, 0., 0., DELTAP] for a in amps])
    if radial:
        _, st, _, _ = ref_oracle.track_radial(X.copy(), NTURN)
    else:
        _, st, _, _ = ref_oracle.track(X.copy(), NTURN, radius=0.0)
    lines = []
    for a, ok in zip(amps, st):
        lines.append("%f %f %f \n" % (angle, a, 1.0 * ok))
        if ok == 0:
            break
    assert st.min() == 0 and len(lines) < 150  # the sweep reaches a loss
    assert path.read_text() == "".join(lines)
    assert len(sig) == len(lines) and flags[-1] == 0.0


def test_cal_tunes_track(ring, native_lib, ref_oracle):
    lat, line = ring
    lat.set_reference()
    ref_oracle.build(lat)
    s = lat.meta["sigma_ip"]
    lo, hi = 0.2, 0.45
    for a in (0.5, 2.0, 4.0):
        x = np.array([a * s, 0., 0.7 * a * s, 0., 0., DELTAP])
        got = api.Cal_Tunes_Track(line, x.copy(), 1024, lo, hi)
        x0 = x.copy()
        x0[0] += 1e-9 if x0[0] < 1e-9 else 0.0
        x0[2] += 1e-9 if x0[2] < 1e-9 else 0.0
        _, so, _, _, tbt = ref_oracle.track_tbt(x0, 1024)
        assert so == 1 and got is not None
        ref = (ref_oracle.fine_tune(tbt[:, 0], None, lo, hi), ref_oracle.fine_tune(tbt[:, 2], None, lo, hi))
        assert abs(got[0] - ref[0]) < 1e-9 and abs(got[1] - ref[1]) < 1e-9, (a, got, ref)
    # the closed-orbit form: a particle on the closed orbit (raised by 1e-9 in
    # x and y) tracked 1,024 turns; its small-amplitude tunes include the
    # beam-beam tune shift of the two interaction points
    q1, q2 = api.Cal_Tunes_Track_orbit(line, 0.0, lo, hi)
    x0 = np.zeros(6)
    x0[:4] = ref_oracle.cal_orbit(0.0)[-1][:4]
    x0[0] += 1e-9 if x0[0] < 1e-9 else 0.0
    x0[2] += 1e-9 if x0[2] < 1e-9 else 0.0
    _, so, _, _, tbt = ref_oracle.track_tbt(x0, 1024)
    ref = (ref_oracle.fine_tune(tbt[:, 0], None, lo, hi), ref_oracle.fine_tune(tbt[:, 2], None, lo, hi))
    assert so == 1 and abs(q1 - ref[0]) < 1e-9 and abs(q2 - ref[1]) < 1e-9, ((q1, q2), ref)
    assert lo < q1 < hi and lo < q2 < hi


def test_cal_chrom_track(ring, native_lib, ref_oracle):
    """Cal_Chrom_Track (simtrack.cpp:21027): the chromaticities are the
    reference's finite differences of the tracked closed-orbit tunes at
    deltap = +3e-4, -3e-4 and 0.  As in the reference, a particle started on
    an off-momentum closed orbit with x above 1e-9 is not displaced, so its
    horizontal "tune" is that of rounding noise; only the vertical tunes,
    whose start is raised by 1e-9, carry a betatron line.  Checked: the
    result equals the formula on this library's Cal_Tunes_Track, whose
    vertical tunes agree with the reference's FineTuneFinder within 1e-8 (the
    line of a 1e-9 m oscillation beside the synchrotron sidebands is flat
    enough at the top that the GPU's and glibc's sincos, which differ in the
    last bit, move its maximum by up to ~6e-9)."""
    lat, line = ring
    lat.set_reference()
    lo, hi = 0.2, 0.45
    got = api.Cal_Chrom_Track(line, lo, hi)
    qp = api.Cal_Tunes_Track_orbit(line, 0.0003, lo, hi)
    qm = api.Cal_Tunes_Track_orbit(line, -0.0003, lo, hi)
    q0 = api.Cal_Tunes_Track_orbit(line, 0.0, lo, hi)
    want = ((qp[0] - qm[0]) / 2. / 0.0003, (qp[1] - qm[1]) / 2. / 0.0003,
            (qp[0] + qm[0] - 2 * q0[0]) / 2. / 0.0003 / 0.0003, (qp[1] + qm[1] - 2 * q0[1]) / 2. / 0.0003 / 0.0003)
    assert got == want
    ref_oracle.build(lat)
    for dp, q in ((0.0003, qp), (-0.0003, qm)):
        x0 = np.zeros(6)
        x0[:4] = ref_oracle.cal_orbit(dp)[-1][:4]
        x0[5] = dp
        x0[0] += 1e-9 if x0[0] < 1e-9 else 0.0
        x0[2] += 1e-9 if x0[2] < 1e-9 else 0.0
        _, so, _, _, tbt = ref_oracle.track_tbt(x0, 1024)
        assert so == 1
        assert abs(q[1] - ref_oracle.fine_tune(tbt[:, 2], None, lo, hi)) < 1e-8
