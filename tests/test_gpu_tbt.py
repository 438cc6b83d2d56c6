"""Turn-by-turn tracking and its diagnostics on the GPU against the compiled
reference (needs a B200).

* Track_tbt (simtrack.cpp:20841-20860): the record x_tbt (start of every
  turn up to the turn of the loss) and the loss outputs, bit for bit.
* Track_tbt_Lyapunov (21243-21306): the output file, byte for byte, against
  the reference's own run on a thin-lens ring.
* Track_tbt_FMA (21179-21241): the same grid rows as the reference (which
  particles survive 2,048 turns), and for a sample of rows every tune within
  1e-9 of the reference's FineTuneFinder on the reference's own record (the
  GPU tune finder's sincos and glibc's differ in the last bit, which moves
  the flat top of a DFT peak by far less)."""
import os

import numpy as np
import pytest

from lattice_zoo import thin_fodo_ring, zoo, zoo_particles
from simtrack_b200 import api
from simtrack_b200 import lattices as lt

pytestmark = pytest.mark.gpu

SIGMA = 1e-3  # amplitude unit of the maps on the thin-lens ring [m]


def _same(a, b):
    return np.array_equal(np.nan_to_num(a, nan=7.0), np.nan_to_num(b, nan=7.0))


@pytest.mark.parametrize("which", ["zoo", "fodo"])
def test_track_tbt_record(which, native_lib, ref_oracle):
    if which == "zoo":
        lat, X, nt = zoo(), zoo_particles(), 3
    else:
        lat = lt.fodo_ring()
        a = np.linspace(0.0, 0.03, 12)
        X = np.zeros((12, 6))
        X[:, 0] = a
        X[:, 2] = 0.5 * a
        X[-1, 0] = 0.2  # rejected by the entry check: nothing recorded
        nt = 60
    line = lt.build_line(lat)
    x, st, ltn, lp, tbt = api.Track_tbt(line, X, nt)
    ref_oracle.build(lat)
    lost = 0
    for i, x0 in enumerate(X):
        xo, so, lo, po, to = ref_oracle.track_tbt(x0, nt)
        assert (st[i], ltn[i], lp[i]) == (so, lo, po), f"particle {i}"
        assert _same(tbt[i], to), f"particle {i}: record differs"
        assert _same(x[i], xo), f"particle {i}: final coordinates differ"
        lost += so == 0
    assert lost > 0  # losses (entry check or in tracking) are covered


@pytest.mark.parametrize("which,bpm", [("zoo", 0), ("zoo", 17), ("fodo", 600), ("fodo", 1200)])
def test_track_tbt_bpm_record(which, bpm, native_lib, ref_oracle):
    """Track_tbt with a BPM index (simtrack.cpp:20884): the record after
    element `bpm` in every turn that reaches it, losses before and after the
    element included."""
    if which == "zoo":
        lat, X, nt = zoo(), zoo_particles(), 3
    else:
        lat = lt.fodo_ring()
        a = np.linspace(0.0, 0.03, 12)
        X = np.zeros((12, 6))
        X[:, 0] = a
        X[:, 2] = 0.5 * a
        X[-1, 0] = 0.2
        nt = 60
    line = lt.build_line(lat)
    x, st, ltn, lp, tbt = api.Track_tbt(line, X, nt, bpm_index=bpm)
    ref_oracle.build(lat)
    for i, x0 in enumerate(X):
        xo, so, lo, po, to = ref_oracle.track_tbt_bpm(x0, nt, bpm)
        assert (st[i], ltn[i], lp[i]) == (so, lo, po), f"particle {i}"
        assert _same(tbt[i], to), f"particle {i}: record differs"
        assert _same(x[i], xo), f"particle {i}: final coordinates differ"


@pytest.mark.parametrize("bpm", [0, 12, 33])
def test_track_tbt_spin_bpm_record(bpm, native_lib, ref_oracle):
    """Track_tbt_spin with a BPM index (simtrack.cpp:20907): the nine
    coordinates after element `bpm` in every turn that reaches it."""
    from lattice_zoo import spin_particles, spin_zoo
    lat = spin_zoo()
    line = lt.build_line(lat)
    X = spin_particles()
    nt = 3
    x, st, ltn, lp, tbt = api.Track_tbt(line, X, nt, spin=True, bpm_index=bpm)
    ref_oracle.build(lat)
    for i, x0 in enumerate(X):
        xo, so, lo, po, to = ref_oracle.track_tbt_bpm(x0, nt, bpm)
        assert (st[i], ltn[i], lp[i]) == (so, lo, po), f"particle {i}"
        assert _same(tbt[i], to), f"particle {i}: record differs"


def test_track_tbt_spin_record(native_lib, ref_oracle):
    """Track_tbt_spin (simtrack.cpp:20863): the nine-coordinate record."""
    from lattice_zoo import spin_particles, spin_zoo
    lat = spin_zoo()
    line = lt.build_line(lat)
    X = spin_particles()
    nt = 3
    x, st, ltn, lp, tbt = api.Track_tbt(line, X, nt, spin=True)
    ref_oracle.build(lat)
    for i, x0 in enumerate(X):
        xo, so, lo, po, to = ref_oracle.track_tbt(x0, nt)
        assert (st[i], ltn[i], lp[i]) == (so, lo, po), f"particle {i}"
        assert _same(tbt[i], to), f"particle {i}: record differs"


def test_lyapunov_file_matches_reference(native_lib, ref_oracle, tmp_path, monkeypatch):
    lat = thin_fodo_ring()
    line = lt.build_line(lat)
    rows = api.Track_tbt_Lyapunov(line, 0.0, SIGMA, SIGMA, tmp_path / "gpu.dat")
    ref_oracle.build(lat)
    monkeypatch.chdir(tmp_path)
    ref_oracle.L.ref_track_tbt_lyapunov(ref_oracle.line, 0.0, SIGMA, SIGMA)
    ours = (tmp_path / "gpu.dat").read_text()
    ref = (tmp_path / "Lmap-output.dat").read_text()
    assert 5000 < rows == len(ref.splitlines()) < 11425  # some twins are lost
    assert ours == ref


def test_fma_matches_reference(native_lib, ref_oracle, tmp_path):
    lat = thin_fodo_ring()
    line = lt.build_line(lat)
    lo, hi = 0.25, 0.35
    rows = api.Track_tbt_FMA(line, 0.0, SIGMA, SIGMA, tmp_path / "fma.dat", tune_low=lo, tune_high=hi)
    text = (tmp_path / "fma.dat").read_text().splitlines()
    assert rows == len(text)
    vals = np.array([[float(v) for v in r.split()] for r in text])
    # the rows: every grid point of the quarter disc that survives 2,048 turns
    ref_oracle.build(lat)
    grid = [(i, j) for i in range(61) for j in range(61) if (1.0 * i * i + 1.0 * j * j) ** 0.5 <= 6. / 0.1]
    orbit = ref_oracle.cal_orbit(0.0)[-1]
    X = np.zeros((len(grid), 6))
    for p, (i, j) in enumerate(grid):
        # the reference's start (Track_tbt_FMA, simtrack.cpp:21203-21216)
        x = [i * 0.1 * SIGMA + 0., 0., j * 0.1 * SIGMA, 0., 0., 0.0]
        for k in range(4):
            x[k] = x[k] + orbit[k]
        if x[0] < 1.0e-09:
            x[0] = x[0] + 1.0e-09
        if x[2] < 1.0e-09:
            x[2] = x[2] + 1.0e-09
        X[p] = x
    _, st, _, _ = ref_oracle.track(X.copy(), 2048, radius=0.0)
    expect = [g for g, s in zip(grid, st) if s == 1]
    assert 100 < len(expect) < len(grid)  # the outer amplitudes are lost
    assert [(round(a / 0.1), round(b / 0.1)) for a, b in vals[:, :2]] == expect
    assert text[0].startswith("0 0 ") and text[1].startswith("0.000000000000000000e+00 ")
    rng = np.random.default_rng(5)
    for r in rng.choice(len(expect), 40, replace=False):
        i, j = expect[r]
        x0 = X[grid.index((i, j))]
        _, so, _, _, tbt = ref_oracle.track_tbt(x0, 2048)
        assert so == 1
        ref_t = [ref_oracle.fine_tune(tbt[a:b, k], None, lo, hi)
                 for k, (a, b) in ((0, (0, 1024)), (0, (1023, 2047)), (2, (0, 1024)), (2, (1023, 2047)))]
        got = vals[r, 2:6]
        assert np.max(np.abs(got - ref_t)) < 1e-9, (i, j, got, ref_t)
        assert vals[r, 6] == got[0] - got[1] and vals[r, 7] == got[2] - got[3]
