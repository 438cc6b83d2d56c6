"""Synchrotron radiation on the GPU (GP.radiate) against the compiled
reference (needs a B200).

Ring: `lattices.electron_ring` (3 GeV electrons, 40 cells of sector dipoles
with 5 radiating slices each (SBEND_Pass's radiating branch,
simtrack.cpp:4740-4748: radiate1 with quantum excitation) and combined-
function SBENDMULTs (5437-5463: radiate with the midpoint field of
cal_Bfield), thick quadrupoles, sextupoles, RF).  The reference's radiate1
takes its deviates from GSL, which is absent; both sides use the
per-particle counter-based stream (tests/test_radiation.py pins it).  The
reference is the correctly rounded build (its cos matches the tracker's).

Tolerance as in test_gpu_parity: 1e-12 relative with the per-coordinate rms
floor; loss turn and element exact.
"""
import numpy as np
import pytest

import oracle_bridge
from simtrack_b200 import api
from simtrack_b200 import lattices as lt
from simtrack_b200._native import SimTrackError
from simtrack_b200.api import Table
from test_gpu_parity import assert_close_traj
from test_radiation import normals

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def radiation_off_afterwards():
    yield
    api.Set_Radiation(False)
    oracle_bridge.reference_radiation_off()


@pytest.fixture(scope="module")
def ring():
    lat = lt.electron_ring()
    tab = Table(lt.build_line(lat))
    api.Set_Radiation(False)
    return lat, tab


def _need_ref():
    if not oracle_bridge.ref_available(cr=True):
        pytest.skip("compiled reference oracle (oracle/_ref) not built here")


def _particles(n, seed=3):
    rng = np.random.default_rng(seed)
    X = np.zeros((n, 6))
    X[:, 0] = rng.normal(0, 1e-3, n)
    X[:, 1] = rng.normal(0, 1e-4, n)
    X[:, 2] = rng.normal(0, 1e-3, n)
    X[:, 3] = rng.normal(0, 1e-4, n)
    X[:, 5] = rng.normal(0, 5e-4, n)
    return X


def test_device_stream_equals_host(native_lib):
    for seed, pid, k0 in ((1324, 0, 0), (99, 12345, 2**34 + 7)):
        assert np.array_equal(normals(native_lib, seed, pid, k0, 500_000, 0),
                              normals(native_lib, seed, pid, k0, 500_000, -1))


def test_every_element_vs_reference(ring):
    _need_ref()
    lat, tab = ring
    ref = oracle_bridge.RefOracle(cr=True)
    ref.build(lat)
    X = _particles(4)
    nt = 200
    xg, st, ltn, lp, dump = tab.track_probe(X.copy(), nt)
    for i, x0 in enumerate(X):
        ref.L.ref_rng_id_base(i)  # the probe's particle i draws from stream i
        xo, so, lo, po, do = ref.track_dump(x0, nt, 0.0)
        assert (st[i], ltn[i], lp[i]) == (so, lo, po), f"particle {i}"
        assert_close_traj(dump[i], do, f"particle {i}")
    # radiation is on: the momentum deviation differs from the tracking without it
    plain = lt.electron_ring(radiate=False)
    ref.build(plain)
    xp = ref.track_dump(X[0], nt, 0.0)[0]
    assert abs(xp[5] - xg[0, 5]) > 1e-7


def test_grid_vs_reference(ring):
    _need_ref()
    lat, tab = ring
    import dataclasses
    X = _particles(256, seed=11)
    X[::16, 0] *= 8.0  # some particles start near the 10 mm aperture
    nt = 400
    xg, sg, lg, pg = tab.track_host(X.copy(), nt, 0.01)
    xo, so, lo, po = oracle_bridge.ref_track_parallel(dataclasses.replace(lat, aperture_radius=0.01), X, nt, cr=True)
    assert np.array_equal(sg, so)
    lost = so == 0
    assert lost.any() and not lost.all()
    assert np.array_equal(lg[lost], lo[lost]) and np.array_equal(pg[lost], po[lost])
    assert_close_traj(xg[~lost], xo[~lost], "survivors")


def test_launch_shape_and_turn_blocks_do_not_change_the_stream(ring):
    import torch
    lat, tab = ring
    X = _particles(3000, seed=5)
    nt = 60
    results = []
    for v in (0, 1, 3, 7, 15):  # 7: two particles per thread
        tab.set_variant(v)
        results.append(tab.track_host(X.copy(), nt))
    for r in results[1:]:
        for a, b in zip(results[0], r):
            assert np.array_equal(a, b)
    tab.set_variant(1)
    dev = torch.device("cuda", 0)
    c = [torch.tensor(np.ascontiguousarray(X[:, k]), device=dev) for k in range(6)]
    lt_ = torch.full((len(X),), -1, dtype=torch.int32, device=dev)
    le_ = torch.zeros(len(X), dtype=torch.int32, device=dev)
    tab.track_device(c, lt_, le_, 0, nt // 2)
    tab.track_device(c, lt_, le_, nt // 2, nt - nt // 2)
    torch.cuda.synchronize()
    xs = np.stack([t.cpu().numpy() for t in c], 1)
    alive = lt_.cpu().numpy() < 0
    assert np.array_equal(alive, results[0][1] == 1)
    assert np.array_equal(xs[alive], results[0][0][alive])


def test_unsupported_uses_are_rejected(ring):
    lat, tab = ring
    with pytest.raises(SimTrackError):
        tab.track_radial_host(_particles(4), 2)
    with pytest.raises(SimTrackError):
        api.Scan([tab], [_particles(64)])


def test_spin_tracking_with_radiation_vs_reference():
    """Track_Spin with GP.radiate: SBEND_sPass and SBENDMULT_sPass apply
    radiate() after each slice's spin rotation (simtrack.cpp:7529, 7918; no
    quantum excitation in the spin passes).  Electron G; every element for 50
    turns against the correctly rounded reference."""
    from test_gpu_spin import assert_close9
    _need_ref()
    g_e = 0.00115965218
    lat = lt.electron_ring()
    ref = oracle_bridge.RefOracle(cr=True)
    api.Set_Spin_G(g_e)
    try:
        tab = api.SpinTable(lt.build_line(lat))
        ref.build(lat)
        ref.L.ref_set_spin_g(g_e)
        X = np.zeros((4, 9))
        X[:, :6] = _particles(4, seed=8)
        X[:, 7] = 1.0  # spin along y
        X[1, 6:9] = [0.6, 0.8, 0.0]
        nt = 50
        xg, st, ltn, lp, dump = tab.track_probe(X.copy(), nt)
        for i, x0 in enumerate(X):
            xo, so, lo, po, do = ref.track_spin_dump(x0, nt)
            assert (st[i], ltn[i], lp[i]) == (so, lo, po), f"particle {i}"
            assert_close9(dump[i], do, f"particle {i}")
        assert np.abs(xg[:, 5] - X[:, 5]).max() > 1e-6  # radiation moved the momentum deviation
    finally:
        api.Set_Spin_G(1.7928474)
        ref.L.ref_set_spin_g(1.7928474)


def test_gsbend_photon_emission_vs_reference():
    """GSBEND_Pass's radiating branch (simtrack.cpp:4866-4873): radiate2's
    photon Monte Carlo (Poisson photon count, energies from the spectrum
    table) after each slice, the draws from the per-particle streams on both
    sides.  Every element for 100 turns and a 128-particle grid over 200 turns
    against the correctly rounded reference."""
    import dataclasses
    _need_ref()
    lat = lt.electron_ring(gsbend=True)
    tab = Table(lt.build_line(lat))
    ref = oracle_bridge.RefOracle(cr=True)
    ref.build(lat)
    X = _particles(4, seed=21)
    nt = 100
    xg, st, ltn, lp, dump = tab.track_probe(X.copy(), nt)
    for i, x0 in enumerate(X):
        ref.L.ref_rng_id_base(i)
        xo, so, lo, po, do = ref.track_dump(x0, nt, 0.0)
        assert (st[i], ltn[i], lp[i]) == (so, lo, po), f"particle {i}"
        assert_close_traj(dump[i], do, f"particle {i}")
    plain = lt.electron_ring(gsbend=True, radiate=False)
    ref.build(plain)
    assert abs(ref.track_dump(X[0], nt, 0.0)[0][5] - xg[0, 5]) > 1e-7  # photons were emitted
    Y = _particles(128, seed=22)
    xg2, sg2, lg2, pg2 = tab.track_host(Y.copy(), 200, 0.01)
    xo2, so2, lo2, po2 = oracle_bridge.ref_track_parallel(dataclasses.replace(lat, aperture_radius=0.01), Y, 200,
                                                          cr=True)
    assert np.array_equal(sg2, so2)
    lost = so2 == 0
    assert np.array_equal(lg2[lost], lo2[lost]) and np.array_equal(pg2[lost], po2[lost])
    assert_close_traj(xg2[~lost], xo2[~lost], "survivors")


@pytest.mark.parametrize("gsbend", [False, True])
def test_srloss_particle_vs_reference(gsbend):
    """Cal_SRLoss_Particle (simtrack.cpp:20768-20781): one pass through
    every element but the RF cavities, radiating (radiate1 in the sector
    bends or radiate2's photons in the GSBENDs, radiate in the combined-
    function bends), from particle 0's stream on both sides; exit coordinates
    within the parity tolerance and the loss within 1e-10 relative.  Without
    radiation nothing but the cavities changes pt: the loss is exactly 0."""
    _need_ref()
    lat = lt.electron_ring(gsbend=gsbend)
    line = lt.build_line(lat)
    ref = oracle_bridge.RefOracle(cr=True)
    ref.build(lat)
    ref.L.ref_rng_id_base(0)
    for x0 in (np.zeros(6), np.array([1e-3, 1e-4, -5e-4, 2e-5, 0.0, 3e-4])):
        xg, xo = x0.copy(), x0.copy()
        lg = api.Cal_SRLoss_Particle(line, xg)
        lo = ref.L.ref_cal_srloss_particle(ref.line, xo.ctypes.data)
        assert_close_traj(xg[None], xo[None], "exit")
        assert lo < -0.2 and abs(lg - lo) <= 1e-10 * abs(lo), (lg, lo)
    x = np.array([0.2, 0, 0, 0, 0, 0.0])  # Track()'s entry test would stop it
    with pytest.raises(SimTrackError):
        api.Cal_SRLoss_Particle(line, x)
    assert x[0] == 0.2 and not x[1:].any()
    api.Set_Radiation(False)
    plain = lt.build_line(lt.electron_ring(gsbend=gsbend, radiate=False))
    x = np.array([1e-3, 1e-4, -5e-4, 2e-5, 0.0, 3e-4])
    assert api.Cal_SRLoss_Particle(plain, x) == 0.0 and x[5] == 3e-4
