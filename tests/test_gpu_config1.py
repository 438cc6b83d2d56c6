"""The headline configuration against the compiled reference (needs a B200).

Ring: the synthetic RHIC-like ring with seed-1 triplet errors (1,810
elements: thick quadrupoles, exact sector bends, thin sextupoles, order-10
triplet multipoles with Nint = 8, 6D beam-beam at two IPs, RF at 28 and
197 MHz, 30 mm circular aperture).  Reference loop: Track,
simtrack.cpp:20791-20814.

* Every coordinate after every element for 1,000 turns, five particles
  (core, mid amplitude, just inside the dynamic aperture, off momentum by
  +-1e-3), against the reference built with correctly rounded
  transcendentals (oracle/crlibm_shim.cpp); the first 100 turns also against
  the reference as built with the host C library.
* The DA grid of the configuration (64 amplitudes 0-12 sigma x 11 angles x 5
  momentum offsets = 3,520 particles) for 1,000 turns: every particle's
  stable flag, loss turn and loss element, and the survivors' final
  coordinates, against the correctly rounded reference; against the plain
  reference, the loss turn of every particle more than one amplitude step
  from its ray's aperture boundary.
* The batched scan (work list, compaction between turn blocks, CUDA graphs)
  on three seeds against the correctly rounded reference directly.

Tolerance: |gpu - reference| <= 1e-12 * max(|reference|, s_k), s_k the rms of
coordinate k over the compared set; loss turn and element exact.
"""
import numpy as np
import pytest

import oracle_bridge
from simtrack_b200 import lattices as lt
from simtrack_b200.api import Scan, Table
from test_gpu_parity import assert_close_traj

pytestmark = pytest.mark.gpu

NAMP, AMAX, NANG = 64, 12.0, 11
DELTAS = [-1e-3, -5e-4, 0.0, 5e-4, 1e-3]


def _need_ref(cr):
    if not oracle_bridge.ref_available(cr=cr):
        pytest.skip("compiled reference oracle (oracle/_ref) not built here")


def _five_particles(lat):
    sig = lat.meta["sigma_ip"]

    def at(a, deg, dp):
        t = np.deg2rad(deg)
        return [a * np.cos(t) * sig, 0.0, a * np.sin(t) * sig, 0.0, 0.0, dp]

    step = AMAX / (NAMP - 1)
    return np.array([at(1.0, 45.0, 0.0),          # core
                     at(4.0, 30.0, 0.0),          # mid amplitude
                     at(41 * step, 7.5, 0.0),     # just inside the aperture of the 7.5 degree ray
                     at(3.0, 45.0, 1e-3),         # off momentum
                     at(3.0, 45.0, -1e-3)])


@pytest.fixture(scope="module")
def ring():
    lat = lt.rhic_like_ring(seed=1)
    return lat, Table(lt.build_line(lat))


def test_every_element_1000_turns(ring):
    _need_ref(True)
    lat, tab = ring
    ref = oracle_bridge.RefOracle(cr=True)
    ref.build(lat)
    X = _five_particles(lat)
    nt = 1000
    xg, st, ltn, lp, dump = tab.track_probe(X.copy(), nt, lat.aperture_radius)
    for i, x0 in enumerate(X):
        xo, so, lo, po, do = ref.track_dump(x0, nt)
        assert (st[i], ltn[i], lp[i]) == (so, lo, po), f"particle {i}"
        assert so == 1, f"particle {i} was meant to survive 1,000 turns"
        for t0 in range(0, nt, 100):  # compare in blocks of turns to bound memory
            assert_close_traj(dump[i, t0:t0 + 100], do[t0:t0 + 100], f"particle {i} turns {t0}-{t0 + 99}")
        assert_close_traj(xg[i], xo, f"particle {i} final")


def test_every_element_100_turns_plain_reference(ring):
    _need_ref(False)
    lat, tab = ring
    ref = oracle_bridge.RefOracle(cr=False)
    ref.build(lat)
    X = _five_particles(lat)
    nt = 100
    xg, st, ltn, lp, dump = tab.track_probe(X.copy(), nt, lat.aperture_radius)
    for i, x0 in enumerate(X):
        xo, so, lo, po, do = ref.track_dump(x0, nt)
        assert (st[i], ltn[i], lp[i]) == (so, lo, po), f"particle {i}"
        assert_close_traj(dump[i], do, f"particle {i}")


def _boundary_index(stable):
    """Per ray (rows), the first lost amplitude index (NAMP if none)."""
    lost = stable == 0
    return np.where(lost.any(axis=1), np.argmax(lost, axis=1), NAMP)


def test_da_grid_1000_turns(ring):
    _need_ref(True)
    _need_ref(False)
    lat, tab = ring
    X = lt.da_grid(lat, NAMP, AMAX, NANG, DELTAS)
    assert X.shape == (3520, 6)
    nt = 1000
    xg, st, ltn, lp = tab.track_host(X.copy(), nt, lat.aperture_radius)
    xo, so, lo, po = oracle_bridge.ref_track_parallel(lat, X, nt, cr=True)
    assert np.array_equal(st, so)
    lost = so == 0
    assert np.array_equal(ltn[lost], lo[lost]) and np.array_equal(lp[lost], po[lost])
    assert 0 < lost.sum() < len(X)  # the grid reaches past the dynamic aperture
    surv = ~lost
    assert_close_traj(xg[surv], xo[surv], "grid survivors")
    # against the reference's own C library: loss turns agree away from the
    # aperture boundary (one amplitude step either side of it may differ)
    xp, sp, lpt, ppo = oracle_bridge.ref_track_parallel(lat, X, nt, cr=False)
    rays = len(DELTAS) * NANG
    b = _boundary_index(sp.reshape(rays, NAMP))
    amp = np.tile(np.arange(NAMP), rays).reshape(rays, NAMP)
    far = (np.abs(amp - b[:, None]) > 1).ravel()
    assert np.array_equal(st[far], sp[far])
    lost_far = far & (sp == 0)
    assert np.array_equal(ltn[lost_far], lpt[lost_far]) and np.array_equal(lp[lost_far], ppo[lost_far])
    # DA per ray within one amplitude step of the plain reference's
    bg = _boundary_index(st.reshape(rays, NAMP))
    assert np.max(np.abs(bg - b)) <= 1


def test_batched_scan_1000_turns():
    """Scan kernels (work list, tracking, compaction every 128 turns, CUDA
    graphs) on three seeds, every 4th grid particle, against the reference."""
    _need_ref(True)
    nseed, nt = 3, 1000
    lats = [lt.rhic_like_ring(seed=s + 1) for s in range(nseed)]
    tabs = [Table(lt.build_line(lat)) for lat in lats]
    xs = [lt.da_grid(lat, NAMP, AMAX, NANG, DELTAS)[::4].copy() for lat in lats]
    sc = Scan(tabs, xs, aperture_radius=lats[0].aperture_radius)
    sc.autotune(16)
    sc.run(nt, turns_per_block=128, use_graph=True)
    lt_s, le_s, x_s = sc.results()
    off = 0
    for s in range(nseed):
        n = len(xs[s])
        xo, so, lo, po = oracle_bridge.ref_track_parallel(lats[s], xs[s], nt, cr=True)
        exp_lt = np.where(so == 1, -1, lo)
        assert np.array_equal(lt_s[off:off + n], exp_lt), f"seed {s + 1}"
        lost = so == 0
        assert lost.any() and not lost.all()
        assert np.array_equal(le_s[off:off + n][lost], po[lost]), f"seed {s + 1}"
        assert_close_traj(x_s[off:off + n][~lost], xo[~lost], f"seed {s + 1} survivors")
        off += n
