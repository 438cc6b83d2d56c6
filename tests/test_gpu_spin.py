"""Spin tracking parity: the GPU Track_Spin against the reference's own
Track_Spin / Element::sPass (needs a B200).

Tolerance as for orbit tracking: every one of the nine coordinates (orbit
and spin vector) after every element agrees to 1e-12 relative with the
per-coordinate rms floor; loss turn and element match exactly.  The
reference's outputs come from the compiled reference when it is built and
from the golden fixture tests/golden/spin_zoo.npz (made from it) otherwise."""
from pathlib import Path

import numpy as np
import pytest

from lattice_zoo import spin_particles, spin_zoo
from simtrack_b200 import lattices as lt
from simtrack_b200.api import SpinTable, Table
from simtrack_b200._native import SimTrackError

pytestmark = pytest.mark.gpu

RTOL = 1e-12
GOLDEN = Path(__file__).resolve().parent / "golden" / "spin_zoo.npz"


def assert_close9(gpu, ora, what=""):
    g = gpu.reshape(-1, 9)
    o = ora.reshape(-1, 9)
    reached = ~np.isnan(o[:, 0])
    assert np.array_equal(reached, ~np.isnan(g[:, 0])), f"{what}: different element coverage"
    g, o = g[reached], o[reached]
    floor = np.maximum(np.sqrt(np.mean(o * o, axis=0)), 1e-300)
    bad = np.abs(g - o) > RTOL * np.maximum(np.abs(o), floor)
    if bad.any():
        i, k = np.argwhere(bad)[0]
        raise AssertionError(f"{what}: entry {i} coord {k}: gpu {g[i, k]!r} reference {o[i, k]!r} "
                             f"({bad.sum()} entries over tolerance)")


def test_spin_zoo_every_element_vs_golden(native_lib):
    lat = spin_zoo()
    tab = SpinTable(lt.build_line(lat))
    g = np.load(GOLDEN)
    X = g["x0"]
    nt = int(g["nturn"])
    xg, st, ltn, lp, dump = tab.track_probe(X.copy(), nt)
    for i in range(len(X)):
        assert (st[i], ltn[i], lp[i]) == tuple(g["loss"][i]), f"particle {i}"
        assert_close9(dump[i], g["dump"][i], f"spin zoo particle {i}")


def test_spin_zoo_every_element_vs_reference(native_lib, ref_oracle):
    lat = spin_zoo()
    tab = SpinTable(lt.build_line(lat))
    ref_oracle.build(lat)
    X = spin_particles()
    nt = 3
    xg, st, ltn, lp, dump = tab.track_probe(X.copy(), nt)
    for i, x0 in enumerate(X):
        xo, so, lo, po, do = ref_oracle.track_spin_dump(x0, nt)
        assert (st[i], ltn[i], lp[i]) == (so, lo, po), f"particle {i}"
        assert_close9(dump[i], do, f"spin zoo particle {i}")


def _eic_particles(lat, n=6, seed=3):
    rng = np.random.default_rng(seed)
    sig = lat.meta["sigma_ip"]
    X = np.zeros((n, 9))
    X[:, 0] = rng.uniform(-4, 4, n) * sig
    X[:, 2] = rng.uniform(-4, 4, n) * sig
    X[:, 4] = rng.uniform(-0.05, 0.05, n)
    X[:, 5] = rng.uniform(-5e-4, 5e-4, n)
    s = rng.normal(0, 1, (n, 3)) * [0.05, 1.0, 0.05]
    X[:, 6:] = s / np.linalg.norm(s, axis=1, keepdims=True)
    return X


def test_spin_eic_ring_every_element_one_turn(native_lib, ref_oracle):
    lat = lt.eic_like_ring(seed=1)
    tab = SpinTable(lt.build_line(lat))
    ref_oracle.build(lat)
    X = _eic_particles(lat, n=3)
    xg, st, ltn, lp, dump = tab.track_probe(X.copy(), 1)
    for i, x0 in enumerate(X):
        xo, so, lo, po, do = ref_oracle.track_spin_dump(x0, 1)
        assert (st[i], ltn[i], lp[i]) == (so, lo, po)
        assert_close9(dump[i], do, f"eic particle {i}")


def test_spin_eic_ring_many_turns(native_lib, ref_cr_oracle):
    """Final coordinates and spin after 300 turns, and the unit length of the
    spin, against the reference built with correctly rounded transcendentals:
    with the host C library's own functions, an occasional last-bit
    difference of an arcsine (glibc is not correctly rounded for every
    argument) starts a divergence that these particles amplify to 1e-7 within
    300 turns."""
    ref_oracle = ref_cr_oracle
    lat = lt.eic_like_ring(seed=2)
    tab = SpinTable(lt.build_line(lat))
    ref_oracle.build(lat)
    X = _eic_particles(lat, n=8, seed=5)
    nt = 300
    xg, st, ltn, lp = tab.track_host(X.copy(), nt)
    xo, so, lo, po = ref_oracle.track_spin(X.copy(), nt)
    assert np.array_equal(st, so) and np.array_equal(ltn, lo) and np.array_equal(lp, po)
    alive = st == 1
    assert alive.any()
    assert_close9(xg[alive], xo[alive], "eic final")
    # the spin stays a unit vector up to the rounding of ~7e6 rotations
    # (the reference's rotations round identically)
    norm = np.linalg.norm(xg[alive, 6:], axis=1)
    assert np.max(np.abs(norm - 1.0)) < 1e-10


def test_tables_keep_to_their_mode(native_lib):
    import torch
    lat = spin_zoo()
    line = lt.build_line(lat)
    spin_tab, orbit_tab = SpinTable(line), Table(line)
    with pytest.raises(SimTrackError, match="spin"):
        Table.track_host(spin_tab, np.zeros((2, 6)), 1)
    with pytest.raises(SimTrackError, match="spin"):
        SpinTable.track_host(orbit_tab, np.zeros((2, 9)), 1)
    # a device call through the spin entry point updates the nine arrays in place
    x = torch.tensor(spin_particles()[:3].T.copy(), device="cuda:0")
    lost = torch.full((3,), -1, dtype=torch.int32, device="cuda:0")
    le = torch.zeros(3, dtype=torch.int32, device="cuda:0")
    spin_tab.track_device([x[k] for k in range(9)], lost, le, 0, 1)
    torch.cuda.synchronize()
    xh, st, _, _ = spin_tab.track_host(spin_particles()[:3].copy(), 1)
    np.testing.assert_array_equal(x.cpu().numpy().T, xh)


def test_spin_launch_variants_agree_and_autotune(native_lib):
    """Every launch variant of the spin kernel gives the same bits (same maps,
    different CTA shapes and register budgets), and the autotuner leaves the
    inputs untouched and picks one of them."""
    import torch
    from simtrack_b200.api import NUM_SPIN_VARIANTS
    lat = lt.eic_like_ring(seed=3)
    tab = SpinTable(lt.build_line(lat))
    X = _eic_particles(lat, n=200, seed=9)
    coords = [torch.tensor(X[:, k].copy(), device="cuda:0") for k in range(9)]
    tune = tab.autotune(coords, 1, 0.03)
    assert tune["chosen"] in tune["ms"]
    assert np.array_equal(torch.stack(coords, 1).cpu().numpy(), X)
    ref = None
    for v in range(NUM_SPIN_VARIANTS):
        try:
            tab.set_variant(v)
        except SimTrackError:
            continue  # a shared-memory variant the table does not fit
        out = tab.track_host(X.copy(), 3, 0.03)
        if ref is None:
            ref = out
        else:
            for a, b in zip(ref, out):
                assert np.array_equal(a, b), f"variant {v}"
    assert ref is not None
