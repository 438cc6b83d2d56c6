"""Segmented shared-memory staging (needs a B200).

The reference's own RHIC lattice (Example1/parameters_input, read by our
MAD-X reader; 6,858 elements, too large for one shared-memory copy) is
tracked through the seg_* launch variants, which stage the table segment by
segment into two shared-memory buffers with bulk copies.  Against the
compiled reference (its reader and Track(), simtrack.cpp:13591, 20791):
every coordinate after every element, and the loss outputs; all segmented
variants and segment sizes give the same bits.
"""
import lzma
from pathlib import Path

import numpy as np
import pytest

from simtrack_b200 import api
from simtrack_b200._native import SimTrackError
from test_gpu_parity import assert_close_traj

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
SEG_VARIANTS = [11, 12, 13]  # seg_b1024_r64, seg_b768_r85, seg_b512_r128


@pytest.fixture(scope="module")
def rhic(tmp_path_factory):
    path = tmp_path_factory.mktemp("rhic") / "parameters_input"
    path.write_bytes(lzma.decompress((GOLDEN / "rhic_example1.tfs.xz").read_bytes()))
    api.Set_RefPartEnergy(100.0, 938.27201, 1, 1)
    api.Set_Flags(False, False)
    line = api.Line()
    line.read_madx(str(path))
    return path, line


def _particles():
    return np.array([[1e-3, 0, 5e-4, 0, 0, 0], [-2e-3, 1e-5, 1e-3, -2e-6, 0.01, 3e-4],
                     [4e-3, 0, -3e-3, 0, 0, -5e-4]])


def test_table_is_planned_in_segments(rhic):
    path, line = rhic
    tab = api.Table(line)
    assert line.Ncell == 6858
    info = tab.info()
    assert not info["smem"]
    seg = tab.segments()
    assert seg["nseg"] >= 2 and 0 < seg["bytes"] <= info["table_bytes"]
    tab.set_segment_bytes(16384)
    assert tab.segments()["nseg"] > seg["nseg"]
    with pytest.raises(SimTrackError):
        tab.set_segment_bytes(512)


def test_every_element_through_segments_vs_reference(rhic, ref_oracle):
    path, line = rhic
    tab = api.Table(line)
    tab.set_variant(SEG_VARIANTS[0])
    ref_oracle.L.ref_set_ref_energy(100.0, 938.27201, 1.0, 1.0)
    ref_oracle.L.ref_set_flags(0, 0)
    ref_oracle.read_madx(str(path))
    X = _particles()
    nt = 8
    xg, st, ltn, lp, dump = tab.track_probe(X.copy(), nt)
    for i, x0 in enumerate(X):
        xo, so, lo, po, do = ref_oracle.track_dump(x0, nt)
        assert (st[i], ltn[i], lp[i]) == (so, lo, po), f"particle {i}"
        assert_close_traj(dump[i], do, f"particle {i}")
        if so:
            assert_close_traj(xg[i], xo, f"particle {i} final")


def test_segment_variants_and_sizes_agree_with_reference(rhic, ref_oracle):
    path, line = rhic
    tab = api.Table(line)
    rng = np.random.default_rng(5)
    n, nt = 300, 12
    X = np.zeros((n, 6))
    X[:, 0] = rng.normal(0, 2e-3, n)
    X[:, 2] = rng.normal(0, 2e-3, n)
    X[:, 4] = rng.normal(0, 0.05, n)
    X[:, 5] = rng.normal(0, 5e-4, n)
    ref_oracle.L.ref_set_ref_energy(100.0, 938.27201, 1.0, 1.0)
    ref_oracle.L.ref_set_flags(0, 0)
    ref_oracle.read_madx(str(path))
    xo, so, lo, po = ref_oracle.track(X[:40].copy(), nt, radius=0.0)
    results = []
    for nbytes in (None, 32768):
        if nbytes:
            tab.set_segment_bytes(nbytes)
        for v in SEG_VARIANTS:
            tab.set_variant(v)
            results.append(tab.track_host(X.copy(), nt))
    tab.set_variant(3)  # the L1 path, no staging
    results.append(tab.track_host(X.copy(), nt))
    first = results[0]
    for r in results[1:]:
        for a, b in zip(first, r):
            assert np.array_equal(a, b)
    xg, sg, lg, pg = first
    assert np.array_equal(sg[:40], so) and np.array_equal(lg[:40], lo) and np.array_equal(pg[:40], po)
    ok = so == 1
    assert_close_traj(xg[:40][ok], xo[ok], "grid")


def test_autotuner_picks_a_runnable_staging(rhic):
    import torch
    path, line = rhic
    tab = api.Table(line)
    X = _particles()
    coords = [torch.tensor(np.repeat(X[:, k], 2000).copy(), device="cuda:0") for k in range(6)]
    tune = tab.autotune(coords, 1)
    assert tune["ms"][tune["chosen"]] > 0
    assert all(v < 0 for k, v in tune["ms"].items() if k.startswith("smem_"))  # the table does not fit whole
    assert any(v > 0 for k, v in tune["ms"].items() if k.startswith("seg_"))
    seg = tab.segments()
    assert seg["nseg"] >= 2
