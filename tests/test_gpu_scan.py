"""Batched DA scan (work list + tracking + compaction + CUDA graphs) against
per-seed single-lattice tracking, and its stop/resume controls: the abort
flag set from another host thread, the wall-clock budget, checkpoint and
restore (needs a B200)."""
import numpy as np
import pytest

from simtrack_b200 import lattices as lt
from simtrack_b200._native import STB_EABORTED, STB_ETIMEOUT, SimTrackError
from simtrack_b200.api import NUM_SCAN_VARIANTS, Scan, Table

pytestmark = pytest.mark.gpu


def seed_setup(nseed, namp=16, nang=4, amax=14.0):
    tabs, xs, lats = [], [], []
    for s in range(nseed):
        lat = lt.rhic_like_ring(seed=s + 1)
        line = lt.build_line(lat)
        tabs.append(Table(line))
        lats.append((lat, line))
        xs.append(lt.da_grid(lat, namp, amax, nang, [0.0, 5e-4]))
    return tabs, xs, lats


@pytest.mark.parametrize("use_graph", [True, False])
def test_scan_matches_single_table_tracking(use_graph):
    nseed, nturn, tpb = 3, 300, 64
    tabs, xs, lats = seed_setup(nseed)
    sc = Scan(tabs, xs, aperture_radius=0.03)
    sc.configure(variant=2, chunk=64)
    sc.run(nturn, turns_per_block=tpb, use_graph=use_graph)
    lt_s, le_s, x_s = sc.results()
    off = 0
    lost_any = 0
    for s in range(nseed):
        n = len(xs[s])
        xr, st, ltn, lp = tabs[s].track_host(xs[s].copy(), nturn, 0.03)
        exp_lt = np.where(st == 1, -1, ltn)
        assert np.array_equal(lt_s[off:off + n], exp_lt), f"seed {s}"
        lost = st == 0
        assert np.array_equal(le_s[off:off + n][lost], lp[lost])
        assert np.array_equal(x_s[off:off + n], xr)
        lost_any += int(lost.sum())
        off += n
    assert lost_any > 0  # the grid reaches beyond the dynamic aperture
    assert sc.stats()["turns"] == nturn


def test_scan_variants_agree():
    tabs, xs, lats = seed_setup(2, namp=12, nang=3)
    ref = None
    for v in range(NUM_SCAN_VARIANTS):
        sc = Scan(tabs, xs, aperture_radius=0.03)
        try:
            sc.configure(variant=v, chunk=128)
        except Exception:
            continue
        sc.run(130, turns_per_block=40)
        res = sc.results()
        if ref is None:
            ref = res
        else:
            for a, b in zip(ref, res):
                assert np.array_equal(a, b)


def test_scan_turn_by_turn_record_and_retire():
    import torch

    from simtrack_b200.api import RETIRED

    tabs, xs, lats = seed_setup(2, namp=12, nang=3)
    sc = Scan(tabs, xs, aperture_radius=0.03)
    n = sc.n
    nrec = 24
    tbt = torch.full((nrec, 4, n), float("nan"), dtype=torch.float64, device="cuda:0")
    sc.set_tbt(tbt, nrec)
    sc.run(10, turns_per_block=5)
    # retire every third particle (x0 order) after 10 turns
    mask = np.zeros(n, dtype=bool)
    mask[::3] = True
    lt10, _, _ = sc.results()
    sc.retire(mask)
    sc.run(30, turns_per_block=8)
    lt_s, le_s, x_s = sc.results()
    rec = tbt.cpu().numpy()
    # reference: per-seed single-table tracking one turn at a time
    off = 0
    for s in range(2):
        m = len(xs[s])
        coords = torch.tensor(xs[s].T.copy(), dtype=torch.float64, device="cuda:0").contiguous()
        lost = torch.full((m,), -1, dtype=torch.int32, device="cuda:0")
        le = torch.zeros(m, dtype=torch.int32, device="cuda:0")
        for t in range(nrec):
            tabs[s].track_device([coords[k] for k in range(6)], lost, le, t, 1, 0.03)
            c = coords.cpu().numpy()
            l = lost.cpu().numpy()
            live = l < 0
            if t >= 10:
                live &= ~mask[off:off + m]
            for k, row in enumerate((0, 1, 2, 3)):
                got = rec[t, k, off:off + m]
                assert np.array_equal(got[live], c[row][live]), f"seed {s} turn {t} coord {k}"
        off += m
    retired = (lt10 < 0) & mask
    assert retired.any()
    assert np.all(lt_s[retired] == RETIRED)
    # the others follow the plain scan exactly
    plain = Scan(tabs, xs, aperture_radius=0.03)
    plain.run(40, turns_per_block=8)
    lt_p, le_p, x_p = plain.results()
    keep = ~retired
    assert np.array_equal(lt_s[keep], lt_p[keep])
    assert np.array_equal(x_s[keep], x_p[keep])


def _small_scan(tabs, xs):
    sc = Scan(tabs, xs, aperture_radius=0.03)
    sc.configure(variant=2, chunk=64)
    return sc


def test_checkpoint_resume_equals_uninterrupted(tmp_path):
    tabs, xs, lats = seed_setup(2, namp=12, nang=3)
    whole = _small_scan(tabs, xs)
    whole.run(300, turns_per_block=64)
    ref = whole.results()
    first = _small_scan(tabs, xs)
    first.run(128, turns_per_block=64)
    path = tmp_path / "scan.ckpt"
    first.checkpoint(path)
    second = _small_scan(tabs, xs)
    second.restore(path)
    assert second.stats()["turns"] == 128
    second.run(172, turns_per_block=64)
    got = second.results()
    for a, b in zip(ref, got):
        assert np.array_equal(a, b)
    assert second.stats()["turns"] == 300
    # a checkpoint of another scan is refused
    other = Scan(tabs[:1], xs[:1], aperture_radius=0.03)
    with pytest.raises(SimTrackError, match="different scan"):
        other.restore(path)


def test_abort_flag_stops_at_a_block_boundary_and_resumes():
    import threading
    import time
    tabs, xs, lats = seed_setup(2, namp=12, nang=3)
    whole = _small_scan(tabs, xs)
    whole.run(400, turns_per_block=8, use_graph=True)
    ref = whole.results()
    sc = _small_scan(tabs, xs)
    sc.set_abort(True)
    with pytest.raises(SimTrackError) as e:
        sc.run(400, turns_per_block=8)
    assert e.value.code == STB_EABORTED and sc.stats()["turns"] == 0
    sc.set_abort(False)
    err = []

    def worker():
        try:
            sc.run(400, turns_per_block=8, use_graph=True)
        except SimTrackError as ex:
            err.append(ex)

    th = threading.Thread(target=worker)
    th.start()
    time.sleep(0.3)
    sc.set_abort(True)  # from another host thread, while the run is on the device
    th.join(timeout=300)
    assert not th.is_alive()
    done = sc.stats()["turns"]
    if err:  # the run was stopped part way (it may also have finished first)
        assert err[0].code == STB_EABORTED
        assert done % 8 == 0 and done < 400
    sc.set_abort(False)
    sc.run(400 - done, turns_per_block=8)
    for a, b in zip(ref, sc.results()):
        assert np.array_equal(a, b)


def test_wall_clock_budget_stops_and_resumes():
    tabs, xs, lats = seed_setup(2, namp=12, nang=3)
    whole = _small_scan(tabs, xs)
    whole.run(256, turns_per_block=16)
    sc = _small_scan(tabs, xs)
    sc.set_budget(1e-6)
    with pytest.raises(SimTrackError) as e:
        sc.run(256, turns_per_block=16)
    assert e.value.code == STB_ETIMEOUT
    done = sc.stats()["turns"]
    assert done % 16 == 0 and done < 256
    sc.set_budget(0)
    sc.run(256 - done, turns_per_block=16)
    for a, b in zip(whole.results(), sc.results()):
        assert np.array_equal(a, b)


def test_packed_work_items_agree():
    """Packed and spread work items give the same bits."""
    tabs, xs, lats = seed_setup(2, namp=12, nang=3)
    res = []
    for pack in (False, True):
        sc = Scan(tabs, xs, aperture_radius=0.03)
        sc.configure(variant=2, chunk=128)
        sc.set_packing(pack)
        assert sc.packing() == pack
        sc.run(200, turns_per_block=50)
        res.append(sc.results())
    for a, b in zip(*res):
        assert np.array_equal(a, b)
