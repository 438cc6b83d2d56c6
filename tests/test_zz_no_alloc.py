"""stb_track_seeds_static (static device scratch, no allocation) against
stb_track_device on each seed table, over two calls in a row (needs a B200).

Collected last on purpose: it must pass both in a fresh process and after
every other test has used the device."""
import ctypes

import numpy as np
import pytest

from simtrack_b200 import lattices as lt
from simtrack_b200._native import STB_EINVAL, lib
from simtrack_b200.api import Table, track_seeds_static

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _setup():
    lats = [lt.rhic_like_ring(seed=1), lt.rhic_like_ring(seed=2), lt.fodo_ring()]
    tabs = [Table(lt.build_line(lat)) for lat in lats]
    a = np.linspace(0.0, 0.04, 48)
    fodo = np.zeros((len(a), 6))
    fodo[:, 0] = a
    fodo[:, 2] = 0.5 * a
    fodo[:, 5] = 2e-4
    xs = [lt.da_grid(lats[0], 24, 14.0, 4, [0.0, 5e-4]),
          lt.da_grid(lats[1], 20, 14.0, 3, [-5e-4]),
          fodo]
    return tabs, xs


def test_static_matches_track_device_two_calls():
    tabs, xs = _setup()
    n_per = [len(x) for x in xs]
    n = sum(n_per)
    x0 = np.concatenate(xs, axis=0)
    dev = torch.device("cuda:0")
    coords = torch.tensor(x0.T.copy(), dtype=torch.float64, device=dev).contiguous()
    lost_turn = torch.full((n,), -1, dtype=torch.int32, device=dev)
    lost_elem = torch.zeros(n, dtype=torch.int32, device=dev)
    ref_c = [torch.tensor(x.T.copy(), dtype=torch.float64, device=dev).contiguous() for x in xs]
    ref_lt = [torch.full((len(x),), -1, dtype=torch.int32, device=dev) for x in xs]
    ref_le = [torch.zeros(len(x), dtype=torch.int32, device=dev) for x in xs]
    turn0 = 0
    for nturn in (150, 170):
        track_seeds_static(tabs, n_per, coords, lost_turn, lost_elem, turn0, nturn, 0.03)
        for s, t in enumerate(tabs):
            t.track_device([ref_c[s][k] for k in range(6)], ref_lt[s], ref_le[s], turn0, nturn, 0.03)
        torch.cuda.synchronize()
        turn0 += nturn
        got_c = coords.cpu().numpy()
        got_lt = lost_turn.cpu().numpy()
        got_le = lost_elem.cpu().numpy()
        off = 0
        for s in range(len(tabs)):
            m = n_per[s]
            exp_c = ref_c[s].cpu().numpy()
            # identical arithmetic in the same order: bit-exact agreement
            assert np.array_equal(got_c[:, off:off + m], exp_c), f"seed {s} after turn {turn0}"
            assert np.array_equal(got_lt[off:off + m], ref_lt[s].cpu().numpy()), f"seed {s}"
            assert np.array_equal(got_le[off:off + m], ref_le[s].cpu().numpy()), f"seed {s}"
            off += m
    lost = got_lt >= 0
    assert lost.any() and (~lost).any()  # the grids straddle the dynamic aperture


def test_static_rejects_oversize_requests():
    """Through the C ABI with NULL buffers: the size limits are checked before
    anything touches the device."""
    tabs, xs = _setup()

    def call(tables, n_per):
        arr = (ctypes.c_void_p * len(tables))(*[t._h for t in tables])
        nps = (ctypes.c_long * len(n_per))(*n_per)
        return lib().stb_track_seeds_static(arr, len(tables), nps, *([None] * 8), 0, 10, 0.0, None)

    assert call(tabs[:1], [1 << 21]) == STB_EINVAL
    assert b"particles" in lib().stb_last_error()
    assert call(tabs[:1] * 65, [1] * 65) == STB_EINVAL
    assert b"seed count" in lib().stb_last_error()


def test_python_wrapper_checks_buffers():
    tabs, xs = _setup()
    dev = torch.device("cuda:0")
    n = 10
    c = torch.zeros((6, n), dtype=torch.float64, device=dev)
    lt_ = torch.full((n,), -1, dtype=torch.int32, device=dev)
    le_ = torch.zeros(n, dtype=torch.int32, device=dev)
    with pytest.raises(ValueError):
        track_seeds_static(tabs[:1], [n + 1], c, lt_, le_, 0, 1)
    with pytest.raises(ValueError):
        track_seeds_static(tabs[:1], [n], c.float(), lt_, le_, 0, 1)
    with pytest.raises(ValueError):
        track_seeds_static(tabs[:1], [n], c, lt_.long(), le_, 0, 1)
    with pytest.raises(ValueError):
        track_seeds_static(tabs[:1], [n], c.cpu(), lt_, le_, 0, 1)
