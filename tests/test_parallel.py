"""Sharding and the rank collectives of the multi-GPU path, as world-size-2
gloo process groups on the CPU (127.0.0.1 rendezvous)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from simtrack_b200.parallel import seeds_for_rank, shard_bounds


def test_shard_bounds_cover_exactly():
    for n in (0, 1, 7, 64, 1048576, 1048577):
        for world in (1, 2, 3, 8):
            spans = [shard_bounds(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            for (a, b), (c, d) in zip(spans, spans[1:]):
                assert b == c
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1
    assert seeds_for_rank(list(range(1, 65)), 1, 2) == list(range(33, 65))
    with pytest.raises(ValueError):
        shard_bounds(10, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    from simtrack_b200.parallel import gather_concat, reduce_scalar
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # per-rank "device time" and particle count, as bench.py reduces them
        tmax = reduce_scalar(10.0 + rank, "max")
        ntot = reduce_scalar(100 * (rank + 1), "sum")
        # uneven per-rank results (lost turns of each rank's particle shard)
        lo, hi = shard_bounds(5, rank, world)
        lost = np.arange(lo, hi, dtype=np.int32) * 10
        rows = np.stack([np.arange(lo, hi), np.arange(lo, hi) * 2], axis=1).astype(np.float64)
        g1 = gather_concat(lost)
        g2 = gather_concat(rows)
        q.put((rank, tmax, ntot, g1.tolist(), g2.tolist()))
    finally:
        dist.destroy_process_group()


def test_gloo_two_ranks_reduce_and_gather():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, tmax, ntot, g1, g2 in out:
        assert tmax == 11.0
        assert ntot == 300.0
        assert g1 == [0, 10, 20, 30, 40]
        assert g2 == [[i, 2 * i] for i in range(5)]


def fake_scan(nseed, seed0, namp=16, nang=3, deltas=(-1e-3, 0.0, 1e-3), amax=12.0, nturn=1000):
    """Stands in for one rank's batched GPU scan: a deterministic loss pattern
    per (seed, momentum offset, angle, amplitude)."""
    from simtrack_b200.da import DAResult, da_from_lost
    nd = len(deltas)
    lt_ = np.full((nseed, nd, nang, namp), -1, dtype=np.int64)
    for s in range(nseed):
        sd = seed0 + s
        for d in range(nd):
            for a in range(nang):
                edge = (3 * sd + 5 * d + 7 * a) % namp
                lt_[s, d, a, edge:] = 10 * sd + np.arange(namp - edge)
    amps = np.linspace(0.0, amax, namp)
    return DAResult(nseed, namp, nang, list(deltas), amax, nturn, lt_, da_from_lost(lt_, amps, nturn), wall_s=1.0 + s)


def _scan_worker(rank, world, port, nseed, q):
    import datetime

    import torch.distributed as dist

    from simtrack_b200.da import sharded_da_scan
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        r = sharded_da_scan(nseed=nseed, scan=fake_scan, seed0=5, namp=16, nang=3, deltas=(-1e-3, 0.0, 1e-3),
                            amax=12.0, nturn=1000)
        q.put((rank, r.lost_turn.tolist(), r.da.tolist(), r.wall_s))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,nseed", [(2, 7), (3, 7), (3, 2)])
def test_sharded_scan_gathers_seeds_in_order(world, nseed):
    """Seed sharding across gloo ranks, the gather order and the DA assembly
    equal one process scanning every seed (a rank may get no seeds)."""
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_scan_worker, args=(r, world, port, nseed, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    whole = fake_scan(nseed, 5)
    for rank, lt_, da, wall in out:
        assert np.array_equal(np.array(lt_), whole.lost_turn)
        assert np.array_equal(np.array(da), whole.da)
        assert wall >= 1.0
