"""Dynamic-aperture scans on the GPU.

The reference finds the DA angle by angle with a bisection of twin-particle
Track() calls (Track_DA, simtrack.cpp:21389-21441) or by a radial sweep that
stops at the first loss (Track_DA_Radial_Uniform, simtrack.cpp:21736-21764).
Here every initial condition of a grid (amplitudes x angles x momentum
offsets, for every error seed) is tracked at once by the batched scan, and the
DA of a ray is read off the loss turns: the largest grid amplitude below which
every particle of the ray survived all turns.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from . import lattices
from .api import Scan, Table


@dataclass
class DAResult:
    nseed: int
    namp: int
    nang: int
    deltas: List[float]
    amax: float
    nturn: int
    lost_turn: np.ndarray  # [nseed, ndelta, nang, namp], -1 = survived
    da: np.ndarray         # [nseed, ndelta, nang] in units of sigma
    wall_s: float = 0.0
    device_ms: float = 0.0
    stats: dict = field(default_factory=dict)

    @property
    def da_per_angle(self) -> np.ndarray:
        """[nseed, nang]: minimum over momentum offsets."""
        return self.da.min(axis=1)


def da_from_lost(lost_turn: np.ndarray, amps: np.ndarray, nturn: int) -> np.ndarray:
    """lost_turn [..., namp] (-1 or >= nturn: survived) -> DA [...]: the largest
    amplitude a_k such that every amplitude <= a_k survived (0 if the first
    grid point is lost)."""
    surv = (lost_turn < 0) | (lost_turn >= nturn)
    # index of the first lost amplitude along the last axis
    first_lost = np.where(~surv, np.arange(surv.shape[-1]), surv.shape[-1]).min(axis=-1)
    out = np.where(first_lost > 0, amps[np.maximum(first_lost - 1, 0)], 0.0)
    return out


def grids_for(lats: Sequence[lattices.Lattice], namp, amax, nang, deltas):
    return [lattices.da_grid(lat, namp, amax, nang, deltas) for lat in lats]


def rhic_da_scan(nseed: int = 64, namp: int = 64, amax: float = 12.0, nang: int = 11,
                 deltas: Sequence[float] = (-1e-3, -5e-4, 0.0, 5e-4, 1e-3), nturn: int = 100000,
                 turns_per_block: int = 256, use_graph: bool = True, device: int = 0, seed0: int = 1,
                 variant: int = -1, chunk: int = 0, particle_mask: Optional[np.ndarray] = None) -> DAResult:
    """Batched DA scan of the RHIC-like ring with seeds seed0..seed0+nseed-1
    (64 amplitudes 0..12 sigma x 11 angles x 5 momentum offsets per seed by
    default).  particle_mask [nseed, ndelta, nang, namp] (optional) restricts
    tracking to the selected initial conditions; the others count as lost at
    turn 0 in the result only if they are not tracked (see DAResult.lost_turn)."""
    lats = [lattices.rhic_like_ring(seed=seed0 + s) for s in range(nseed)]
    tables = [Table(lattices.build_line(lat), device) for lat in lats]
    grids = grids_for(lats, namp, amax, nang, deltas)
    nd = len(deltas)
    if particle_mask is not None:
        m = particle_mask.reshape(nseed, -1)
        grids = [g[m[s]] for s, g in enumerate(grids)]
    t0 = time.perf_counter()
    sc = Scan(tables, grids, aperture_radius=lats[0].aperture_radius, device=device)
    if variant >= 0 or chunk > 0:
        sc.configure(variant, chunk)
    else:
        sc.autotune(nturn=min(16, max(1, nturn)))
    sc.run(nturn, turns_per_block, use_graph)
    lt, le, x = sc.results()
    wall = time.perf_counter() - t0
    full = np.full((nseed, nd * nang * namp), -1, dtype=np.int64)
    off = 0
    for s in range(nseed):
        n = len(grids[s])
        if particle_mask is not None:
            full[s, m[s]] = lt[off:off + n]
        else:
            full[s] = lt[off:off + n]
        off += n
    full = full.reshape(nseed, nd, nang, namp)
    amps = np.linspace(0.0, amax, namp)
    st = sc.stats()
    return DAResult(nseed, namp, nang, list(deltas), amax, nturn, full, da_from_lost(full, amps, nturn),
                    wall_s=wall, device_ms=st["device_ms"], stats=st)


def sharded_da_scan(nseed: int = 64, scan=None, **kw) -> Optional[DAResult]:
    """A DA scan over seeds seed0..seed0+nseed-1 split across the ranks of
    the default process group (contiguous seed shares, no exchange while
    tracking); the per-seed loss turns are gathered to every rank in seed
    order and the full result is returned (wall time: slowest rank).
    `scan(nseed=, seed0=, **kw) -> DAResult` runs one rank's share
    (rhic_da_scan, the batched GPU scan, by default)."""
    from .parallel import gather_concat, reduce_scalar, shard_bounds
    import torch.distributed as dist
    scan = scan or rhic_da_scan
    world = dist.get_world_size() if dist.is_available() and dist.is_initialized() else 1
    rank = dist.get_rank() if world > 1 else 0
    seed0 = kw.pop("seed0", 1)
    lo, hi = shard_bounds(nseed, rank, world)
    part = scan(nseed=hi - lo, seed0=seed0 + lo, **kw) if hi > lo else None
    namp = kw.get("namp", 64)
    nang = kw.get("nang", 11)
    deltas = list(kw.get("deltas", (-1e-3, -5e-4, 0.0, 5e-4, 1e-3)))
    amax = kw.get("amax", 12.0)
    nturn = kw.get("nturn", 100000)
    shape = (len(deltas), nang, namp)
    local = part.lost_turn if part is not None else np.zeros((0,) + shape, dtype=np.int64)
    full = gather_concat(local.astype(np.int64))
    wall = reduce_scalar(part.wall_s if part is not None else 0.0, "max")
    amps = np.linspace(0.0, amax, namp)
    return DAResult(nseed, namp, nang, deltas, amax, nturn, full, da_from_lost(full, amps, nturn), wall_s=wall)
