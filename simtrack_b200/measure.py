"""Throughput measurements beyond bench.py's headline workload.

`python -m simtrack_b200.measure spin` times spin tracking (Track_Spin on
the GPU) of the EIC-like ring: `nseed` error seeds x `n` particles each, all
seeds' launches issued on their own CUDA streams and timed together with CUDA
events; prints one JSON line.  `python -m simtrack_b200.measure radial` does
the same for Track_Radial on the RHIC-like ring.
"""
from __future__ import annotations

import argparse
import json
import math

import numpy as np

from . import lattices
from .api import SpinTable, Table


def _beam(lat, n, seed, spin):
    rng = np.random.default_rng(seed)
    X = lattices.gaussian_beam(lat, n, seed=seed)
    if not spin:
        return X
    s = rng.normal(0, 1, (n, 3)) * [0.05, 1.0, 0.05]
    s /= np.linalg.norm(s, axis=1, keepdims=True)
    return np.concatenate([X, s], axis=1)


def run(kind: str = "spin", nseed: int = 16, n: int = 2048, nturn: int = 200, warmup: int = 20, device: int = 0):
    import torch
    dev = torch.device("cuda", device)
    spin = kind == "spin"
    tabs, coords, losts, flops = [], [], [], 0.0
    for s in range(nseed):
        lat = lattices.eic_like_ring(seed=s + 1) if spin else lattices.rhic_like_ring(seed=s + 1)
        line = lattices.build_line(lat)
        t = SpinTable(line, device) if spin else Table(line, device)
        tabs.append(t)
        X = _beam(lat, n, 1000 + s, spin)
        coords.append([torch.tensor(np.ascontiguousarray(X[:, k]), device=dev) for k in range(X.shape[1])])
        losts.append((torch.full((n,), -1, dtype=torch.int32, device=dev), torch.zeros(n, dtype=torch.int32,
                                                                                      device=dev)))
        flops = t.info()["flops_per_turn"]
    radius = lat.aperture_radius
    streams = [torch.cuda.Stream(dev) for _ in range(nseed)]

    def launch(turn0, nt):
        for t, c, (lt, le), st in zip(tabs, coords, losts, streams):
            if spin:
                t.track_device(c, lt, le, turn0, nt, radius, st.cuda_stream)
            else:
                t.track_radial_device(c, lt, le, turn0, nt, radius, st.cuda_stream)

    launch(0, warmup)
    torch.cuda.synchronize(dev)
    alive0 = sum(int((lt < 0).sum()) for lt, _ in losts)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    cur = torch.cuda.current_stream(dev)
    e0.record(cur)
    for st in streams:
        st.wait_event(e0)
    launch(warmup, nturn)
    for st in streams:
        cur.wait_stream(st)
    e1.record(cur)
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1)
    alive1 = sum(int((lt < 0).sum()) for lt, _ in losts)
    pt = 0.5 * (alive0 + alive1) * nturn
    line = {"measure": f"{kind} tracking", "ring": "EIC-like (spin)" if spin else "RHIC-like (Track_Radial)",
            "seeds": nseed, "particles_per_seed": n, "turns": nturn, "ms": ms, "particle_turns_per_s": pt / (ms * 1e-3),
            "flops_per_particle_turn": flops, "tflops": pt * flops / (ms * 1e-3) / 1e12, "alive": [alive0, alive1]}
    print(json.dumps(line))
    return line


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("kind", choices=["spin", "radial"])
    ap.add_argument("--seeds", type=int, default=16)
    ap.add_argument("--particles", type=int, default=2048)
    ap.add_argument("--turns", type=int, default=200)
    a = ap.parse_args(argv)
    run(a.kind, a.seeds, a.particles, a.turns)


if __name__ == "__main__":
    main()
