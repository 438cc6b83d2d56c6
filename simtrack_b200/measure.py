"""Throughput measurements beyond bench.py's headline workload.

`python -m simtrack_b200.measure spin` times spin tracking (Track_Spin on
the GPU) of the EIC-like ring: `nseed` error seeds x `n` particles each, all
seeds' launches issued on their own CUDA streams and timed together with CUDA
events; prints one JSON line.  `python -m simtrack_b200.measure radial` does
the same for Track_Radial on the RHIC-like ring.  `python -m
simtrack_b200.measure elements` times the tracking kernel on single-type
lattices (400 identical drifts, thick quadrupoles, sector bends, thin
sextupoles; 40 thick multipoles of order 9; 100 beam-beam maps; 200 RF
cavities) over 1,048,576 particles: the per-element-type cost behind the
RHIC-like ring's turn time.
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


def element_costs(n: int = 1 << 20, device: int = 0) -> dict:
    """Picoseconds per element-particle of the autotuned tracking kernel on
    single-type lattices (one JSON line per type)."""
    import torch
    from .lattices import ElementSpec as S, Lattice, mult_args
    gamma = 100000.0 / lattices.PROTON_MASS_MEV
    err = [0.0, 0.29] + [1e-4 * (-1) ** k * math.factorial(k) / 0.031 ** (k - 1) * 0.29 for k in range(2, 10)] + [0.0]
    cases = {
        "drift": ([("DRIFT", (1.0,))], 400),
        "quad_thick_nint4": ([("QUAD", (1.1, 0.1, 0.0), {"Nint": 4}), ("QUAD", (1.1, -0.1, 0.0), {"Nint": 4})], 200),
        "sbend": ([("SBEND", (5.8, 0.0145, 0.0, 0.0))], 400),
        "sext_thin": ([("SEXT", (0.0, 0.6, 0.0))], 400),
        "mult_thick_nint8_order9": ([("MULT", mult_args(2.0, err, [0.0] * 11), {"Nint": 8}),
                                     ("MULT", mult_args(2.0, [-e for e in err], [0.0] * 11), {"Nint": 8})], 20),
        "bb6d_5slices": ([("BEAMBEAM", (6, 2e11, 1.0, 0.3, 5, 2.4e-8, 0.6, 0.0, 2.4e-8, 0.6, 0.0))], 100),
        "rfcav_thin": ([("RFCAV", (0.0, 3.0, 197e6, 0.0))], 200),
    }
    rng = np.random.default_rng(1)
    X = np.zeros((n, 6))
    X[:, 0] = rng.normal(0, 1e-4, n)
    X[:, 2] = rng.normal(0, 1e-4, n)
    X[:, 5] = rng.normal(0, 1e-4, n)
    dev = torch.device("cuda", device)
    out = {}
    for name, (specs, reps) in cases.items():
        els = [S(sp[0], f"e{r}_{i}", sp[1], sp[2] if len(sp) > 2 else {}) for r in range(reps)
               for i, sp in enumerate(specs)]
        tab = Table(lattices.build_line(Lattice("mb", els, gamma)), device)
        coords = [torch.tensor(np.ascontiguousarray(X[:, k]), device=dev) for k in range(6)]
        tune = tab.autotune(coords, 1)
        lost = torch.full((n,), -1, dtype=torch.int32, device=dev)
        le = torch.zeros(n, dtype=torch.int32, device=dev)
        tab.track_device(coords, lost, le, 1, 1)
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        tab.track_device(coords, lost, le, 2, 2)
        e1.record()
        torch.cuda.synchronize(dev)
        ms = e0.elapsed_time(e1) / 2
        info = tab.info()
        ne = info["elements"]
        out[name] = {"ps_per_element_particle": ms * 1e9 / (n * ne), "flops_per_element": info["flops_per_turn"] / ne,
                     "tflops": info["flops_per_turn"] * n / (ms * 1e-3) / 1e12, "variant": tune["chosen"],
                     "elements": ne, "ms_per_turn": ms, "alive": int((lost < 0).sum())}
        print(json.dumps({name: out[name]}), flush=True)
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("kind", choices=["spin", "radial", "elements"])
    ap.add_argument("--seeds", type=int, default=16)
    ap.add_argument("--particles", type=int, default=2048)
    ap.add_argument("--turns", type=int, default=200)
    a = ap.parse_args(argv)
    if a.kind == "elements":
        element_costs()
    else:
        run(a.kind, a.seeds, a.particles, a.turns)


if __name__ == "__main__":
    main()
