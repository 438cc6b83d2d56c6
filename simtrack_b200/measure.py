"""Throughput measurements beyond bench.py's headline workload.

`python -m simtrack_b200.measure spin` times spin tracking (Track_Spin on
the GPU) of the EIC-like ring: `nseed` error seeds x `n` particles each, all
seeds' launches issued on their own CUDA streams and timed together with CUDA
events; prints one JSON line.  `python -m simtrack_b200.measure radial` does
the same for Track_Radial on the RHIC-like ring.  `python -m
simtrack_b200.measure launch --case quad --variant 1 --particles 1048576
--turns 1` runs exactly two launches of the tracking kernel (a warm-up and
the timed one) on one single-type lattice or the ring, the form the ncu
summaries capture.  `python -m simtrack_b200.measure contraction --turns 1000` compares the FMA-contracted
kernel with the strict one on the RHIC-like ring's DA grid (divergence, DA,
loss turns, throughput).  `python -m simtrack_b200.measure elements` times
the tracking kernel on single-type
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
    chosen = []
    if spin:  # launch variant per seed table, tuned on its own particles
        for t, c in zip(tabs, coords):
            chosen.append(t.autotune(c, 1, radius)["chosen"])
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
            "flops_per_particle_turn": flops, "tflops": pt * flops / (ms * 1e-3) / 1e12, "alive": [alive0, alive1],
            "variants": sorted(set(chosen))}
    print(json.dumps(line))
    return line


def _single_type_lattice(name: str):
    """The single-type lattices of element_costs (name: drift, quad, sbend,
    sext, mult, bb6d, rfcav), or the RHIC-like ring with seed-1 errors (rhic)."""
    from .lattices import ElementSpec as S, Lattice, mult_args
    if name == "rhic":
        return lattices.rhic_like_ring(seed=1)
    gamma = 100000.0 / lattices.PROTON_MASS_MEV
    err = [0.0, 0.29] + [1e-4 * (-1) ** k * math.factorial(k) / 0.031 ** (k - 1) * 0.29 for k in range(2, 10)] + [0.0]
    cases = {
        "drift": ([("DRIFT", (1.0,))], 400),
        "quad": ([("QUAD", (1.1, 0.1, 0.0), {"Nint": 4}), ("QUAD", (1.1, -0.1, 0.0), {"Nint": 4})], 200),
        "sbend": ([("SBEND", (5.8, 0.0145, 0.0, 0.0))], 400),
        "sext": ([("SEXT", (0.0, 0.6, 0.0))], 400),
        "mult": ([("MULT", mult_args(2.0, err, [0.0] * 11), {"Nint": 8}),
                  ("MULT", mult_args(2.0, [-e for e in err], [0.0] * 11), {"Nint": 8})], 20),
        "bb6d": ([("BEAMBEAM", (6, 2e11, 1.0, 0.3, 5, 2.4e-8, 0.6, 0.0, 2.4e-8, 0.6, 0.0))], 100),
        "rfcav": ([("RFCAV", (0.0, 3.0, 197e6, 0.0))], 200),
    }
    specs, reps = cases[name]
    els = [S(sp[0], f"e{r}_{i}", sp[1], sp[2] if len(sp) > 2 else {}) for r in range(reps) for i, sp in enumerate(specs)]
    return Lattice("mb_" + name, els, gamma)


def one_launch(case: str = "rhic", n: int = 1 << 20, variant: int = 1, nturn: int = 1, device: int = 0) -> dict:
    """Exactly two launches of the tracking kernel with a fixed launch variant
    (a warm-up turn, then `nturn` turns timed with CUDA events) on one lattice
    of _single_type_lattice: the form profilers capture (skip one launch,
    capture one).  Gaussian beam for the ring, small offsets for the
    single-type lattices.  Prints one JSON line."""
    import torch
    from .api import variant_name
    lat = _single_type_lattice(case)
    if case == "rhic":
        X = lattices.gaussian_beam(lattices.rhic_like_ring(seed=None, bb=False), n, seed=7)
    else:
        rng = np.random.default_rng(1)
        X = np.zeros((n, 6))
        X[:, 0] = rng.normal(0, 1e-4, n)
        X[:, 2] = rng.normal(0, 1e-4, n)
        X[:, 5] = rng.normal(0, 1e-4, n)
    tab = Table(lattices.build_line(lat), device)
    tab.set_variant(variant)
    dev = torch.device("cuda", device)
    c = [torch.tensor(np.ascontiguousarray(X[:, k]), device=dev) for k in range(6)]
    lt = torch.full((n,), -1, dtype=torch.int32, device=dev)
    le = torch.zeros(n, dtype=torch.int32, device=dev)
    r = lat.aperture_radius
    tab.track_device(c, lt, le, 0, 1, r)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    tab.track_device(c, lt, le, 1, nturn, r)
    e1.record()
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / nturn
    info = tab.info()
    out = {"case": case, "particles": n, "variant": variant_name(variant), "ms_per_turn": ms,
           "elements": info["elements"], "flops_per_turn": info["flops_per_turn"],
           "tflops": info["flops_per_turn"] * n / (ms * 1e-3) / 1e12,
           "ps_per_element_particle": ms * 1e9 / (n * info["elements"]), "alive": int((lt < 0).sum())}
    print(json.dumps(out))
    return out


def spin_launch(n: int = 2048, variant: int = 10, nturn: int = 3, seed: int = 1, device: int = 0) -> dict:
    """Exactly two launches of the spin kernel with a fixed launch variant on
    one seed of the EIC-like ring (a warm-up turn, then `nturn` turns timed
    with CUDA events): the form the spin kernel's profile captures.  Prints
    one JSON line."""
    import torch
    from .api import spin_variant_name
    lat = lattices.eic_like_ring(seed=seed)
    tab = SpinTable(lattices.build_line(lat), device)
    tab.set_variant(variant)
    X = _beam(lat, n, 1000 + seed, True)
    dev = torch.device("cuda", device)
    c = [torch.tensor(np.ascontiguousarray(X[:, k]), device=dev) for k in range(9)]
    lt = torch.full((n,), -1, dtype=torch.int32, device=dev)
    le = torch.zeros(n, dtype=torch.int32, device=dev)
    r = lat.aperture_radius
    tab.track_device(c, lt, le, 0, 1, r)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    tab.track_device(c, lt, le, 1, nturn, r)
    e1.record()
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / nturn
    f = tab.info()["flops_per_turn"]
    out = {"case": "eic_spin", "particles": n, "variant": spin_variant_name(variant), "ms_per_turn": ms,
           "particle_turns_per_s": n / (ms * 1e-3), "tflops": f * n / (ms * 1e-3) / 1e12,
           "alive": int((lt < 0).sum())}
    print(json.dumps(out))
    return out


def compaction(nseed: int = 64, n: int = 16384, device: int = 0) -> dict:
    """Two turn blocks of one turn each of a batched scan with nseed seeds x n
    Gaussian particles (spread work items of 256, the L1 variant), every
    particle alive: the form the compaction kernels are profiled in (each
    block ends with the four compaction passes over all live particles).
    Prints one JSON line."""
    from .api import Scan
    lats = [lattices.rhic_like_ring(seed=s + 1) for s in range(nseed)]
    tabs = [Table(lattices.build_line(lat), device) for lat in lats]
    base = lattices.rhic_like_ring(seed=None, bb=False)
    xs = [lattices.gaussian_beam(base, n, seed=100 + s) for s in range(nseed)]
    sc = Scan(tabs, xs, aperture_radius=lats[0].aperture_radius, device=device)
    sc.configure(variant=2, chunk=256)
    sc.run(2, turns_per_block=1, use_graph=False)
    out = {"measure": "scan compaction", "seeds": nseed, "particles": sc.n, "stats": sc.stats()}
    print(json.dumps(out))
    return out


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


def contraction(nturn: int = 1000, every: int = 10, n_rate: int = 1 << 20, rate_turns: int = 4, device: int = 0,
                seed: int = 1) -> dict:
    """The fast contraction policy (FMA-contracted kernel) against the strict
    kernel on the DA grid of the RHIC-like ring (64 amplitudes x 11 angles x 5
    momentum offsets): per particle the first checked turn at which any
    coordinate differs from the strict trajectory by more than 1e-12
    relative (rms floor per coordinate), the DA per ray of both, and the loss
    turns away from each ray's boundary; plus both kernels' particle-turns/s
    on n_rate Gaussian particles.  Prints one JSON line."""
    import torch
    from .da import da_from_lost
    dev = torch.device("cuda", device)
    lat = lattices.rhic_like_ring(seed=seed)
    namp, amax, nang, deltas = 64, 12.0, 11, [-1e-3, -5e-4, 0.0, 5e-4, 1e-3]
    X = lattices.da_grid(lat, namp, amax, nang, deltas)
    n = len(X)
    tabs = {}
    for pol in ("strict", "fast"):
        t = Table(lattices.build_line(lat), device)
        t.set_contraction(pol)
        tabs[pol] = t
    st = {p: [torch.tensor(np.ascontiguousarray(X[:, k]), device=dev) for k in range(6)] for p in tabs}
    lost = {p: (torch.full((n,), -1, dtype=torch.int32, device=dev), torch.zeros(n, dtype=torch.int32, device=dev))
            for p in tabs}
    first_div = torch.full((n,), -1, dtype=torch.int64, device=dev)
    r = lat.aperture_radius
    for t0 in range(0, nturn, every):
        k = min(every, nturn - t0)
        for p, t in tabs.items():
            t.track_device(st[p], lost[p][0], lost[p][1], t0, k, r)
        a = torch.stack(st["strict"], 1)
        b = torch.stack(st["fast"], 1)
        both = (lost["strict"][0] < 0) & (lost["fast"][0] < 0)
        floor = torch.sqrt(torch.mean(a[both] ** 2, 0)) if both.any() else torch.ones(6, device=dev)
        rel = ((a - b).abs() / torch.maximum(a.abs(), floor)).amax(1)
        diverged = (rel > 1e-12) | (lost["strict"][0] != lost["fast"][0])
        first_div = torch.where((first_div < 0) & diverged, torch.full_like(first_div, t0 + k), first_div)
    torch.cuda.synchronize(dev)
    fd = first_div.cpu().numpy()
    lts = lost["strict"][0].cpu().numpy().reshape(len(deltas) * nang, namp)
    ltf = lost["fast"][0].cpu().numpy().reshape(len(deltas) * nang, namp)
    amps = np.linspace(0.0, amax, namp)
    da_s, da_f = da_from_lost(lts, amps, nturn), da_from_lost(ltf, amps, nturn)
    step = amps[1] - amps[0]

    def first_lost(lt_):
        lostm = (lt_ >= 0) & (lt_ < nturn)
        return np.where(lostm.any(1), np.argmax(lostm, 1), namp)

    b = first_lost(lts)
    far = np.abs(np.arange(namp)[None, :] - b[:, None]) > 1
    surv = lts < 0
    out = {"measure": "contraction policy divergence", "ring": "RHIC-like", "seed": seed, "particles": n,
           "turns": nturn, "checked_every": every,
           "diverged_particles": int((fd >= 0).sum()),
           "surviving_particles_strict": int(surv.sum()),
           "first_divergence_turn_percentiles": {q: (float(np.percentile(fd[fd >= 0], q)) if (fd >= 0).any() else None)
                                                 for q in (5, 25, 50, 75, 95)},
           "never_diverged_survivors": int(((fd < 0) & surv.ravel()).sum()),
           "rays": int(len(b)), "rays_da_differs": int((da_s != da_f).sum()),
           "max_da_difference_sigma": float(np.max(np.abs(da_s - da_f))), "amplitude_step_sigma": float(step),
           "loss_turn_mismatches_away_from_boundary": int((lts[far] != ltf[far]).sum()),
           "particles_away_from_boundary": int(far.sum())}
    # throughput of both kernels on the Gaussian throughput workload
    Xg = lattices.gaussian_beam(lattices.rhic_like_ring(seed=None, bb=False), n_rate, seed=12345)
    rates = {}
    for pol, t in tabs.items():
        c = [torch.tensor(np.ascontiguousarray(Xg[:, k]), device=dev) for k in range(6)]
        tune = t.autotune(c, 1, r)
        lt_ = torch.full((n_rate,), -1, dtype=torch.int32, device=dev)
        le_ = torch.zeros(n_rate, dtype=torch.int32, device=dev)
        t.track_device(c, lt_, le_, 0, 1, r)
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        t.track_device(c, lt_, le_, 1, rate_turns, r)
        e1.record()
        torch.cuda.synchronize(dev)
        ms = e0.elapsed_time(e1)
        alive = int((lt_ < 0).sum())
        rates[pol] = {"particle_turns_per_s": alive * rate_turns / (ms * 1e-3), "variant": tune["chosen"],
                      "flops_per_particle_turn": t.info()["flops_per_turn"]}
    out["throughput"] = rates
    print(json.dumps(out))
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("kind", choices=["spin", "radial", "elements", "contraction", "launch", "compaction",
                                     "spin_launch"])
    ap.add_argument("--case", default="rhic")
    ap.add_argument("--variant", type=int, default=1)
    ap.add_argument("--seeds", type=int, default=16)
    ap.add_argument("--particles", type=int, default=2048)
    ap.add_argument("--turns", type=int, default=200)
    a = ap.parse_args(argv)
    if a.kind == "elements":
        element_costs()
    elif a.kind == "contraction":
        contraction(nturn=a.turns)
    elif a.kind == "launch":
        one_launch(a.case, a.particles, a.variant, a.turns)
    elif a.kind == "compaction":
        compaction(a.seeds, a.particles)
    elif a.kind == "spin_launch":
        spin_launch(a.particles, a.variant, a.turns)
    else:
        run(a.kind, a.seeds, a.particles, a.turns)


if __name__ == "__main__":
    main()
