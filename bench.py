"""Benchmark: FP64 particle-turns/s of element-by-element tracking on one B200.

Workload (the throughput run of the synthetic RHIC-like ring): 1,810
elements (216 arc FODO cells, two low-beta triplet IRs with seeded b3..b10 /
a3..a10 errors, 6D weak-strong beam-beam at both IPs, RF at 28/197 MHz,
circular 30 mm aperture), 1,048,576 particles from a seeded 6D Gaussian,
FP64.  One step = one launch of the tracking kernel over all particles for
`--turns-per-step` turns.  Inputs are resident in HBM when the timed region
starts; a 256 MiB buffer is written between timed steps to flush L2 (the
particle arrays, 48 MiB, would otherwise stay L2-resident).

Prints one JSON line.  `--impl reference` times the reference's own CPU
Track() (oracle/_ref compiled from the SimTrack source; the C restatement
oracle/port where that was not built) on the host cores, one worker process
per core, on a bounded sample of the same workload.

Multi-GPU (torchrun, one rank per GPU): particles shard with no data-path
exchange.  Each rank tracks its own 1,048,576 particles (weak scaling); the
step time is the max over ranks of the device time, `value` the particle-turns
of all ranks divided by it.
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "FP64 particle-turns/s"
UNIT = "particle-turns/s"
WORKLOAD = "RHIC-like ring (1,810 elements, seed-1 IR errors, 2 BB6D IPs) x 1,048,576 Gaussian particles, FP64"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--particles", type=int, default=1 << 20)
    ap.add_argument("--turns-per-step", type=int, default=4)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-procs", type=int, default=0)
    ap.add_argument("--variant", type=int, default=-1, help="force a kernel launch variant (skips the autotuner)")
    return ap.parse_args()


# ----------------------------------------------------------------------------
# CPU baseline: the reference's Track() on host cores (oracle; measurement only)

def _cpu_kind():
    return "reference" if (ROOT / "oracle" / "_ref" / "libsimtrack_ref.so").exists() else "port"


def _cpu_worker(args):
    seed, x_chunk, nturn, reps = args
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_bridge
    from simtrack_b200 import lattices
    lat = lattices.rhic_like_ring(seed=seed)
    o = oracle_bridge.RefOracle() if _cpu_kind() == "reference" else oracle_bridge.PortOracle()
    o.build(lat)
    out = []
    for _ in range(reps):
        t0 = time.perf_counter()
        o.track(x_chunk, nturn)
        out.append((time.perf_counter() - t0, len(x_chunk) * nturn))
    return out


def cpu_rates(seed, x, nturn, reps, procs):
    """Per-rep aggregate particle-turns/s over `procs` worker processes."""
    import numpy as np
    procs = max(1, min(procs, len(x)))
    chunks = np.array_split(x, procs)
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        res = pool.map(_cpu_worker, [(seed, c, nturn, reps) for c in chunks])
    rates = []
    for r in range(reps):
        t = max(w[r][0] for w in res)
        rates.append(sum(w[r][1] for w in res) / t)
    return rates, procs


def ensure_oracle():
    if _cpu_kind() == "port" and not (ROOT / "oracle" / "_build" / "libsimtrack_port.so").exists():
        subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "port"], check=True)


def gaussian(n, seed=12345):
    from simtrack_b200 import lattices
    lat = lattices.rhic_like_ring(seed=None, bb=False)
    return lattices.gaussian_beam(lat, n, seed=seed)


# ----------------------------------------------------------------------------
# clocks sampled during the timed region

class ClockSampler:
    def __init__(self, gpu_index: int):
        vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
        ids = [v.strip() for v in vis.split(",") if v.strip()]
        gpu = ids[gpu_index] if gpu_index < len(ids) else str(gpu_index)
        self.samples, self.stop_flag, self.gpu = [], threading.Event(), gpu

    def _run(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        while not self.stop_flag.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={q}", "--format=csv,noheader,nounits"],
                                     capture_output=True, text=True, timeout=5).stdout.strip()
                if out:
                    self.samples.append([v.strip() for v in out.split(",")])
            except Exception:
                pass
            self.stop_flag.wait(0.2)

    def __enter__(self):
        self.t = threading.Thread(target=self._run, daemon=True)
        self.t.start()
        return self

    def __exit__(self, *a):
        self.stop_flag.set()
        self.t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[4 + i].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


# ----------------------------------------------------------------------------

def reused_drift_ops(lat) -> int:
    """Operations of the reference's count that the kernel does not execute a
    second time: at each Yoshida slice boundary of a thick quadrupole,
    sextupole, octupole or multipole the closing and opening drifts are
    identical, and the second one adds the first one's increments (3
    additions instead of a 16-operation drift)."""
    n = 0
    for e in lat.elements:
        if e.type in ("QUAD", "SKEWQ", "SEXT", "OCT", "MULT") and float(e.args[0]) > 0.0:
            strengths = e.args[1:] if e.type != "MULT" else e.args[1:]
            if any(float(v) != 0.0 for v in strengths):
                n += (int(e.setp.get("Nint", 1)) - 1) * (16 - 3)
    return n


def roofline_traffic():
    """DRAM bytes per launch of the tracking kernel from the committed ncu summary, if any."""
    f = ROOT / "profiles" / "track_kernel_rhic_like.md"
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        if line.startswith("traffic_bytes_per_launch_full_workload:"):
            try:
                return float(line.split(":", 1)[1].strip())
            except ValueError:
                return None
    return None


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    ensure_oracle()
    procs = a.cpu_procs or os.cpu_count() or 1
    nturn = 100
    per_proc = 16
    x = gaussian(per_proc * procs)
    rates, procs = cpu_rates(a.seed, x, nturn, a.warmup + a.steps, procs)
    timed = rates[a.warmup:]
    # whole-run rate = total particle-turns / total time of the timed reps
    pt = per_proc * procs * nturn
    total_t = sum(pt / r for r in timed)
    v = pt * len(timed) / total_t
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": 1e3 * total_t / len(timed), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "particles": per_proc * procs, "turns_per_step": nturn},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": procs, "kind": _cpu_kind(),
                             "sample": f"{procs} processes x {per_proc} particles x {nturn} turns per step"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(a):
    import numpy as np
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    # CPU baseline first (spawned processes, before any CUDA state exists).
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        ensure_oracle()
        procs = a.cpu_procs or os.cpu_count() or 1
        per_proc, nturn = 32, 2000
        xs = gaussian(per_proc * procs, seed=777)
        rates, procs = cpu_rates(a.seed, xs, nturn, 1, procs)
        cpu = {"value": rates[0], "unit": UNIT, "cores": procs, "kind": _cpu_kind(),
               "sample": f"{procs} processes x {per_proc} Gaussian particles x {nturn} turns of the same ring"}

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))

    from simtrack_b200 import lattices
    from simtrack_b200.api import Table
    from simtrack_b200.parallel import reduce_scalar
    from simtrack_b200._native import lib
    import ctypes

    lat = lattices.rhic_like_ring(seed=a.seed)
    line = lattices.build_line(lat)
    tab = Table(line, device=local)
    info = tab.info()
    n, T = a.particles, a.turns_per_step
    X = lattices.gaussian_beam(lat, n, seed=12345 + rank)
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)

    coords0 = [torch.tensor(np.ascontiguousarray(X[:, k]), device=dev) for k in range(6)]
    coords = [c.clone() for c in coords0]
    lt_ = torch.full((n,), -1, dtype=torch.int32, device=dev)
    le_ = torch.zeros(n, dtype=torch.int32, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    if a.variant >= 0:
        tab.set_variant(a.variant)
        tune = {"ms": {}}
    else:
        tune = tab.autotune(coords, nturn=1, aperture_radius=lat.aperture_radius)
    info = tab.info()

    peak = ctypes.c_double()
    rc = lib().stb_fp64_peak(local, ctypes.byref(peak))
    fp64_peak = peak.value if rc == 0 else None

    turn = 0
    for _ in range(a.warmup):
        tab.track_device(coords, lt_, le_, turn, T, lat.aperture_radius, stream.cuda_stream)
        turn += T
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    alive0 = int((lt_ < 0).sum())
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(a.steps)]
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        for s in range(a.steps):
            flush.fill_(s & 0xFF)
            evs[s][0].record(stream)
            tab.track_device(coords, lt_, le_, turn, T, lat.aperture_radius, stream.cuda_stream)
            evs[s][1].record(stream)
            turn += T
        torch.cuda.synchronize()
    ms_steps = [e0.elapsed_time(e1) for e0, e1 in evs]
    ms = sum(ms_steps)
    alive1 = int((lt_ < 0).sum())
    # particle-turns actually tracked: particles lost inside the timed region count
    # only up to their loss turn; approximate with the mean of alive counts.
    pt_rank = 0.5 * (alive0 + alive1) * T * a.steps
    # device time: max over ranks; particle-turns: sum over ranks
    ms = reduce_scalar(ms, "max")
    pt_total = reduce_scalar(pt_rank, "sum")
    value = pt_total / (ms * 1e-3)

    # The same steps with the FMA-contracted kernel (contraction policy
    # "fast"), reported beside the strict number; every rank runs it.
    tab.set_contraction("fast")
    tune_f = tab.autotune(coords0, nturn=1, aperture_radius=lat.aperture_radius) if a.variant < 0 else None
    coords_f = [c.clone() for c in coords0]
    lt_f = torch.full((n,), -1, dtype=torch.int32, device=dev)
    le_f = torch.zeros(n, dtype=torch.int32, device=dev)
    turn_f = 0
    for _ in range(a.warmup):
        tab.track_device(coords_f, lt_f, le_f, turn_f, T, lat.aperture_radius, stream.cuda_stream)
        turn_f += T
    torch.cuda.synchronize()
    alive0_f = int((lt_f < 0).sum())
    evf = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(a.steps)]
    for s_ in range(a.steps):
        flush.fill_(s_ & 0xFF)
        evf[s_][0].record(stream)
        tab.track_device(coords_f, lt_f, le_f, turn_f, T, lat.aperture_radius, stream.cuda_stream)
        evf[s_][1].record(stream)
        turn_f += T
    torch.cuda.synchronize()
    ms_f = reduce_scalar(sum(e0.elapsed_time(e1) for e0, e1 in evf), "max")
    pt_f = reduce_scalar(0.5 * (alive0_f + int((lt_f < 0).sum())) * T * a.steps, "sum")
    fast_info = tab.info()
    tab.set_contraction("strict")
    tab.set_variant(info["variant"])

    # e2e through the host-buffer C ABI (stb_track_host, the Track() form):
    # pinned host AoS coordinates and input flags in, Track()'s outputs out,
    # one call per step with its copies and layout conversion inside the
    # timed region, on every rank; whole-job rate = all ranks' particle-turns
    # over the slowest rank's time
    pin = lambda arr: torch.from_numpy(np.ascontiguousarray(arr)).pin_memory().numpy()
    xh = pin(X)
    st_h = pin(np.ones(n, dtype=np.int32))
    lt_h = pin(np.zeros(n, dtype=np.int32))
    lp_h = pin(np.zeros(n, dtype=np.int32))
    P = lambda arr, t: arr.ctypes.data_as(ctypes.POINTER(t))

    def host_call(nt):
        st_h[:] = 1
        rc_ = lib().stb_track_host(tab._h, P(xh, ctypes.c_double), n, nt, lat.aperture_radius, P(st_h, ctypes.c_int),
                                   P(lt_h, ctypes.c_int), P(lp_h, ctypes.c_int))
        if rc_ != 0:
            raise RuntimeError(f"stb_track_host failed: {lib().stb_last_error()}")

    host_call(1)  # warm-up: grows the table's device staging
    xh[:] = X
    reps = max(2, min(a.steps, 4))
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(reps):
        host_call(T)
    e2e_s = reduce_scalar(time.perf_counter() - t0, "max")
    e2e_pt = reduce_scalar(0.5 * (n + int(st_h.sum())) * T * reps, "sum")
    e2e = {"value": e2e_pt / e2e_s, "unit": UNIT, "h2d_bytes_per_step": world * (n * 6 * 8 + n * 4),
           "d2h_bytes_per_step": world * (n * 6 * 8 + n * 4 * 3),
           "note": "stb_track_host per rank: pinned AoS host x[n*6] and input flags in, coordinates and "
                   "Track()'s stable/lost_turn/lost_post out, one call per step (host wall clock)"}

    if rank == 0:
        kernel_ms = ms / a.steps
        flops_launch = info["flops_per_turn"] * 0.5 * (alive0 + alive1) * T
        achieved = flops_launch / (kernel_ms * 1e-3) / 1e12
        roof = {"bound": "fp64", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
                "frac": (achieved / fp64_peak) if fp64_peak else None,
                "peak_source": "measured FP64 FMA probe (stb_fp64_peak) on this GPU",
                "flops_per_particle_turn": info["flops_per_turn"],
                "work_note": "achieved counts the reference's operations (hoisted form); of them the kernel does "
                             "not re-execute the second of two identical drifts at Yoshida slice boundaries "
                             "(ops_reused_per_particle_turn), whose increments it adds again bit for bit",
                "ops_reused_per_particle_turn": reused_drift_ops(lat),
                "traffic": roofline_traffic(),
                "traffic_source": "dram__bytes_read.sum + dram__bytes_write.sum of one ncu capture of this kernel "
                                  "(profiles/track_kernel_rhic_like.md), scaled to this launch's particle-turns; "
                                  "not measured in this run"}
        value_f = pt_f / (ms_f * 1e-3)
        ach_f = value_f / world * info["flops_per_turn"] / 1e12
        fast = {"value": value_f, "unit": UNIT, "ms_per_step": ms_f / a.steps, "achieved_tflops": ach_f,
                "frac": (ach_f / fp64_peak) if fp64_peak else None, "kernel_variant": fast_info["variant_name"],
                "note": "same workload and steps with the FMA-contracted kernel (contraction policy fast); "
                        "its results differ from the reference's in the last bits"}
        line_out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
                    "warmup": a.warmup, "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak",
                    "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                    "config": {"workload": WORKLOAD, "particles_per_gpu": n, "turns_per_step": T,
                               "elements": info["elements"], "l2": "256 MiB flush between timed steps",
                               "parallelism": f"particle shards x{world}, no exchange",
                               "kernel_variant": info["variant_name"], "kernel_variant_index": info["variant"],
                               "autotune_ms_1turn": {k: round(v, 3) for k, v in tune["ms"].items()}},
                    "roofline": roof, "fast_contraction": fast, "cpu_baseline": cpu, "e2e": e2e,
                    "gpu_launches": a.steps,
                    "clocks": clk.summary(), "alive": [alive0, alive1]}
        print(json.dumps(line_out), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
