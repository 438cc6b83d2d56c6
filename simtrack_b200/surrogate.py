"""Surrogate-pruned dynamic-aperture scan.

The plain scan tracks every initial condition of every seed for the full turn
count.  Here the batched scan first tracks all of them for `nrec` turns while
recording x, px, y, py turn by turn; the early-turn features (stb_tbt_features:
initial amplitudes, momentum offset, angle, the FineTuneFinder tunes of two
`window`-turn windows and their drift, the action spread and the largest
amplitude reached) feed the MLP classifier (stb_mlp_*: bf16 tcgen05 GEMMs with
FP32 accumulation, trained by its own AdamW step), which predicts survival to
the full turn count.  Particles classified with confidence >= `confidence`
are retired from the scan, except a random audit fraction; every uncertain
particle and the audit sample are tracked to the full turn count by the plain
FP64 kernel.  The DA of a ray then comes from the tracked loss turns where
available and from the prediction for retired particles.

No reference counterpart: the reference tracks every particle to the end
(Track_DA, simtrack.cpp:21389-21441).
"""
from __future__ import annotations

import json
import math
import time
from dataclasses import asdict, dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from . import lattices
from .api import MLP, NUM_FEATURES, RETIRED, Scan, Table, fine_tune, tbt_features
from .da import da_from_lost
from .optics import one_turn_jacobian, twiss_from_matrix


@dataclass
class SurrogateConfig:
    nturn: int = 100000          # full turn count (the label: survival to it)
    nrec: int = 1024             # turns tracked by everyone, recorded for the features
    window: int = 512            # tune windows [0, window) and [nrec - window, nrec)
    tune_lower: float = 0.2      # FineTuneFinder search window (fractional tunes)
    tune_upper: float = 0.45
    confidence: float = 0.99
    audit: float = 0.02
    turns_per_block: int = 256
    hidden: int = 256
    batch: int = 4096
    epochs: int = 150
    lr: float = 2e-3
    weight_decay: float = 1e-2
    seed: int = 0
    # "ray": retire by the structure of the DA ray (see ray_policy);
    # "confidence": retire every particle classified with `confidence`
    policy: str = "ray"
    band_lo: int = 2             # amplitude steps tracked below the predicted first loss of a ray
    band_hi: int = 2             # ... and above it
    retune: bool = True          # re-choose the scan's launch variant for the survivors of retirement


@dataclass
class EarlyPhase:
    scan: Scan
    alive: np.ndarray            # [n] bool: alive after nrec turns
    features: np.ndarray         # [n_alive, 12] float32 (rows of the alive particles, x0 order)
    lost_turn: np.ndarray        # [n] loss turns after nrec turns (-1 alive)
    seconds: dict = field(default_factory=dict)


def ring_setup(seeds: Sequence[int], namp=64, amax=12.0, nang=11, deltas=(-1e-3, -5e-4, 0.0, 5e-4, 1e-3),
               device: int = 0):
    lats = [lattices.rhic_like_ring(seed=s) for s in seeds]
    tables = [Table(lattices.build_line(lat), device) for lat in lats]
    grids = [lattices.da_grid(lat, namp, amax, nang, deltas) for lat in lats]
    return lats, tables, grids


def optics_at_start(lat: lattices.Lattice, table: Table) -> tuple:
    """(beta_x, alpha_x, beta_y, alpha_y, emit_x, emit_y): periodic Twiss from
    the GPU one-turn Jacobian, geometric emittances from the normalised one."""
    tw = twiss_from_matrix(one_turn_jacobian(table))
    beta = math.sqrt(1.0 - 1.0 / lat.gamma ** 2)
    emit = lat.meta.get("emit_norm", 2.5e-6) / (beta * lat.gamma)
    return (tw.beta_x, tw.alpha_x, tw.beta_y, tw.alpha_y, emit, emit)


def early_phase(tables, grids, radius: float, twiss6, cfg: SurrogateConfig, device: int = 0) -> EarlyPhase:
    """Tracks every particle nrec turns with the turn-by-turn record on, then
    computes the features of the survivors on the GPU."""
    import torch
    dev = torch.device("cuda", device)
    t0 = time.perf_counter()
    sc = Scan(tables, grids, aperture_radius=radius, device=device)
    sc.autotune(nturn=16)
    n = sc.n
    tbt = torch.empty((cfg.nrec, 4, n), dtype=torch.float64, device=dev)
    sc.set_tbt(tbt, cfg.nrec)
    sc.run(cfg.nrec, cfg.turns_per_block)
    sc.set_tbt(None, 0)
    lt, _, _ = sc.results()
    alive = lt < 0
    t1 = time.perf_counter()
    idx = torch.from_numpy(np.nonzero(alive)[0]).to(dev)
    na = int(idx.numel())
    sub = tbt.index_select(2, idx).contiguous()  # [nrec, 4, n_alive]
    del tbt
    tunes = torch.empty((4, na), dtype=torch.float64, device=dev)
    w, plane = cfg.window, 4 * na
    starts = (0, cfg.nrec - w)
    for k, (t_start, row) in enumerate([(starts[0], 0), (starts[0], 2), (starts[1], 0), (starts[1], 2)]):
        fine_tune(sub, w, na, plane, cfg.tune_lower, cfg.tune_upper, tunes[k], offset=t_start * plane + row * na,
                  device=device)
    x0 = torch.tensor(np.concatenate(grids, axis=0)[alive].T.copy(), dtype=torch.float64, device=dev)
    feats = torch.empty((na, NUM_FEATURES), dtype=torch.float32, device=dev)
    tbt_features(sub, x0, tunes, twiss6, feats, device=device)
    torch.cuda.synchronize(dev)
    t2 = time.perf_counter()
    return EarlyPhase(sc, alive, feats.cpu().numpy(), lt, {"track_nrec": t1 - t0, "features": t2 - t1})


class Standardizer:
    def __init__(self, feats: np.ndarray):
        self.mean = feats.mean(axis=0)
        self.std = feats.std(axis=0) + 1e-6

    def __call__(self, f: np.ndarray) -> np.ndarray:
        return ((f - self.mean) / self.std).astype(np.float32)


def train(feats: np.ndarray, labels: np.ndarray, cfg: SurrogateConfig, device: int = 0):
    """Trains the classifier (label 1: survives the full turn count) with
    class-balanced weights; returns (mlp, standardizer, loss history)."""
    import torch
    dev = torch.device("cuda", device)
    std = Standardizer(feats)
    X = torch.tensor(std(feats), device=dev)
    Y = torch.tensor(labels.astype(np.int32), device=dev)
    n1 = max(1, int(labels.sum()))
    n0 = max(1, len(labels) - n1)
    wv = np.where(labels == 1, 0.5 * len(labels) / n1, 0.5 * len(labels) / n0).astype(np.float32)
    W = torch.tensor(wv, device=dev)
    mlp = MLP(NUM_FEATURES, cfg.hidden, 2, max_batch=cfg.batch, seed=cfg.seed, device=device)
    rng = np.random.default_rng(cfg.seed)
    n = len(labels)
    bs = min(cfg.batch, (n // 16) * 16)  # the GEMMs take batches in multiples of 16
    if bs < 16:
        raise ValueError("too few training samples")
    steps_per_epoch = n // bs
    total = cfg.epochs * steps_per_epoch
    hist = []
    step = 0
    for ep in range(cfg.epochs):
        perm = torch.from_numpy(rng.permutation(n)).to(dev)
        for b in range(steps_per_epoch):
            lr = cfg.lr * 0.5 * (1.0 + math.cos(math.pi * step / total))  # cosine decay
            mlp.set_adamw(lr=lr, weight_decay=cfg.weight_decay)
            sel = perm[b * bs:(b + 1) * bs]
            loss = mlp.train_step(X.index_select(0, sel).contiguous(), Y.index_select(0, sel).contiguous(),
                                  W.index_select(0, sel).contiguous())
            step += 1
        hist.append(loss)
    return mlp, std, hist


def predict(mlp: MLP, std: Standardizer, feats: np.ndarray, device: int = 0) -> np.ndarray:
    """P(survive) per row."""
    import torch
    dev = torch.device("cuda", device)
    n = len(feats)
    npad = max(16, -(-n // 16) * 16)  # rows padded to a multiple of 16
    X = torch.zeros((npad, feats.shape[1]), dtype=torch.float32, device=dev)
    if n:
        X[:n] = torch.tensor(std(feats), device=dev)
    out = torch.empty((npad, 2), dtype=torch.float32, device=dev)
    for b in range(0, npad, mlp.max_batch):
        e = min(npad, b + mlp.max_batch)
        mlp.forward(X[b:e], out[b:e])
    return out[:n, 1].cpu().numpy()


def ray_policy(lost_early: np.ndarray, p: np.ndarray, namp: int, confidence: float, band_lo: int,
               band_hi: int):
    """Which particles to stop tracking, using the structure of a DA ray.

    Particles come in rays of `namp` amplitudes (smallest first) and the DA
    of a ray is set by its first lost particle.  With kL the first amplitude
    lost during the early turns and kP = min(kL, first amplitude the
    classifier calls lost):
      * particles above kL are retired: a known loss sits below them, so they
        cannot move the DA (exact);
      * particles in [kP - band_lo, kP + band_hi] stay tracked;
      * elsewhere below kL, particles with P(survive) >= confidence are retired
        as stable; the rest stay tracked.  Particles the classifier calls lost
        are never retired on its word alone: a wrong "lost" would lower the DA.

    lost_early, p: [n] arrays in grid order (p = nan where lost early).
    Returns (retire[n], retire_as_stable[n])."""
    L = np.asarray(lost_early, dtype=bool).reshape(-1, namp)
    P = np.nan_to_num(np.asarray(p, dtype=np.float64).reshape(-1, namp), nan=0.0)
    idx = np.arange(namp)[None, :]
    kL = np.where(L.any(axis=1), L.argmax(axis=1), namp)[:, None]
    pred_lost = ~L & (P < 0.5)
    kp = np.where(pred_lost.any(axis=1), pred_lost.argmax(axis=1), namp)[:, None]
    kP = np.minimum(kL, kp)
    alive = ~L
    above_known = idx > kL
    band = (idx >= kP - band_lo) & (idx <= kP + band_hi)
    stable = alive & ~above_known & ~band & (P >= confidence)
    retire = (alive & above_known) | stable
    return retire.ravel(), stable.ravel()


@dataclass
class PrunedResult:
    lost_turn: np.ndarray        # [n] tracked loss turn, RETIRED for retired particles
    predicted_survive: np.ndarray  # [n] final survival used for the DA (tracked or predicted)
    retired: np.ndarray          # [n] bool
    audited: np.ndarray          # [n] bool (confident but tracked anyway)
    p_survive: np.ndarray        # [n] classifier output (nan where not evaluated)
    seconds: dict
    particle_turns: float
    lost_early: np.ndarray       # [n] lost during the first nrec turns


def pruned_scan(tables, grids, radius, twiss6, mlp: MLP, std: Standardizer, cfg: SurrogateConfig, namp: int,
                device: int = 0, rng_seed: int = 1) -> PrunedResult:
    t0 = time.perf_counter()
    ep = early_phase(tables, grids, radius, twiss6, cfg, device)
    t1 = time.perf_counter()
    n = ep.scan.n
    p = np.full(n, np.nan)
    p[ep.alive] = predict(mlp, std, ep.features, device)
    if cfg.policy == "ray":
        cand, cand_stable = ray_policy(~ep.alive, p, namp, cfg.confidence, cfg.band_lo, cfg.band_hi)
    else:
        cand = np.zeros(n, dtype=bool)
        cand[ep.alive] = (p[ep.alive] >= cfg.confidence) | (p[ep.alive] <= 1.0 - cfg.confidence)
        cand_stable = cand & (np.nan_to_num(p) >= 0.5)
    rng = np.random.default_rng(rng_seed)
    audit = cand & (rng.random(n) < cfg.audit)
    retire = cand & ~audit
    ep.scan.retire(retire)
    t2 = time.perf_counter()
    # One turn block compacts the retired particles away; the launch variant
    # is then chosen again for the few survivors, whose tracking is bound by
    # the latency of one particle-turn rather than by throughput.
    rest = cfg.nturn - cfg.nrec
    first = min(cfg.turns_per_block, rest)
    ep.scan.run(first, cfg.turns_per_block)
    if cfg.retune and rest > first:
        ep.scan.autotune(nturn=16)
    ep.scan.run(rest - first, cfg.turns_per_block)
    lt, _, _ = ep.scan.results()
    t3 = time.perf_counter()
    survive = np.where(retire, cand_stable, (lt < 0) | (lt >= cfg.nturn))
    # particle-turns actually tracked
    tracked_to = np.where(lt == RETIRED, cfg.nrec, np.where(lt < 0, cfg.nturn, lt + 1))
    secs = dict(ep.seconds)
    secs.update({"early_total": t1 - t0, "classify_retire": t2 - t1, "track_rest": t3 - t2, "total": t3 - t0})
    return PrunedResult(lt, survive, retire, audit, p, secs, float(tracked_to.sum()), ~ep.alive)


def da_of(survive: np.ndarray, nseed: int, nd: int, nang: int, namp: int, amax: float) -> np.ndarray:
    lost = np.where(survive, -1, 0).reshape(nseed, nd, nang, namp)
    return da_from_lost(lost, np.linspace(0.0, amax, namp), 1)


def plain_scan(tables, grids, radius, cfg: SurrogateConfig, device: int = 0):
    """Every particle to its loss or the full turn count, one persistent scan;
    the launch variant (and work-item packing) tuned on the first turns, as the
    pruned scan tunes its own phases."""
    t0 = time.perf_counter()
    sc = Scan(tables, grids, aperture_radius=radius, device=device)
    sc.autotune(nturn=16)
    sc.run(cfg.nturn, cfg.turns_per_block)
    lt, _, _ = sc.results()
    wall = time.perf_counter() - t0
    tracked_to = np.where(lt < 0, cfg.nturn, lt + 1)
    return lt, wall, float(tracked_to.sum())


def compare(res: PrunedResult, lt_plain: np.ndarray, wall_plain: float, pt_plain: float, nseed: int, nd: int,
            nang: int, namp: int, amax: float, cfg: SurrogateConfig) -> dict:
    """DA per ray and cost of a pruned scan against the plain scan of the same seeds."""
    surv_plain = (lt_plain < 0) | (lt_plain >= cfg.nturn)
    da_plain = da_of(surv_plain, nseed, nd, nang, namp, amax)
    da_sur = da_of(res.predicted_survive, nseed, nd, nang, namp, amax)
    err = np.abs(da_sur - da_plain)
    retired, aud = res.retired, res.audited
    wrong = retired & (res.predicted_survive != surv_plain)
    p_aud = res.p_survive[aud]
    audit_acc = float(((np.nan_to_num(p_aud) >= 0.5) == surv_plain[aud]).mean()) if aud.any() else float("nan")
    return {
        "plain": {"wall_s": wall_plain, "particle_turns": pt_plain},
        "pruned": {"wall_s": res.seconds["total"], "seconds": res.seconds, "particle_turns": res.particle_turns,
                   "retired": int(retired.sum()), "audited": int(aud.sum()),
                   "tracked_to_end": int((~retired & ~res.lost_early).sum()),
                   "alive_at_nrec": int((~res.lost_early).sum()),
                   "retired_with_other_outcome": int(wrong.sum()), "audit_accuracy": audit_acc},
        "speedup_wall": wall_plain / res.seconds["total"],
        "speedup_particle_turns": pt_plain / res.particle_turns,
        "da_plain_mean_sigma": float(da_plain.mean()),
        "da_error_sigma": {"max": float(err.max()), "mean": float(err.mean()),
                           "per_angle_max": err.max(axis=(0, 1)).tolist(),
                           "rays_differing": int((err > 1e-12).sum()), "rays": int(err.size)},
        "da_step_sigma": amax / (namp - 1),
    }


def experiment(train_seeds: Sequence[int], test_seeds: Sequence[int], namp=64, amax=12.0, nang=11,
               deltas=(-1e-3, -5e-4, 0.0, 5e-4, 1e-3), cfg: Optional[SurrogateConfig] = None, device: int = 0,
               log=print, artifacts: Optional[str] = None) -> dict:
    """Trains on train_seeds (labels from their full-length plain tracking),
    then runs the plain and the surrogate-pruned scan on test_seeds and
    compares DA per ray and wall time.  With `artifacts`, the trained
    network, the feature scaling, the plain scan's loss turns and the
    classifier's outputs on the test seeds are saved there (npz) for
    pruned_from_artifacts."""
    cfg = cfg or SurrogateConfig()
    nd = len(deltas)
    # --- training data: early phase + continuation to the full turn count
    lats, tables, grids = ring_setup(train_seeds, namp, amax, nang, deltas, device)
    radius = lats[0].aperture_radius
    twiss6 = optics_at_start(lats[0], tables[0])
    log(f"optics at start: {twiss6}")
    t0 = time.perf_counter()
    ep = early_phase(tables, grids, radius, twiss6, cfg, device)
    ep.scan.run(cfg.nturn - cfg.nrec, cfg.turns_per_block)
    lt_train, _, _ = ep.scan.results()
    t_label = time.perf_counter() - t0
    y = ((lt_train < 0) | (lt_train >= cfg.nturn))[ep.alive].astype(np.int32)
    log(f"training data: {int(ep.alive.sum())} survivors of {len(lt_train)} after {cfg.nrec} turns, "
        f"{int(y.sum())} survive {cfg.nturn}; labelling took {t_label:.1f} s")
    t0 = time.perf_counter()
    mlp, std, hist = train(ep.features, y, cfg, device)
    t_train = time.perf_counter() - t0
    p_tr = predict(mlp, std, ep.features, device)
    acc_tr = float(((p_tr >= 0.5) == (y == 1)).mean())
    log(f"trained in {t_train:.1f} s, final loss {hist[-1]:.4f}, train accuracy {acc_tr:.4f}")
    del ep, tables
    # --- held-out seeds: plain scan, then the pruned scan
    lats, tables, grids = ring_setup(test_seeds, namp, amax, nang, deltas, device)
    lt_plain, wall_plain, pt_plain = plain_scan(tables, grids, radius, cfg, device)
    log(f"plain scan: {wall_plain:.1f} s")
    res = pruned_scan(tables, grids, radius, twiss6, mlp, std, cfg, namp, device)
    log(f"pruned scan: {res.seconds['total']:.1f} s {res.seconds}")
    out = {"train_seeds": list(train_seeds), "test_seeds": list(test_seeds),
           "grid": {"namp": namp, "amax_sigma": amax, "nang": nang, "deltas": list(deltas)},
           "config": asdict(cfg), "optics_at_start": twiss6,
           "train": {"samples": int(len(y)), "survive_fraction": float(y.mean()), "seconds": t_train,
                     "label_seconds": t_label, "accuracy": acc_tr, "loss_last": hist[-1]}}
    out.update(compare(res, lt_plain, wall_plain, pt_plain, len(test_seeds), nd, nang, namp, amax, cfg))
    if artifacts:
        np.savez_compressed(artifacts, params=mlp.get_params(), std_mean=std.mean, std_std=std.std,
                            lt_plain=lt_plain, wall_plain=wall_plain, pt_plain=pt_plain, p=res.p_survive,
                            lost_early=res.lost_early, twiss6=np.array(twiss6),
                            test_seeds=np.array(test_seeds), namp=namp, nang=nang, amax=amax,
                            deltas=np.array(deltas), hidden=cfg.hidden, nturn=cfg.nturn, nrec=cfg.nrec)
    return out


def pruned_from_artifacts(path: str, cfg: Optional[SurrogateConfig] = None, device: int = 0, log=print) -> dict:
    """Re-runs only the pruned scan of the test seeds with a network and plain
    scan saved by experiment(artifacts=...), e.g. to try another policy."""
    a = np.load(path)
    cfg = cfg or SurrogateConfig()
    cfg.nturn, cfg.nrec, cfg.hidden = int(a["nturn"]), int(a["nrec"]), int(a["hidden"])
    namp, nang, amax = int(a["namp"]), int(a["nang"]), float(a["amax"])
    deltas = tuple(float(d) for d in a["deltas"])
    seeds = [int(s) for s in a["test_seeds"]]
    mlp = MLP(NUM_FEATURES, cfg.hidden, 2, max_batch=cfg.batch, seed=cfg.seed, device=device)
    mlp.set_params(a["params"])
    std = Standardizer.__new__(Standardizer)
    std.mean, std.std = a["std_mean"], a["std_std"]
    lats, tables, grids = ring_setup(seeds, namp, amax, nang, deltas, device)
    res = pruned_scan(tables, grids, lats[0].aperture_radius, tuple(a["twiss6"]), mlp, std, cfg, namp, device)
    log(f"pruned scan: {res.seconds['total']:.1f} s {res.seconds}")
    out = {"test_seeds": seeds, "config": asdict(cfg), "plain_from": path}
    out.update(compare(res, a["lt_plain"], float(a["wall_plain"]), float(a["pt_plain"]), len(seeds), len(deltas),
                       nang, namp, amax, cfg))
    return out


def evaluate_saved(path: str, seeds: Sequence[int], cfg: Optional[SurrogateConfig] = None, device: int = 0,
                   log=print, plain: bool = True) -> dict:
    """Plain and pruned scans of `seeds` (e.g. seeds neither trained nor used
    to choose the retirement policy) with the network saved by
    experiment(artifacts=...).  With plain=False only the pruned scan runs
    (its wall time and tracking work, e.g. for a seed count whose plain scan
    is measured elsewhere)."""
    a = np.load(path)
    cfg = cfg or SurrogateConfig()
    cfg.nturn, cfg.nrec, cfg.hidden = int(a["nturn"]), int(a["nrec"]), int(a["hidden"])
    namp, nang, amax = int(a["namp"]), int(a["nang"]), float(a["amax"])
    deltas = tuple(float(d) for d in a["deltas"])
    mlp = MLP(NUM_FEATURES, cfg.hidden, 2, max_batch=cfg.batch, seed=cfg.seed, device=device)
    mlp.set_params(a["params"])
    std = Standardizer.__new__(Standardizer)
    std.mean, std.std = a["std_mean"], a["std_std"]
    lats, tables, grids = ring_setup(seeds, namp, amax, nang, deltas, device)
    radius = lats[0].aperture_radius
    out = {"eval_seeds": list(seeds), "config": asdict(cfg), "model_from": path,
           "grid": {"namp": namp, "amax_sigma": amax, "nang": nang, "deltas": list(deltas)}}
    if not plain:
        res = pruned_scan(tables, grids, radius, tuple(a["twiss6"]), mlp, std, cfg, namp, device)
        log(f"pruned scan: {res.seconds['total']:.1f} s {res.seconds}")
        out["pruned"] = {"wall_s": res.seconds["total"], "seconds": res.seconds,
                         "particle_turns": res.particle_turns, "retired": int(res.retired.sum()),
                         "audited": int(res.audited.sum()),
                         "tracked_to_end": int((~res.retired & ~res.lost_early).sum())}
        return out
    lt_plain, wall_plain, pt_plain = plain_scan(tables, grids, radius, cfg, device)
    log(f"plain scan: {wall_plain:.1f} s")
    res = pruned_scan(tables, grids, radius, tuple(a["twiss6"]), mlp, std, cfg, namp, device)
    log(f"pruned scan: {res.seconds['total']:.1f} s {res.seconds}")
    out.update(compare(res, lt_plain, wall_plain, pt_plain, len(seeds), len(deltas), nang, namp, amax, cfg))
    return out


def replay_policies(path: str, confidences=(0.99, 0.999), bands=((0, 0), (2, 2), (3, 3), (4, 4)), audit=0.02,
                    seed: int = 1) -> list:
    """Offline replay of the retirement policy on a saved experiment (no GPU):
    for each confidence and band, the particles that would stay tracked to
    the end and the rays whose DA would differ from the plain scan's."""
    a = np.load(path)
    namp, nang, amax = int(a["namp"]), int(a["nang"]), float(a["amax"])
    nd, nseed, nturn = len(a["deltas"]), len(a["test_seeds"]), int(a["nturn"])
    truth = (a["lt_plain"] < 0) | (a["lt_plain"] >= nturn)
    lost_early, p = a["lost_early"], a["p"]
    da_true = da_of(truth, nseed, nd, nang, namp, amax)
    rows = []
    for c in confidences:
        for lo, hi in bands:
            retire, stable = ray_policy(lost_early, p, namp, c, lo, hi)
            aud = retire & (np.random.default_rng(seed).random(len(retire)) < audit)
            retire = retire & ~aud
            err = np.abs(da_of(np.where(retire, stable, truth), nseed, nd, nang, namp, amax) - da_true)
            rows.append({"confidence": c, "band": [lo, hi], "tracked_to_end": int((~lost_early & ~retire).sum()),
                         "rays_differing": int((err > 1e-12).sum()), "da_error_max_sigma": float(err.max())})
    return rows


def main(argv=None):
    import argparse
    ap = argparse.ArgumentParser(description="surrogate-pruned vs plain DA scan of the RHIC-like ring")
    ap.add_argument("--train-seeds", type=int, default=32)
    ap.add_argument("--test-seeds", type=int, default=32)
    ap.add_argument("--nturn", type=int, default=100000)
    ap.add_argument("--namp", type=int, default=64)
    ap.add_argument("--nang", type=int, default=11)
    ap.add_argument("--epochs", type=int, default=150)
    ap.add_argument("--policy", default="ray", choices=["ray", "confidence"])
    ap.add_argument("--band", type=int, nargs=2, default=[2, 2], metavar=("LO", "HI"))
    ap.add_argument("--confidence", type=float, default=0.99)
    ap.add_argument("--artifacts", default="", help="save (or, with --pruned-only, load) the trained network etc.")
    ap.add_argument("--pruned-only", action="store_true")
    ap.add_argument("--replay", action="store_true", help="offline policy replay on --artifacts (no GPU)")
    ap.add_argument("--eval-seeds", type=int, nargs=2, default=None, metavar=("FIRST", "COUNT"),
                    help="plain and pruned scans of new seeds with the network saved in --artifacts")
    ap.add_argument("--no-plain", action="store_true", help="with --eval-seeds: run the pruned scan only")
    ap.add_argument("--out", default="")
    a = ap.parse_args(argv)
    cfg = SurrogateConfig(nturn=a.nturn, epochs=a.epochs, policy=a.policy, band_lo=a.band[0], band_hi=a.band[1],
                          confidence=a.confidence)
    if a.replay:
        for r in replay_policies(a.artifacts):
            print(json.dumps(r))
        return
    if a.eval_seeds:
        res = evaluate_saved(a.artifacts, list(range(a.eval_seeds[0], a.eval_seeds[0] + a.eval_seeds[1])), cfg,
                             plain=not a.no_plain)
    elif a.pruned_only:
        res = pruned_from_artifacts(a.artifacts, cfg)
    else:
        train_seeds = list(range(1, a.train_seeds + 1))
        test_seeds = list(range(a.train_seeds + 1, a.train_seeds + a.test_seeds + 1))
        res = experiment(train_seeds, test_seeds, namp=a.namp, nang=a.nang, cfg=cfg,
                         artifacts=a.artifacts or None)
    js = json.dumps(res, indent=1)
    print(js)
    if a.out:
        with open(a.out, "w") as f:
            f.write(js)


if __name__ == "__main__":
    main()
