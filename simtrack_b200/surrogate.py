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


@dataclass
class PrunedResult:
    lost_turn: np.ndarray        # [n] tracked loss turn, RETIRED for retired particles
    predicted_survive: np.ndarray  # [n] final survival used for the DA (tracked or predicted)
    retired: np.ndarray          # [n] bool
    audited: np.ndarray          # [n] bool (confident but tracked anyway)
    p_survive: np.ndarray        # [n] classifier output (nan where not evaluated)
    seconds: dict
    particle_turns: float


def pruned_scan(tables, grids, radius, twiss6, mlp: MLP, std: Standardizer, cfg: SurrogateConfig,
                device: int = 0, rng_seed: int = 1) -> PrunedResult:
    t0 = time.perf_counter()
    ep = early_phase(tables, grids, radius, twiss6, cfg, device)
    t1 = time.perf_counter()
    n = ep.scan.n
    p = np.full(n, np.nan)
    p[ep.alive] = predict(mlp, std, ep.features, device)
    conf = np.zeros(n, dtype=bool)
    conf[ep.alive] = (p[ep.alive] >= cfg.confidence) | (p[ep.alive] <= 1.0 - cfg.confidence)
    rng = np.random.default_rng(rng_seed)
    audit = conf & (rng.random(n) < cfg.audit)
    retire = conf & ~audit
    ep.scan.retire(retire)
    t2 = time.perf_counter()
    ep.scan.run(cfg.nturn - cfg.nrec, cfg.turns_per_block)
    lt, _, _ = ep.scan.results()
    t3 = time.perf_counter()
    survive = np.where(retire, p >= 0.5, (lt < 0) | (lt >= cfg.nturn))
    # particle-turns actually tracked
    tracked_to = np.where(lt == RETIRED, cfg.nrec, np.where(lt < 0, cfg.nturn, lt + 1))
    secs = dict(ep.seconds)
    secs.update({"early_total": t1 - t0, "classify_retire": t2 - t1, "track_rest": t3 - t2, "total": t3 - t0})
    return PrunedResult(lt, survive, retire, audit, p, secs, float(tracked_to.sum()))


def da_of(survive: np.ndarray, nseed: int, nd: int, nang: int, namp: int, amax: float) -> np.ndarray:
    lost = np.where(survive, -1, 0).reshape(nseed, nd, nang, namp)
    return da_from_lost(lost, np.linspace(0.0, amax, namp), 1)


def plain_scan(tables, grids, radius, cfg: SurrogateConfig, device: int = 0):
    t0 = time.perf_counter()
    sc = Scan(tables, grids, aperture_radius=radius, device=device)
    sc.run(cfg.nturn, cfg.turns_per_block)
    lt, _, _ = sc.results()
    wall = time.perf_counter() - t0
    tracked_to = np.where(lt < 0, cfg.nturn, lt + 1)
    return lt, wall, float(tracked_to.sum())


def experiment(train_seeds: Sequence[int], test_seeds: Sequence[int], namp=64, amax=12.0, nang=11,
               deltas=(-1e-3, -5e-4, 0.0, 5e-4, 1e-3), cfg: Optional[SurrogateConfig] = None, device: int = 0,
               log=print) -> dict:
    """Trains on train_seeds (labels from their full-length plain tracking),
    then runs the plain and the surrogate-pruned scan on test_seeds and
    compares DA per angle and wall time."""
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
    res = pruned_scan(tables, grids, radius, twiss6, mlp, std, cfg, device)
    log(f"pruned scan: {res.seconds['total']:.1f} s {res.seconds}")
    nseed = len(test_seeds)
    surv_plain = (lt_plain < 0) | (lt_plain >= cfg.nturn)
    da_plain = da_of(surv_plain, nseed, nd, nang, namp, amax)
    da_sur = da_of(res.predicted_survive, nseed, nd, nang, namp, amax)
    err = np.abs(da_sur - da_plain)
    retired = res.retired
    wrong = retired & (res.predicted_survive != surv_plain)
    aud = res.audited
    p_aud = res.p_survive[aud]
    audit_acc = float(((p_aud >= 0.5) == surv_plain[aud]).mean()) if aud.any() else float("nan")
    out = {
        "train_seeds": list(train_seeds), "test_seeds": list(test_seeds),
        "grid": {"namp": namp, "amax_sigma": amax, "nang": nang, "deltas": list(deltas)},
        "config": asdict(cfg),
        "optics_at_start": twiss6,
        "train": {"samples": int(len(y)), "survive_fraction": float(y.mean()), "seconds": t_train,
                  "label_seconds": t_label, "accuracy": acc_tr, "loss_last": hist[-1]},
        "plain": {"wall_s": wall_plain, "particle_turns": pt_plain},
        "pruned": {"wall_s": res.seconds["total"], "seconds": res.seconds, "particle_turns": res.particle_turns,
                   "retired": int(retired.sum()), "audited": int(aud.sum()),
                   "alive_at_nrec": int(np.isfinite(res.p_survive).sum()),
                   "retired_misclassified": int(wrong.sum()), "audit_accuracy": audit_acc},
        "speedup_wall": wall_plain / res.seconds["total"],
        "speedup_particle_turns": pt_plain / res.particle_turns,
        "da_plain_mean_sigma": float(da_plain.mean()),
        "da_error_sigma": {"max": float(err.max()), "mean": float(err.mean()),
                           "per_angle_max": err.max(axis=(0, 1)).tolist(),
                           "rays_differing": int((err > 1e-12).sum()), "rays": int(err.size)},
        "da_step_sigma": amax / (namp - 1),
    }
    return out


def main(argv=None):
    import argparse
    ap = argparse.ArgumentParser(description="surrogate-pruned vs plain DA scan of the RHIC-like ring")
    ap.add_argument("--train-seeds", type=int, default=32)
    ap.add_argument("--test-seeds", type=int, default=32)
    ap.add_argument("--nturn", type=int, default=100000)
    ap.add_argument("--namp", type=int, default=64)
    ap.add_argument("--nang", type=int, default=11)
    ap.add_argument("--epochs", type=int, default=150)
    ap.add_argument("--out", default="")
    a = ap.parse_args(argv)
    cfg = SurrogateConfig(nturn=a.nturn, epochs=a.epochs)
    train_seeds = list(range(1, a.train_seeds + 1))
    test_seeds = list(range(a.train_seeds + 1, a.train_seeds + a.test_seeds + 1))
    res = experiment(train_seeds, test_seeds, namp=a.namp, nang=a.nang, cfg=cfg)
    js = json.dumps(res, indent=1)
    print(js)
    if a.out:
        with open(a.out, "w") as f:
            f.write(js)


if __name__ == "__main__":
    main()
