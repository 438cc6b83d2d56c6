"""FineTuneFinder (simtrack.cpp:2288, 2321): the C restatement against the
reference's own outputs (golden fixture and, when built, the live reference),
and the GPU tune finder and surrogate feature kernel against them."""
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden" / "fine_tune.npz"


def _golden():
    d = np.load(GOLDEN)
    return d["x"], d["px"], d["windows"], d["tunes"]


def test_port_matches_golden(port_oracle):
    xs, pxs, windows, tunes = _golden()
    for s, (x, px) in enumerate(zip(xs, pxs)):
        for w, (lo, hi, with_px) in enumerate(windows):
            got = port_oracle.fine_tune(x, px if with_px else None, lo, hi)
            assert got == tunes[s, w], (s, w, got, tunes[s, w])


def test_port_matches_live_reference(port_oracle, ref_oracle):
    rng = np.random.default_rng(3)
    for n in (64, 300, 1024):
        i = np.arange(n)
        q = rng.uniform(0.05, 0.45)
        x = np.cos(2 * np.pi * q * i + 0.3) + rng.normal(0, 1e-2, n)
        px = -np.sin(2 * np.pi * q * i + 0.3)
        for lo, hi in ((0.0, 0.5), (q - 0.02, q + 0.03)):
            assert port_oracle.fine_tune(x, None, lo, hi) == ref_oracle.fine_tune(x, None, lo, hi)
            assert port_oracle.fine_tune(x, px, lo, hi) == ref_oracle.fine_tune(x, px, lo, hi)


def test_pure_line_found():
    """A single line is found to well below the coarse step (the residual
    few 1e-6 is the leakage of the real signal's mirror line, no window)."""
    from oracle_bridge import PortOracle, port_available
    if not port_available():
        pytest.skip("port oracle not built")
    o = PortOracle()
    i = np.arange(512)
    for q in (0.2113, 0.31234567, 0.4401):
        assert abs(o.fine_tune(np.cos(2 * np.pi * q * i), None, 0.0, 0.5) - q) < 1e-5


@pytest.mark.gpu
def test_gpu_fine_tune_matches_reference_outputs(native_lib):
    import torch

    from simtrack_b200.api import fine_tune
    xs, pxs, windows, tunes = _golden()
    nsig, n = xs.shape
    # signals interleaved like a turn-by-turn record: sample i of signal j at i*stride + j
    stride = nsig + 5
    X = np.zeros((n, stride))
    P = np.zeros((n, stride))
    X[:, :nsig] = xs.T
    P[:, :nsig] = pxs.T
    Xd = torch.tensor(X, dtype=torch.float64, device="cuda:0")
    Pd = torch.tensor(P, dtype=torch.float64, device="cuda:0")
    out = torch.empty(nsig, dtype=torch.float64, device="cuda:0")
    for w, (lo, hi, with_px) in enumerate(windows):
        fine_tune(Xd, n, nsig, stride, lo, hi, out, px=Pd if with_px else None)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        # same search, same summation order; the device sin/cos may differ
        # from the host's in the last bit, which moves the flat-topped peak
        # by far less than 1e-9
        assert np.max(np.abs(got - tunes[:, w])) < 1e-9, (w, got - tunes[:, w])


@pytest.mark.gpu
def test_gpu_features_match_numpy(native_lib):
    import torch

    from simtrack_b200.api import tbt_features
    rng = np.random.default_rng(11)
    n, nturn = 700, 64
    tw = (12.3, -0.7, 20.1, 1.1, 2.5e-8, 2.6e-8)
    tbt = rng.normal(0, 1e-3, (nturn, 4, n))
    x0 = rng.normal(0, 1e-3, (6, n))
    tunes = rng.uniform(0.2, 0.4, (4, n))
    dev = "cuda:0"
    out = torch.empty((n, 12), dtype=torch.float32, device=dev)
    tbt_features(torch.tensor(tbt, device=dev), torch.tensor(x0, device=dev), torch.tensor(tunes, device=dev), tw,
                 out)
    got = out.cpu().numpy()
    bx, ax, by, ay, ex, ey = tw

    def action(x, p, b, a):
        pn = a * x + b * p
        return 0.5 * (x * x + pn * pn) / b

    jx0 = action(x0[0], x0[1], bx, ax)
    jy0 = action(x0[2], x0[3], by, ay)
    j = action(tbt[:, 0], tbt[:, 1], bx, ax) / ex + action(tbt[:, 2], tbt[:, 3], by, ay) / ey
    jmax, jmin = j.max(axis=0), j.min(axis=0)
    j0 = jx0 / ex + jy0 / ey
    ampx, ampy = np.sqrt(2 * jx0 / ex), np.sqrt(2 * jy0 / ey)
    exp = np.stack([ampx, ampy, x0[5] * 1e3, np.arctan2(ampy, ampx), tunes[0], tunes[1], tunes[2], tunes[3],
                    np.log10(np.abs(tunes[0] - tunes[2]) + 1e-10), np.log10(np.abs(tunes[1] - tunes[3]) + 1e-10),
                    np.log10((jmax - jmin) / (j0 + 0.5) + 1e-8), np.sqrt(2 * jmax)], axis=1).astype(np.float32)
    np.testing.assert_allclose(got, exp, rtol=2e-6, atol=1e-6)
