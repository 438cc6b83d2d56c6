"""tcgen05 BF16 surrogate kernels (needs a B200).

* The GEMM kernel against a plain PyTorch FP32 reference of the same product
  (bf16 inputs, FP32 accumulation): relative tolerance 2e-5 of the row scale.
* Forward probabilities, loss and every parameter gradient of the full
  network against the NumPy oracle (oracle/mlp_oracle.py), which rounds to
  bf16 at the same points: tolerances 2e-3 relative (bf16 re-rounding of
  values that differ in their last FP32 bits can flip one bf16 ulp).
* A few hundred AdamW steps separate a two-class toy problem.
"""
import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def bf16_tensor(a):
    return torch.tensor(np.asarray(a, dtype=np.float32), device="cuda").to(torch.bfloat16).contiguous()


@pytest.mark.parametrize("M,N,K", [(256, 256, 256), (300, 16, 272), (128, 256, 4096), (2, 256, 64), (4096, 256, 16)])
def test_tcgen05_gemm_matches_torch_fp32(native_lib, M, N, K):
    rng = np.random.default_rng(M + N + K)
    A = bf16_tensor(rng.standard_normal((M, K)))
    B = bf16_tensor(rng.standard_normal((N, K)))
    C = torch.zeros((M, N), dtype=torch.float32, device="cuda")
    rc = native_lib.stb_mlp_gemm_test(A.data_ptr(), K, B.data_ptr(), K, M, N, K, C.data_ptr(), N, 0)
    assert rc == 0, native_lib.stb_last_error()
    ref = A.float() @ B.float().T
    scale = ref.abs().amax(dim=1, keepdim=True) + 1e-6
    err = ((C - ref).abs() / scale).max().item()
    assert err < 2e-5, err


def test_gradients_match_numpy_oracle(native_lib):
    import mlp_oracle
    from simtrack_b200.api import MLP
    nin, H, nout, B = 12, 256, 2, 512
    rng = np.random.default_rng(5)
    params = mlp_oracle.init_params(nin, H, nout, seed=3)
    x = rng.standard_normal((B, nin)).astype(np.float32)
    y = (x[:, 0] + 0.5 * x[:, 3] - x[:, 7] > 0).astype(np.int32)
    w = rng.uniform(0.5, 1.5, B).astype(np.float32)
    m = MLP(nin, H, nout, max_batch=B)
    m.set_params(params)
    xt, yt, wt = (torch.tensor(v, device="cuda") for v in (x, y, w))
    loss = m.gradients(xt, yt, wt)
    g = m.get_params(1)
    ref_loss, ref_p, ref_g = mlp_oracle.forward_backward(params, x, y, w, nin, H, nout)
    assert abs(loss - ref_loss) <= 1e-4 * max(1.0, abs(ref_loss))
    probs = torch.empty((B, nout), device="cuda")
    m.forward(xt, probs)
    assert np.max(np.abs(probs.cpu().numpy() - ref_p)) < 2e-3
    off = 0
    for o, i in [(H, nin), (H, H), (H, H), (nout, H)]:
        for n in (o * i, o):
            a, r = g[off:off + n], ref_g[off:off + n]
            scale = np.abs(r).max() + 1e-12
            assert np.max(np.abs(a - r)) / scale < 2e-3, (off, n)
            off += n


def test_training_separates_toy_problem(native_lib):
    from simtrack_b200.api import MLP
    rng = np.random.default_rng(9)
    n, nin = 8192, 12
    x = rng.standard_normal((n, nin)).astype(np.float32)
    y = ((x[:, 0] ** 2 + x[:, 1] ** 2) < 1.2).astype(np.int32)
    m = MLP(nin, 256, 2, max_batch=1024, seed=1)
    m.set_adamw(lr=2e-3)
    xt, yt = torch.tensor(x, device="cuda"), torch.tensor(y, device="cuda")
    losses = []
    for step in range(300):
        i = (step * 1024) % n
        losses.append(m.train_step(xt[i:i + 1024], yt[i:i + 1024]))
    probs = torch.empty((1024, 2), device="cuda")
    m.forward(xt[:1024], probs)
    acc = ((probs[:, 1] > 0.5).int().cpu().numpy() == y[:1024]).mean()
    assert losses[-1] < 0.5 * losses[0]
    assert acc > 0.95, acc
