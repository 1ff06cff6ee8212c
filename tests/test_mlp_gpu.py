"""GPU: the tcgen05 BF16 training and inference kernels of the learned
closure against the CPU restatement (oracle/mlp.py).

Gradient bar: relative L2 <= 1e-2 per parameter block against the oracle's
BF16 form (same rounding points, FP64 accumulation), <= 5e-2 against the
exact FP64 gradient.  Inference: relative L2 <= 1e-2 against the BF16 form.
"""
import numpy as np
import pytest

from oracle import mlp as ref

pytestmark = pytest.mark.gpu

BLOCKS = {"W1": (ref.OW1, ref.OW2), "W2": (ref.OW2, ref.OW3), "W3": (ref.OW3, ref.OW4), "W4": (ref.OW4, ref.OB1),
          "b1": (ref.OB1, ref.OB2), "b2": (ref.OB2, ref.OB3), "b3": (ref.OB3, ref.OB4), "b4": (ref.OB4, ref.NPAR)}


def _net(params):
    import torch  # noqa: F401  (CUDA context)
    from erf_b200.closure import MLP
    m = MLP()
    m.set_params(params)
    m.set_normalization(np.zeros(13), np.ones(13), np.zeros(9), np.ones(9))
    return m


def _params(seed):
    p = ref.init_params(seed)
    rng = np.random.default_rng(seed + 100)
    p[ref.OB1:ref.OB4] = (0.1 * rng.standard_normal(ref.OB4 - ref.OB1)).astype(np.float32)
    p[ref.OB4:ref.OB4 + ref.NOUT] = (0.1 * rng.standard_normal(ref.NOUT)).astype(np.float32)
    return p


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize("n", [128, 300])
def test_gradient_matches_oracle(n):
    import torch
    p = _params(1)
    rng = np.random.default_rng(n)
    x = rng.standard_normal((n, 13)).astype(np.float32)
    t = rng.standard_normal((n, 9)).astype(np.float32)
    m = _net(p)
    loss, g = m.gradient(torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda(), n)
    m.close()
    p64 = p.astype(np.float64)
    l_bf, g_bf = ref.loss_and_grad(p64, x.astype(np.float64), t.astype(np.float64), bf=True)
    l_ex, g_ex = ref.loss_and_grad(p64, x.astype(np.float64), t.astype(np.float64), bf=False)
    assert abs(loss - l_bf) <= 1e-3 * l_bf, (loss, l_bf)
    for name, (a, b) in BLOCKS.items():
        assert _rel(g[a:b], g_bf[a:b]) <= 1e-2, (name, _rel(g[a:b], g_bf[a:b]))
        assert _rel(g[a:b], g_ex[a:b]) <= 5e-2, (name, _rel(g[a:b], g_ex[a:b]))


def test_inference_matches_oracle():
    import torch
    p = _params(2)
    n = 1000
    x = np.random.default_rng(5).standard_normal((n, 13)).astype(np.float32)
    m = _net(p)
    y = torch.zeros((n, 9), dtype=torch.float32, device="cuda")
    m.infer(torch.from_numpy(x).cuda(), y, n)
    m.close()
    yr = ref.forward(p.astype(np.float64), x.astype(np.float64), bf=True)
    assert _rel(y.cpu().numpy(), yr) <= 1e-2


def test_training_reduces_loss():
    """Adam on the device fits a smooth synthetic map well below the initial loss."""
    import torch
    rng = np.random.default_rng(9)
    n = 16384
    x = rng.standard_normal((n, 13)).astype(np.float32)
    A = rng.standard_normal((13, 9)).astype(np.float32) / 4.0
    t = np.tanh(x @ A) + 0.1 * (x[:, :9] ** 2)
    t = ((t - t.mean(0)) / t.std(0)).astype(np.float32)
    m = _net(ref.init_params(3))
    xd, td = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda()
    l0, _ = m.gradient(xd, td, n)
    m.train(xd, td, n, 2048, 600, 2e-3)
    l1, _ = m.gradient(xd, td, n)
    m.close()
    assert l1 < 0.2 * l0, (l0, l1)
