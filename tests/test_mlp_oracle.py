"""The CPU restatement of the learned closure (oracle/mlp.py): its exact FP64
gradient against central finite differences, its BF16 rounding, and the
padding invariants the CUDA layout relies on."""
import numpy as np

from oracle import mlp


def _batch(n=37, seed=3):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((n, mlp.NIN)), rng.standard_normal((n, mlp.NOUT))


def test_gradient_matches_finite_differences():
    p = mlp.init_params(1).astype(np.float64)
    p[mlp.OB1:mlp.NPAR] = 0.05 * np.random.default_rng(2).standard_normal(mlp.NPAR - mlp.OB1)
    p[mlp.OB4 + mlp.NOUT:] = 0.0
    x, t = _batch()
    _, g = mlp.loss_and_grad(p, x, t)
    rng = np.random.default_rng(4)
    live = [i for i in range(mlp.NPAR)
            if not (mlp.OW1 <= i < mlp.OW2 and (i - mlp.OW1) % mlp.KIN >= mlp.NIN)
            and not (mlp.OW4 <= i < mlp.OB1 and (i - mlp.OW4) // mlp.HID >= mlp.NOUT)
            and not (i >= mlp.OB4 + mlp.NOUT)]
    h = 1e-6
    for i in rng.choice(live, 40, replace=False):
        q = p.copy(); q[i] += h
        lp, _ = mlp.loss_and_grad(q, x, t)
        q[i] -= 2 * h
        lm, _ = mlp.loss_and_grad(q, x, t)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, g[i])


def test_padding_gradients_are_zero():
    p = mlp.init_params(5).astype(np.float64)
    x, t = _batch()
    for bf in (False, True):
        _, g = mlp.loss_and_grad(p, x, t, bf)
        w1 = g[mlp.OW1:mlp.OW2].reshape(mlp.HID, mlp.KIN)
        w4 = g[mlp.OW4:mlp.OB1].reshape(mlp.NOUTP, mlp.HID)
        assert not np.any(w1[:, mlp.NIN:]) and not np.any(w4[mlp.NOUT:]) and not np.any(g[mlp.OB4 + mlp.NOUT:])


def test_bf16_rounding():
    # ties to even at the 8-bit mantissa boundary, exact for representable values
    assert mlp.bf16(np.float32(1.0)) == 1.0
    assert mlp.bf16(np.float32(1.0 + 2.0 ** -8)) == 1.0            # tie -> even
    assert mlp.bf16(np.float32(1.0 + 3 * 2.0 ** -8)) == 1.0 + 2.0 ** -6
    assert mlp.bf16(np.float32(-2.5)) == -2.5
    x = np.random.default_rng(0).standard_normal(1000).astype(np.float32)
    assert np.max(np.abs(mlp.bf16(x) - x) / np.abs(x)) <= 2.0 ** -8


def test_bf16_form_is_close_to_exact():
    p = mlp.init_params(7).astype(np.float64)
    x, t = _batch(256)
    l64, g64 = mlp.loss_and_grad(p, x, t)
    l16, g16 = mlp.loss_and_grad(p, x, t, True)
    assert abs(l16 - l64) <= 2e-2 * l64
    assert np.linalg.norm(g16 - g64) <= 5e-2 * np.linalg.norm(g64)
