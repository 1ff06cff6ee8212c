"""TEST INFRASTRUCTURE ONLY: CPU restatement of the learned subgrid closure.

The network is 13 -> 64 -> 64 -> 64 -> 9 with GELU in its tanh form
(0.5 z (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3)))) after the three hidden layers and a mean squared
error loss sum((y - t)^2) / (n * 9).  Parameters use the padded layout of the
CUDA implementation (erf_b200/csrc/mlp.cu):

    W1[64][16] W2[64][64] W3[64][64] W4[16][64] b1[64] b2[64] b3[64] b4[16]

(columns 13..15 of W1 and rows 9..15 of W4 are padding and stay zero).

Two forms are provided:
  * ``loss_and_grad(..., bf16=False)``: exact FP64 forward and backward (the
    reference for finite-difference checks);
  * ``loss_and_grad(..., bf16=True)``: the same arithmetic with the operands of
    every tensor-core product rounded to BF16 at the points where the CUDA
    kernels round them (inputs, weights, hidden activations, and the
    backpropagated dZ before it enters dW = dZ^T H and dX = dZ W), with FP64
    accumulation standing in for the FP32 tensor-memory accumulators.

Only tests/ may import this module.
"""
from __future__ import annotations

import math

import numpy as np

NIN, KIN, HID, NOUT, NOUTP = 13, 16, 64, 9, 16
OW1 = 0
OW2 = OW1 + HID * KIN
OW3 = OW2 + HID * HID
OW4 = OW3 + HID * HID
OB1 = OW4 + NOUTP * HID
OB2 = OB1 + HID
OB3 = OB2 + HID
OB4 = OB3 + HID
NPAR = OB4 + NOUTP


def bf16(a):
    """Round to bfloat16 (round to nearest, ties to even), returned as float64."""
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
    b = a.view(np.uint32).astype(np.uint64)
    r = ((b >> 16) & 1) + 0x7FFF
    out = ((b + r) & 0xFFFF0000).astype(np.uint32).view(np.float32)
    return out.astype(np.float64)


GELU_C, GELU_A = math.sqrt(2.0 / math.pi), 0.044715


def gelu(z):
    """GELU, tanh form (Hendrycks & Gimpel 2016)."""
    return 0.5 * z * (1.0 + np.tanh(GELU_C * (z + GELU_A * z ** 3)))


def gelu_grad(z):
    t = np.tanh(GELU_C * (z + GELU_A * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * GELU_C * (1.0 + 3.0 * GELU_A * z * z)


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    W1 = p[OW1:OW2].reshape(HID, KIN)
    W2 = p[OW2:OW3].reshape(HID, HID)
    W3 = p[OW3:OW4].reshape(HID, HID)
    W4 = p[OW4:OB1].reshape(NOUTP, HID)
    return W1, W2, W3, W4, p[OB1:OB2], p[OB2:OB3], p[OB3:OB4], p[OB4:NPAR]


def init_params(seed=0):
    """He-style initial weights (deterministic), zero biases, zero padding."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NPAR, dtype=np.float32)
    p[OW1:OW2] = (rng.standard_normal((HID, KIN)) * math.sqrt(2.0 / NIN) * (np.arange(KIN) < NIN)).ravel()
    p[OW2:OW3] = (rng.standard_normal((HID, HID)) * math.sqrt(2.0 / HID)).ravel()
    p[OW3:OW4] = (rng.standard_normal((HID, HID)) * math.sqrt(2.0 / HID)).ravel()
    p[OW4:OB1] = (rng.standard_normal((NOUTP, HID)) * math.sqrt(1.0 / HID) * (np.arange(NOUTP) < NOUT)[:, None]).ravel()
    return p


def forward(p, xn, bf=False):
    """Outputs y [n][9] for normalised inputs xn [n][13]."""
    return _run(p, xn, None, bf)[0]


def loss_and_grad(p, xn, tn, bf=False):
    """(loss, gradient in the padded layout) for normalised inputs/targets."""
    _, loss, grad = _run(p, xn, tn, bf)
    return loss, grad


def _run(p, xn, tn, bf):
    r = bf16 if bf else (lambda a: np.asarray(a, dtype=np.float64))
    W1, W2, W3, W4, b1, b2, b3, b4 = unpack(p)
    n = xn.shape[0]
    X0 = np.zeros((n, KIN))
    X0[:, :NIN] = xn
    X0 = r(X0)
    Ws = [r(W1), r(W2), r(W3), r(W4)]
    bs = [b1, b2, b3, b4]
    H = [X0]
    Z = []
    for layer in range(3):
        z = H[-1] @ Ws[layer].T
        Z.append(z)
        H.append(r(gelu(z + bs[layer])))
    y = H[-1] @ Ws[3].T + b4
    if tn is None:
        return y[:, :NOUT], None, None
    e = np.zeros((n, NOUTP))
    e[:, :NOUT] = y[:, :NOUT] - tn
    inv = 1.0 / (n * NOUT)
    loss = float(np.sum(e * e) * inv)
    dz = 2.0 * e * inv
    g = np.zeros(NPAR)
    offs_w = [OW1, OW2, OW3, OW4]
    offs_b = [OB1, OB2, OB3, OB4]
    for layer in range(3, -1, -1):
        g[offs_b[layer]:offs_b[layer] + dz.shape[1]] = dz.sum(axis=0)
        dzr = r(dz)
        dW = dzr.T @ H[layer]
        g[offs_w[layer]:offs_w[layer] + dW.size] = dW.ravel()
        if layer > 0:
            dx = dzr @ Ws[layer]
            dz = dx * gelu_grad(Z[layer - 1] + bs[layer - 1])
    return y[:, :NOUT], loss, g
