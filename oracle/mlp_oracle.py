"""FP64 CPU reference of the row-size predictor -- TEST INFRASTRUCTURE ONLY.

Checks the engine's MLP kernels (rtspmspm_b200/csrc/mlp.cu).  The network is
8 -> 64 -> 64 -> 2 with ReLU, parameters packed as W1[8x64] b1[64]
W2[64x64] b2[64] W3[64x2] b3[2] (row-major, in x out).  The engine runs it
with BF16 weights (and, in the tensor-core inference, BF16 activations) and
FP32 accumulation; the helpers here round the same operands to BF16 and do
everything else in FP64, so the comparison isolates accumulation error.

Loss: 0.5 * mean over rows of (y0 - t0)^2 + 0.25 (y1 - t1)^2.
No reference counterpart (the reference has no predictor).
"""
from __future__ import annotations

import numpy as np

IN, HID, OUT = 8, 64, 2
LOSS_W = np.array([1.0, 0.25])


def bf16_round(x: np.ndarray) -> np.ndarray:
    """Round-to-nearest-even to bfloat16, returned as float64."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    rounding = ((u >> 16) & 1) + 0x7FFF
    u = ((u + rounding) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p: np.ndarray):
    p = np.asarray(p, dtype=np.float64)
    o = 0
    W1 = p[o:o + IN * HID].reshape(IN, HID); o += IN * HID
    b1 = p[o:o + HID]; o += HID
    W2 = p[o:o + HID * HID].reshape(HID, HID); o += HID * HID
    b2 = p[o:o + HID]; o += HID
    W3 = p[o:o + HID * OUT].reshape(HID, OUT); o += HID * OUT
    b3 = p[o:o + OUT]; o += OUT
    assert o == p.size
    return W1, b1, W2, b2, W3, b3


def forward(params, x, bf16_weights=True, bf16_acts=False):
    """Returns (y, cache). x: rows x 8."""
    ps = bf16_round(params) if bf16_weights else np.asarray(params, np.float64)
    W1, b1, W2, b2, W3, b3 = unpack(ps)
    r = bf16_round if bf16_acts else (lambda v: np.asarray(v, np.float64))
    x = np.asarray(x, np.float64)
    z1 = r(x) @ W1 + b1
    h1 = np.maximum(z1, 0.0)
    z2 = r(h1) @ W2 + b2
    h2 = np.maximum(z2, 0.0)
    y = r(h2) @ W3 + b3
    return y, (x, z1, h1, z2, h2, W1, W2, W3)


def loss_and_grad(params, x, t):
    """Mean loss and the gradient of every parameter (BF16 weights, FP64 math)."""
    y, (x, z1, h1, z2, h2, W1, W2, W3) = forward(params, x)
    n = x.shape[0]
    diff = y - np.asarray(t, np.float64)
    loss = 0.5 * np.mean((diff ** 2) @ LOSS_W)
    dy = diff * LOSS_W / n
    gW3 = h2.T @ dy
    gb3 = dy.sum(0)
    dz2 = (dy @ W3.T) * (z2 > 0)
    gW2 = h1.T @ dz2
    gb2 = dz2.sum(0)
    dz1 = (dz2 @ W2.T) * (z1 > 0)
    gW1 = x.T @ dz1
    gb1 = dz1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return float(loss), g
