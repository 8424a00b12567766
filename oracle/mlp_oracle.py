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


def row_features(A, B):
    """Predictor features of every row of A*B, float32 (rows x 8), restating
    the feature kernel (rtspmspm_b200/csrc/mlp.cu, tile_stats / feature_of):
    |A_r|, products, max / min touched |B_k|, cols of B, output column span,
    the distinct fraction of a 32-product sample and the Erdos-Renyi
    expected distinct count, each log2(1 + x) / 16 except the fraction.
    The sample: rows of at most 32 entries take one product per entry q
    with slot q; longer rows take entry floor(l * len / 32) with slot l; a
    slot picks B row entry hash % |B_k|, hash = r * 2654435761 + slot * 40503
    (mod 2^32).  Returns (features, integer stats dict)."""
    rp = np.asarray(A.row_ptr, np.int64)
    brp = np.asarray(B.row_ptr, np.int64)
    bcol = np.asarray(B.col_idx, np.int64)
    rows = A.rows
    ln = np.diff(rp)
    k = np.asarray(A.col_idx, np.int64)
    row_of = np.repeat(np.arange(rows, dtype=np.int64), ln)
    q = np.arange(k.size, dtype=np.int64) - rp[row_of]
    bs, be = brp[k], brp[k + 1]
    l = be - bs
    sums = np.zeros(rows, np.int64)
    np.add.at(sums, row_of, l)
    mx = np.zeros(rows, np.int64)
    np.maximum.at(mx, row_of, l)
    mn = np.full(rows, np.iinfo(np.int64).max, np.int64)
    np.minimum.at(mn, row_of, l)
    mn[ln == 0] = 0
    nz = l > 0
    lo = np.full(rows, np.iinfo(np.int64).max, np.int64)
    hi = np.full(rows, -1, np.int64)
    np.minimum.at(lo, row_of[nz], bcol[bs[nz]])
    np.maximum.at(hi, row_of[nz], bcol[be[nz] - 1])
    # sample slots
    lr = ln[row_of]
    short = lr <= 32
    slot = np.where(short, q, (32 * q + lr - 1) // np.maximum(lr, 1))
    sampled = nz & (short | ((slot < 32) & ((slot * lr) // 32 == q)))
    r_s, s_s = row_of[sampled], slot[sampled]
    hsh = (((r_s & 0xFFFFFFFF) * 2654435761) + s_s * 40503) & 0xFFFFFFFF
    j = bcol[bs[sampled] + hsh % l[sampled]]
    nsample = np.bincount(r_s, minlength=rows)
    pairs = np.unique(np.stack([r_s, j], 1), axis=0) if r_s.size else np.zeros((0, 2), np.int64)
    distinct = np.bincount(pairs[:, 0], minlength=rows) if pairs.size else np.zeros(rows, np.int64)
    f32 = np.float32
    cols = f32(B.cols)
    fsum = sums.astype(f32)
    span = np.where(hi >= lo, (hi - lo + 1), 0).astype(f32)
    with np.errstate(divide="ignore", invalid="ignore"):
        frac = np.where(nsample > 0, distinct.astype(f32) / np.maximum(nsample, 1).astype(f32), f32(0))
        er = (-cols * np.expm1(-fsum / cols)).astype(f32) if cols > 0 else np.zeros(rows, f32)
    raw = [ln.astype(f32), fsum, mx.astype(f32), mn.astype(f32), np.full(rows, cols, f32), span, None, er]
    feats = np.zeros((rows, IN), f32)
    for i, x in enumerate(raw):
        feats[:, i] = frac if x is None else (np.log2(f32(1) + x) / f32(16)).astype(f32)
    stats = {"len": ln, "sum": sums, "mx": mx, "mn": mn, "lo": lo, "hi": hi,
             "distinct": distinct, "nsample": nsample}
    return feats, stats
