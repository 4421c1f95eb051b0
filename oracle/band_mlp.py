"""CPU restatement of the band MLP's training objective (test infrastructure).

Used only by the tests to check the GPU training kernels: forward, loss and
analytical gradient in FP64, with the same BF16 rounding as the GPU -- of the
weight matrices, the inputs and hidden activations (biases stay FP32), and of
the hidden-layer gradients where they enter the tensor-core products (the
weight gradients of both hidden layers and the back-propagated gradient of
the first; the bias gradients sum the unrounded values) -- with the gradient
passed straight through every rounding, or without any rounding for the
finite-difference check that pins the analytical gradient.

Network: 80 -> 128 (ReLU) -> 128 (ReLU) -> 2; parameters flattened as
W1[128][80], b1[128], W2[128][128], b2[128], W3[2][128], b3[2].
Loss: mean over rows of w_lo (o_lo - t_lo)^2 + w_hi (o_hi - t_hi)^2 with
w_lo = alpha when o_lo > t_lo, w_hi = alpha when o_hi < t_hi, else 1.
The learned band has no counterpart in the reference; this objective is the
one the GPU trainer (phmm_mlp_train.cu) defines.
"""
from __future__ import annotations

import numpy as np

FEAT, HID, OUT = 80, 128, 2
SHAPES = [(HID, FEAT), (HID,), (HID, HID), (HID,), (OUT, HID), (OUT,)]
N_PARAMS = sum(int(np.prod(s)) for s in SHAPES)


def bf16_round(x: np.ndarray) -> np.ndarray:
    """Round to the nearest BF16 (ties to even), returned as float64."""
    f = np.asarray(x, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32).astype(np.float64)
    return np.where(np.isfinite(f), out, f.astype(np.float64))


def unpack(w: np.ndarray):
    parts, off = [], 0
    for s in SHAPES:
        n = int(np.prod(s))
        parts.append(np.asarray(w[off:off + n], np.float64).reshape(s))
        off += n
    return parts


def objective(w: np.ndarray, x: np.ndarray, t: np.ndarray, alpha: float, rounding: bool = True):
    """(outputs [n, 2], loss, gradient [N_PARAMS]) in FP64."""
    W1, b1, W2, b2, W3, b3 = unpack(w)
    if rounding:
        W1, W2, W3 = bf16_round(W1), bf16_round(W2), bf16_round(W3)
    rnd = bf16_round if rounding else (lambda a: a)
    x = rnd(np.asarray(x, np.float64))
    t = np.asarray(t, np.float64)
    n = x.shape[0]
    z1 = x @ W1.T + b1
    h1 = rnd(np.maximum(z1, 0))
    z2 = h1 @ W2.T + b2
    h2 = rnd(np.maximum(z2, 0))
    o = h2 @ W3.T + b3
    e = o - t
    wgt = np.ones_like(e)
    wgt[:, 0] = np.where(e[:, 0] > 0, alpha, 1.0)
    wgt[:, 1] = np.where(e[:, 1] < 0, alpha, 1.0)
    loss = float(np.sum(wgt * e * e) / n)
    do = 2.0 * wgt * e / n
    gW3, gb3 = do.T @ h2, do.sum(0)
    dh2 = (do @ W3) * (z2 > 0)
    gW2, gb2 = rnd(dh2).T @ h1, dh2.sum(0)
    dh1 = (rnd(dh2) @ W2) * (z1 > 0)
    gW1, gb1 = rnd(dh1).T @ x, dh1.sum(0)
    g = np.concatenate([a.ravel() for a in (gW1, gb1, gW2, gb2, gW3, gb3)])
    return o, loss, g


def init_weights(seed: int = 0, out_scale: float = 0.1) -> np.ndarray:
    rng = np.random.default_rng(seed)
    parts = []
    for s in SHAPES:
        if len(s) == 2:
            a = np.sqrt(6.0 / s[1]) * (out_scale if s[0] == OUT else 1.0)
            parts.append(rng.uniform(-a, a, s).ravel())
        else:
            parts.append(rng.uniform(-0.1, 0.1, s))
    return np.concatenate(parts).astype(np.float32)
