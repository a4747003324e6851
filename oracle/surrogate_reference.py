"""TEST INFRASTRUCTURE -- NumPy FP64 restatement of the learned radial
surrogate's network, the checker of its GPU training and inference kernels.

Only tests/ and bench.py import this module.  The network (rascaline_b200's
surrogate.hpp): x = 2 r / r_c - 1, h1 = silu(w1 x + b1), h2 = silu(W2 h1 + b2),
y = W3 h2 + b3, with W2 and W3 rounded to BF16 (round to nearest even) as the
tensor cores read them; the loss is the mean squared error of y against the
normalised targets.  Parameters are packed as w1 [H], b1 [H], W2 [H][H],
b2 [H], W3 [O][H], b3 [O].
"""
import numpy as np


def bf16_round(a):
    """Round float32 values to the nearest BF16 (ties to even), as float64."""
    bits = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    rounded = (bits + 0x7FFF + ((bits >> 16) & 1)) & 0xFFFF0000
    return rounded.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(params, hidden, outputs):
    p = np.asarray(params, dtype=np.float32)
    H, O = hidden, outputs
    o = 0
    w1 = p[o:o + H].astype(np.float64); o += H
    b1 = p[o:o + H].astype(np.float64); o += H
    W2 = bf16_round(p[o:o + H * H]).reshape(H, H); o += H * H
    b2 = p[o:o + H].astype(np.float64); o += H
    W3 = bf16_round(p[o:o + O * H]).reshape(O, H); o += O * H
    b3 = p[o:o + O].astype(np.float64); o += O
    assert o == len(p)
    return w1, b1, W2, b2, W3, b3


def _silu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return z * s, s * (1.0 + z * (1.0 - s))


def forward(params, hidden, outputs, r, cutoff):
    """Normalised outputs y [n, O] and dy/dr [n, O]."""
    w1, b1, W2, b2, W3, b3 = unpack(params, hidden, outputs)
    x = 2.0 * np.asarray(r, dtype=np.float64) / cutoff - 1.0
    z1 = np.outer(x, w1) + b1
    h1, s1 = _silu(z1)
    dh1 = s1 * w1 * (2.0 / cutoff)
    z2 = h1 @ W2.T + b2
    h2, s2 = _silu(z2)
    dh2 = s2 * (dh1 @ W2.T)
    return h2 @ W3.T + b3, dh2 @ W3.T


def loss_and_gradient(params, hidden, outputs, r, targets, cutoff):
    """Mean squared error and its gradient w.r.t. the packed parameters
    (straight through the BF16 rounding)."""
    w1, b1, W2, b2, W3, b3 = unpack(params, hidden, outputs)
    n = len(r)
    x = 2.0 * np.asarray(r, dtype=np.float64) / cutoff - 1.0
    z1 = np.outer(x, w1) + b1
    h1, s1 = _silu(z1)
    z2 = h1 @ W2.T + b2
    h2, s2 = _silu(z2)
    y = h2 @ W3.T + b3
    d = y - targets
    loss = float(np.mean(d * d))
    dy = 2.0 * d / (n * outputs)
    gW3 = dy.T @ h2
    gb3 = dy.sum(axis=0)
    dz2 = (dy @ W3) * s2
    gW2 = dz2.T @ h1
    gb2 = dz2.sum(axis=0)
    dz1 = (dz2 @ W2) * s1
    gw1 = dz1.T @ x
    gb1 = dz1.sum(axis=0)
    return loss, np.concatenate([gw1, gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
