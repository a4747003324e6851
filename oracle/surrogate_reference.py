"""TEST INFRASTRUCTURE -- NumPy FP64 restatement of the learned radial
surrogate's network, the checker of its GPU training and inference kernels.

Only tests/ and bench.py import this module.  The network (rascaline_b200's
surrogate.hpp): x = 2 r / r_c - 1, h1 = silu(w1 x + b1), h2 = silu(W2 h1 + b2),
y = W3 h2 + b3 with the FP32 weights (the tensor cores read W2 and W3 as
sums of three BF16 parts, which reproduce them to 24 significant bits), or
with W2 and W3 rounded to one BF16 each (``bf16=True``, the single-BF16
control); the loss is the mean squared error of y against the normalised
targets.  ``fit_output_layer`` restates the least-squares refit of W3 and b3.
Parameters are packed as w1 [H], b1 [H], W2 [H][H], b2 [H], W3 [O][H],
b3 [O].
"""
import numpy as np


def bf16_round(a):
    """Round float32 values to the nearest BF16 (ties to even), as float64."""
    bits = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    rounded = (bits + 0x7FFF + ((bits >> 16) & 1)) & 0xFFFF0000
    return rounded.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(params, hidden, outputs, bf16=False):
    p = np.asarray(params, dtype=np.float32)
    H, O = hidden, outputs
    weights = bf16_round if bf16 else (lambda a: a.astype(np.float64))
    o = 0
    w1 = p[o:o + H].astype(np.float64); o += H
    b1 = p[o:o + H].astype(np.float64); o += H
    W2 = weights(p[o:o + H * H]).reshape(H, H); o += H * H
    b2 = p[o:o + H].astype(np.float64); o += H
    W3 = weights(p[o:o + O * H]).reshape(O, H); o += O * H
    b3 = p[o:o + O].astype(np.float64); o += O
    assert o == len(p)
    return w1, b1, W2, b2, W3, b3


def _silu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return z * s, s * (1.0 + z * (1.0 - s))


def hidden_features(params, hidden, outputs, r, cutoff, bf16=False):
    """h2 [n, H] and dh2/dr [n, H]."""
    w1, b1, W2, b2, W3, b3 = unpack(params, hidden, outputs, bf16)
    x = 2.0 * np.asarray(r, dtype=np.float64) / cutoff - 1.0
    z1 = np.outer(x, w1) + b1
    h1, s1 = _silu(z1)
    dh1 = s1 * w1 * (2.0 / cutoff)
    z2 = h1 @ W2.T + b2
    h2, s2 = _silu(z2)
    return h2, s2 * (dh1 @ W2.T)


def fit_output_layer(params, hidden, outputs, r, targets, dtargets, cutoff, derivative_weight):
    """Parameters with W3, b3 replaced by the least-squares solution of
    min |[h2, 1] W - y|^2 + lambda |[dh2/dx, 0] W - dy/dx|^2 over the
    samples (normalised targets, ``dtargets`` their r-derivatives;
    x = 2 r / r_c - 1), FP64."""
    H, O = hidden, outputs
    h2, dh2 = hidden_features(params, H, O, r, cutoff)
    dxdr = 0.5 * cutoff
    F = np.hstack([h2, np.ones((len(r), 1))])
    D = np.hstack([dh2 * dxdr, np.zeros((len(r), 1))])
    A = F.T @ F + derivative_weight * D.T @ D
    B = F.T @ targets + derivative_weight * D.T @ (dtargets * dxdr)
    A = A + 1e-13 * np.trace(A) / (H + 1) * np.eye(H + 1)
    W = np.linalg.solve(A, B)
    p = np.array(params, dtype=np.float64)
    o3 = 3 * H + H * H
    p[o3:o3 + O * H] = W[:H].T.reshape(-1)
    p[o3 + O * H:o3 + O * H + O] = W[H]
    return p


def forward(params, hidden, outputs, r, cutoff, bf16=False):
    """Normalised outputs y [n, O] and dy/dr [n, O]."""
    w1, b1, W2, b2, W3, b3 = unpack(params, hidden, outputs, bf16)
    x = 2.0 * np.asarray(r, dtype=np.float64) / cutoff - 1.0
    z1 = np.outer(x, w1) + b1
    h1, s1 = _silu(z1)
    dh1 = s1 * w1 * (2.0 / cutoff)
    z2 = h1 @ W2.T + b2
    h2, s2 = _silu(z2)
    dh2 = s2 * (dh1 @ W2.T)
    return h2 @ W3.T + b3, dh2 @ W3.T


def loss_and_gradient(params, hidden, outputs, r, targets, cutoff, dtargets=None, derivative_weight=0.0):
    """Loss and its gradient w.r.t. the packed parameters, FP64.  The loss is
    the mean squared error of the normalised outputs y, plus
    ``derivative_weight`` times that of dy/dx against ``dtargets`` (dy/dr of
    the normalised targets) times r_c / 2, x = 2 r / r_c - 1.  The gradient
    comes from torch's reverse-mode autograd on the CPU (second derivatives
    through the forward-mode derivative included), an implementation
    independent of the GPU kernels' hand-written backward pass."""
    import torch

    H, O = hidden, outputs
    p = torch.tensor(np.asarray(params, dtype=np.float32).astype(np.float64), requires_grad=True)
    o = 0
    w1 = p[o:o + H]; o += H
    b1 = p[o:o + H]; o += H
    W2 = p[o:o + H * H].reshape(H, H); o += H * H
    b2 = p[o:o + H]; o += H
    W3 = p[o:o + O * H].reshape(O, H); o += O * H
    b3 = p[o:o + O]
    x = torch.tensor(2.0 * np.asarray(r, dtype=np.float64) / cutoff - 1.0)
    z1 = torch.outer(x, w1) + b1
    s1 = torch.sigmoid(z1)
    h1 = z1 * s1
    dh1 = s1 * (1 + z1 * (1 - s1)) * w1
    z2 = h1 @ W2.T + b2
    s2 = torch.sigmoid(z2)
    h2 = z2 * s2
    dh2 = s2 * (1 + z2 * (1 - s2)) * (dh1 @ W2.T)
    y = h2 @ W3.T + b3
    loss = torch.mean((y - torch.tensor(targets)) ** 2)
    if derivative_weight:
        dy = dh2 @ W3.T
        dt = torch.tensor(np.asarray(dtargets, dtype=np.float64)) * (0.5 * cutoff)
        loss = loss + derivative_weight * torch.mean((dy - dt) ** 2)
    loss.backward()
    return float(loss.detach()), p.grad.numpy().copy()
