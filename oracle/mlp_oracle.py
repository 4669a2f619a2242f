"""CPU oracle of the learned (m, s) selector network (TEST INFRASTRUCTURE ONLY).

Only tests/ use it, as the checker of the device kernels in fastctqw_b200/csrc/fx_selector.cu
(inference, fused forward/backward).  FP64 numpy restatement of the same network and loss:
MLP 8 -> 64 -> 64 -> 6 with ReLU, weights in the order W1 [64 x 8], b1, W2 [64 x 64], b2,
W3 [6 x 64], b3; loss per sample = cross-entropy of the first 5 outputs against the class label
+ lambda (o_5 - s)^2, averaged over the batch.
"""
from __future__ import annotations

import numpy as np


def unpack(w):
    w = np.asarray(w, dtype=np.float64)
    o = 0
    out = []
    for shape in ((64, 8), (64,), (64, 64), (64,), (6, 64), (6,)):
        size = int(np.prod(shape))
        out.append(w[o:o + size].reshape(shape))
        o += size
    assert o == w.size == 5126
    return out


def forward(w, x):
    W1, b1, W2, b2, W3, b3 = unpack(w)
    z1 = x @ W1.T + b1
    h1 = np.maximum(z1, 0)
    z2 = h1 @ W2.T + b2
    h2 = np.maximum(z2, 0)
    return h2 @ W3.T + b3, (z1, h1, z2, h2)


def loss_grad(w, x, ym, ys, lam):
    """(mean loss, gradient w.r.t. the 5126 weights) in FP64."""
    x = np.asarray(x, dtype=np.float64)
    n = x.shape[0]
    W1, b1, W2, b2, W3, b3 = unpack(w)
    o, (z1, h1, z2, h2) = forward(w, x)
    logits = o[:, :5]
    mx = logits.max(axis=1, keepdims=True)
    lse = mx[:, 0] + np.log(np.exp(logits - mx).sum(axis=1))
    ds = o[:, 5] - ys
    loss = np.mean(lse - logits[np.arange(n), ym] + lam * ds * ds)
    do = np.zeros_like(o)
    do[:, :5] = np.exp(logits - lse[:, None])
    do[np.arange(n), ym] -= 1.0
    do[:, 5] = 2.0 * lam * ds
    do /= n
    gW3 = do.T @ h2
    gb3 = do.sum(axis=0)
    d2 = (do @ W3) * (z2 > 0)
    gW2 = d2.T @ h1
    gb2 = d2.sum(axis=0)
    d1 = (d2 @ W2) * (z1 > 0)
    gW1 = d1.T @ x
    gb1 = d1.sum(axis=0)
    return loss, np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
