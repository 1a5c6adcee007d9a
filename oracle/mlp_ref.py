"""CPU float64 restatement of the subtree-size model -- TEST INFRASTRUCTURE ONLY.

The oracle for the library's FP16/FP32 MLP kernels (gmkbe_b200/csrc/mlp.cuh):
the same 16-64-64-1 ReLU network, the same parameter layout
(W1[64][16] b1[64] W2[64][64] b2[64] W3[64] b3), the same mean-squared-error
loss, computed in float64 from the FP16-rounded weights and inputs the kernels
read.  Only tests/ import it.
"""
from __future__ import annotations

import numpy as np

F, H = 16, 64
OFF_W1 = 0
OFF_B1 = OFF_W1 + H * F
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H * H
OFF_W3 = OFF_B2 + H
OFF_B3 = OFF_W3 + H
NP = OFF_B3 + 1


def _unpack(p, fp16=True):
    p = np.asarray(p, np.float64)
    if fp16:
        p = p.astype(np.float32).astype(np.float16).astype(np.float64)
    return (p[OFF_W1:OFF_B1].reshape(H, F), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(H, H),
            p[OFF_B2:OFF_W3], p[OFF_W3:OFF_B3], p[OFF_B3])


def forward(p, x, fp16=True):
    """Predictions for x (n, 16), weights and inputs rounded to FP16 as the
    kernels read them (fp16=False: exact float64, for finite differences)."""
    w1, b1, w2, b2, w3, b3 = _unpack(p, fp16)
    x = np.asarray(x, np.float64)
    if fp16:
        x = x.astype(np.float32).astype(np.float16).astype(np.float64)
    h1 = np.maximum(x @ w1.T + b1, 0.0)
    h2 = np.maximum(h1 @ w2.T + b2, 0.0)
    return h2 @ w3 + b3, h1, h2, x


def loss_and_gradient(p, x, y, fp16=True):
    """Mean squared error and its gradient with respect to the parameters."""
    w1, b1, w2, b2, w3, b3 = _unpack(p, fp16)
    out, h1, h2, xr = forward(p, x, fp16)
    y = np.asarray(y, np.float64)
    n = y.size
    e = out - y
    loss = float(np.mean(e * e))
    dout = 2.0 * e / n
    g = np.zeros(NP, np.float64)
    g[OFF_B3] = dout.sum()
    g[OFF_W3:OFF_B3] = dout @ h2
    dh2 = np.outer(dout, w3) * (h2 > 0)
    g[OFF_B2:OFF_W3] = dh2.sum(0)
    g[OFF_W2:OFF_B2] = (dh2.T @ h1).ravel()
    dh1 = (dh2 @ w2) * (h1 > 0)
    g[OFF_B1:OFF_W2] = dh1.sum(0)
    g[OFF_W1:OFF_B1] = (dh1.T @ xr).ravel()
    return loss, g
