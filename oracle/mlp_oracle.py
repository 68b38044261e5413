"""Oracle: the surrogate MLP's forward and backward pass in float64 NumPy.

Test infrastructure only.  It restates the device computation of
csrc/sidr_surrogate.cu -- inputs padded from 40 to 48 columns, BF16 copies of
the inputs, of W1 and W2 and of the hidden activations, ReLU, a 256 -> 1 head
in full precision, mean squared error -- with every rounding to BF16 made at
the same place (bf16=True), or with none (bf16=False, a smooth float64 model
for finite-difference checks of the backward formulas).
"""
from __future__ import annotations

import numpy as np


def bf16(x):
    u = np.asarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint32) << 16
    return r.view(np.float32).astype(np.float64)


def forward(params, x, rounding=True):
    q = bf16 if rounding else (lambda a: np.asarray(a, dtype=np.float64))
    W1, b1, W2, b2, w3, b3 = (np.asarray(params[k], np.float64) for k in
                              ("W1", "b1", "W2", "b2", "w3", "b3"))
    xp = np.zeros((x.shape[0], 48))
    xp[:, :40] = x
    xb = q(xp)
    z1 = xb @ q(W1).T + b1
    h1 = q(np.maximum(z1, 0.0))
    z2 = h1 @ q(W2).T + b2
    h2 = q(np.maximum(z2, 0.0))
    y = h2 @ w3 + b3[0]
    return {"xb": xb, "h1": h1, "h2": h2, "y": y, "W1q": q(W1), "W2q": q(W2)}


def loss_and_grads(params, x, t, rounding=True):
    q = bf16 if rounding else (lambda a: np.asarray(a, dtype=np.float64))
    f = forward(params, x, rounding)
    B = x.shape[0]
    d = f["y"] - np.asarray(t, np.float64)
    loss = np.mean(d * d)
    dy = 2.0 * d / B
    w3 = np.asarray(params["w3"], np.float64)
    g = {"w3": f["h2"].T @ dy, "b3": np.array([dy.sum()])}
    dz2 = np.where(f["h2"] > 0, dy[:, None] * w3[None, :], 0.0)
    g["b2"] = dz2.sum(axis=0)
    dz2q = q(dz2)
    g["W2"] = dz2q.T @ f["h1"]
    dh1 = dz2q @ f["W2q"]
    dz1 = np.where(f["h1"] > 0, dh1, 0.0)
    g["b1"] = dz1.sum(axis=0)
    g["W1"] = q(dz1).T @ f["xb"]
    return loss, g
