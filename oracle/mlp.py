"""FP64 CPU restatement of the selector MLP (12 -> 32 -> 32 -> 6, ReLU),
its masked mean-squared-error loss and the loss gradient.

TEST INFRASTRUCTURE ONLY: the checker of the device forward / backward
kernels (sg_mlp_forward, sg_mlp_gradient).  Parameters use the flat layout of
MlpParams: w1[32][12], b1[32], w2[32][32], b2[32], w3[6][32], b3[6],
mean[12], inv_std[12], lo[12], hi[12]."""
from __future__ import annotations

import numpy as np

IN, HID, OUT = 12, 32, 6
SHAPES = [("w1", (HID, IN)), ("b1", (HID,)), ("w2", (HID, HID)), ("b2", (HID,)), ("w3", (OUT, HID)), ("b3", (OUT,)),
          ("mean", (IN,)), ("inv_std", (IN,)), ("lo", (IN,)), ("hi", (IN,))]
TRAINABLE = ("w1", "b1", "w2", "b2", "w3", "b3")


def unpack(flat):
    out, o = {}, 0
    for name, shp in SHAPES:
        k = int(np.prod(shp))
        out[name] = np.asarray(flat[o:o + k], dtype=np.float64).reshape(shp)
        o += k
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], np.float64).reshape(-1) for name, _ in SHAPES])


def forward(flat, X):
    p = unpack(flat)
    x = (np.asarray(X, np.float64) - p["mean"]) * p["inv_std"]
    a1 = x @ p["w1"].T + p["b1"]
    h1 = np.maximum(a1, 0)
    a2 = h1 @ p["w2"].T + p["b2"]
    h2 = np.maximum(a2, 0)
    y = h2 @ p["w3"].T + p["b3"]
    return y, (x, a1, h1, a2, h2)


def loss_and_grad(flat, X, T, M):
    """loss = mean over samples and outputs of 0.5 * M * (y - T)^2."""
    p = unpack(flat)
    y, (x, a1, h1, a2, h2) = forward(flat, X)
    n = len(X)
    scale = 1.0 / (n * OUT)
    d = (y - T) * M
    loss = 0.5 * np.sum(M * (y - T) ** 2) * scale
    dy = d * scale
    g = {k: np.zeros_like(v) for k, v in p.items()}
    g["w3"] = dy.T @ h2
    g["b3"] = dy.sum(0)
    dh2 = (dy @ p["w3"]) * (a2 > 0)
    g["w2"] = dh2.T @ h1
    g["b2"] = dh2.sum(0)
    dh1 = (dh2 @ p["w2"]) * (a1 > 0)
    g["w1"] = dh1.T @ x
    g["b1"] = dh1.sum(0)
    return loss, pack(g)
