"""Oracle of the precision-tier network (test infrastructure only: the tests
import it as the checker of the CUDA kernels; the product never calls it).

A plain numpy float64 statement of the network the library trains and runs
on the GPU (rslab_tier_mlp_forward / _grad / _train): 8 -> 64 -> 64 -> 3,
ReLU hidden layers, softmax output, weighted mean cross-entropy
sum_s w_s CE_s / sum_s w_s, full-batch Adam (beta 0.9 / 0.999, eps 1e-8).
The network has no counterpart in the reference, so its definition is the
mathematics above; parity with the kernels is within FP32 tolerance.
Parameter layout: W1[64][8], b1[64], W2[64][64], b2[64], W3[3][64], b3[3].
"""
from __future__ import annotations

import numpy as np

IN, HID, OUT = 8, 64, 3
SHAPES = (("W1", (HID, IN)), ("b1", (HID,)), ("W2", (HID, HID)), ("b2", (HID,)), ("W3", (OUT, HID)),
          ("b3", (OUT,)))
NPARAM = sum(int(np.prod(s)) for _, s in SHAPES)


def unpack(p: np.ndarray) -> dict:
    out, o = {}, 0
    for name, shape in SHAPES:
        k = int(np.prod(shape))
        out[name] = np.asarray(p[o:o + k], np.float64).reshape(shape)
        o += k
    return out


def pack(d: dict) -> np.ndarray:
    return np.concatenate([np.asarray(d[name], np.float64).ravel() for name, _ in SHAPES])


def forward(p, x):
    """(probs, cache) for samples x (m x 8)."""
    P = unpack(p)
    x = np.asarray(x, np.float64)
    a1 = x @ P["W1"].T + P["b1"]
    h1 = np.maximum(a1, 0.0)
    a2 = h1 @ P["W2"].T + P["b2"]
    h2 = np.maximum(a2, 0.0)
    z = h2 @ P["W3"].T + P["b3"]
    z = z - z.max(axis=1, keepdims=True)
    e = np.exp(z)
    probs = e / e.sum(axis=1, keepdims=True)
    return probs, (x, h1, h2, z, e)


def loss_and_grad(p, x, y, w=None):
    """Weighted mean cross-entropy and its gradient (flat, the layout above)."""
    P = unpack(p)
    probs, (x, h1, h2, z, e) = forward(p, x)
    m = x.shape[0]
    y = np.asarray(y, np.int64)
    w = np.ones(m) if w is None else np.asarray(w, np.float64)
    ws = w.sum()
    ce = np.log(e.sum(axis=1)) - z[np.arange(m), y]
    loss = float((w * ce).sum() / ws)
    dz = probs.copy()
    dz[np.arange(m), y] -= 1.0
    dz *= (w / ws)[:, None]
    g = {"W3": dz.T @ h2, "b3": dz.sum(0)}
    dh2 = (dz @ P["W3"]) * (h2 > 0)
    g["W2"] = dh2.T @ h1
    g["b2"] = dh2.sum(0)
    dh1 = (dh2 @ P["W2"]) * (h1 > 0)
    g["W1"] = dh1.T @ x
    g["b1"] = dh1.sum(0)
    return loss, pack(g)


def train(p, x, y, w=None, epochs=100, lr=1e-2):
    """Full-batch Adam; returns (params, loss before each step)."""
    p = np.asarray(p, np.float64).copy()
    m1 = np.zeros_like(p)
    v1 = np.zeros_like(p)
    curve = []
    for t in range(1, epochs + 1):
        loss, g = loss_and_grad(p, x, y, w)
        curve.append(loss)
        m1 = 0.9 * m1 + 0.1 * g
        v1 = 0.999 * v1 + 0.001 * g * g
        p -= lr * (m1 / (1 - 0.9 ** t)) / (np.sqrt(v1 / (1 - 0.999 ** t)) + 1e-8)
    return p, np.array(curve)
