"""NumPy restatement of the selector MLP — TEST INFRASTRUCTURE ONLY.

Float64 forward and backward of the 20 -> 64 -> 64 -> 7 ReLU network whose
FP16 parameters the library's selector kernels use (parameter layout:
W1[64][20], b1[64], W2[64][64], b2[64], W3[7][64], b3[7]), with the same
masked mean-squared-error loss, mean over rows x outputs.  The selector has
no counterpart in the reference; this is the checker for the device
gradients.
"""
from __future__ import annotations

import numpy as np

F, H, O = 20, 64, 7
SIZES = [("W1", (H, F)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (O, H)), ("b3", (O,))]
TOTAL = sum(int(np.prod(s)) for _, s in SIZES)


def unpack(p: np.ndarray) -> dict:
    out, off = {}, 0
    for name, shape in SIZES:
        n = int(np.prod(shape))
        out[name] = p[off:off + n].astype(np.float64).reshape(shape)
        off += n
    return out


def pack(d: dict) -> np.ndarray:
    return np.concatenate([d[name].reshape(-1) for name, _ in SIZES])


def forward(p: np.ndarray, x: np.ndarray) -> np.ndarray:
    w = unpack(p)
    h1 = np.maximum(x @ w["W1"].T + w["b1"], 0)
    h2 = np.maximum(h1 @ w["W2"].T + w["b2"], 0)
    return h2 @ w["W3"].T + w["b3"]


def forward_backward(p: np.ndarray, x: np.ndarray, t: np.ndarray, mask: np.ndarray):
    """Returns (loss, gradient vector in the packed layout)."""
    w = unpack(p)
    x = x.astype(np.float64)
    z1 = x @ w["W1"].T + w["b1"]
    h1 = np.maximum(z1, 0)
    z2 = h1 @ w["W2"].T + w["b2"]
    h2 = np.maximum(z2, 0)
    y = h2 @ w["W3"].T + w["b3"]
    scale = 1.0 / (x.shape[0] * O)
    e = (y - t) * mask
    loss = float(np.sum(e * e) * scale)
    dy = 2 * e * scale
    g = {"W3": dy.T @ h2, "b3": dy.sum(0)}
    dz2 = (dy @ w["W3"]) * (z2 > 0)
    g["W2"], g["b2"] = dz2.T @ h1, dz2.sum(0)
    dz1 = (dz2 @ w["W2"]) * (z1 > 0)
    g["W1"], g["b1"] = dz1.T @ x, dz1.sum(0)
    return loss, pack(g)


def adam(master, g, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mh, vh = m / (1 - b1 ** step), v / (1 - b2 ** step)
    return master - lr * mh / (np.sqrt(vh) + eps), m, v
