"""float64 reference of the block-demand MLP -- TEST INFRASTRUCTURE ONLY.

16 -> 64 -> 64 -> 1 with ReLU, mean squared error, flat parameter layout
W1[64][16], b1[64], W2[64][64], b2[64], W3[64], b3 (include/gowalker.h,
GW_MLP_PARAMS).  Used by tests/test_gpu_mlp.py to check the device forward
pass, gradients and training against plain backpropagation in double
precision.
"""
import numpy as np

IN, HID = 16, 64
SIZES = [("W1", (HID, IN)), ("b1", (HID,)), ("W2", (HID, HID)), ("b2", (HID,)), ("W3", (HID,)), ("b3", (1,))]
NPARAMS = sum(int(np.prod(s)) for _, s in SIZES)


def unpack(p):
    out, o = {}, 0
    for name, shape in SIZES:
        n = int(np.prod(shape))
        out[name] = np.asarray(p[o:o + n], dtype=np.float64).reshape(shape)
        o += n
    return out


def pack(d):
    return np.concatenate([d[name].reshape(-1) for name, _ in SIZES])


def forward(p, x):
    w = unpack(p)
    x = np.asarray(x, dtype=np.float64)
    a1 = x @ w["W1"].T + w["b1"]
    h1 = np.maximum(a1, 0)
    a2 = h1 @ w["W2"].T + w["b2"]
    h2 = np.maximum(a2, 0)
    y = h2 @ w["W3"] + w["b3"][0]
    return y, (x, a1, h1, a2, h2)


def loss_and_grad(p, x, t):
    """Mean squared error and its gradient (flat, float64)."""
    w = unpack(p)
    y, (x, a1, h1, a2, h2) = forward(p, x)
    n = len(y)
    e = y - np.asarray(t, dtype=np.float64)
    loss = float((e * e).mean())
    dy = 2 * e / n
    g = {"W3": h2.T @ dy, "b3": np.array([dy.sum()])}
    d2 = np.outer(dy, w["W3"]) * (a2 > 0)
    g["W2"] = d2.T @ h1
    g["b2"] = d2.sum(0)
    d1 = (d2 @ w["W2"]) * (a1 > 0)
    g["W1"] = d1.T @ x
    g["b1"] = d1.sum(0)
    return loss, pack(g)
