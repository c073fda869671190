"""numpy reference of the radiance-cache network (test infrastructure).

`forward_backward` emulates the GPU kernels' arithmetic: weights, inputs,
hidden activations and back-propagated gradients are rounded to bf16 at the
points the kernels round them, and everything else is FP32/FP64.
"""
import numpy as np

LAYERS = [(64, 208), (64, 64), (64, 64), (64, 64), (64, 64), (16, 64)]
EPS = 0.01


def bf16(x):
    """Round float32 to bf16 (round to nearest even) and back."""
    x = np.asarray(x, np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def split(p):
    out, off = [], 0
    for o, i in LAYERS:
        out.append(p[off: off + o * i].reshape(o, i).astype(np.float32))
        off += o * i
    return out


def encode(raw, bound):
    raw = np.asarray(raw, np.float32)
    b = np.asarray(bound, np.float32)
    s = (np.float32(1) / np.maximum(b[3:] - b[:3], np.float32(1e-12))).astype(np.float32)
    q = ((raw[:, :3] - b[:3]) * s).astype(np.float32)
    cols = []
    for a in range(3):
        f = q[:, a].astype(np.float64)
        for k in range(12):
            cols.append(np.sin(np.pi * f * 2 ** k))
            cols.append(np.cos(np.pi * f * 2 ** k))
    for v in range(2):
        w = raw[:, 3 + 3 * v: 6 + 3 * v].astype(np.float64)
        th = np.arccos(np.clip(w[:, 2], -1, 1)) / np.pi
        ph = np.arctan2(w[:, 1], w[:, 0]) / (2 * np.pi) + 0.5
        for u in (th, ph):
            for j in range(32):
                d = (u - (j + 0.5) / 32) * 32
                cols.append(np.exp(-0.5 * d * d))
    cols += [raw[:, 9], raw[:, 10], raw[:, 11]] + [np.zeros(len(raw))] * 5
    return bf16(np.stack(cols, 1).astype(np.float32))


def forward_backward(enc, params, targets):
    """Returns (pred, loss, grads[list per layer]) with the GPU's bf16 rounding points."""
    W = [bf16(w) for w in split(params)]
    n = enc.shape[0]
    h = [enc.astype(np.float32)]
    x = enc.astype(np.float64)
    for l in range(5):
        x = np.maximum(x @ W[l].T.astype(np.float64), 0.0)
        x = bf16(x.astype(np.float32)).astype(np.float64)
        h.append(x.astype(np.float32))
    out = (x @ W[5].T.astype(np.float64)).astype(np.float32)
    pred = out[:, :3]
    y = np.asarray(targets, np.float32)
    den = pred.astype(np.float64) ** 2 + EPS
    e = pred.astype(np.float64) - y
    loss = float(np.sum(e * e / den) / (3 * n))
    d5 = np.zeros((n, 16), np.float32)
    d5[:, :3] = (2 * e / den / (3 * n)).astype(np.float32)
    d = bf16(d5).astype(np.float64)
    grads = [None] * 6
    grads[5] = (d.T @ h[5].astype(np.float64)).astype(np.float32)
    for l in range(4, -1, -1):
        da = d @ W[l + 1].astype(np.float64)
        da = da * (h[l + 1] > 0)
        d = bf16(da.astype(np.float32)).astype(np.float64)
        grads[l] = (d.T @ h[l].astype(np.float64)).astype(np.float32)
    return pred, loss, grads
