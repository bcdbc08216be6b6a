"""Test infrastructure, not product code: the CPU oracle of the learned denoiser's network.

The same U-Net as threert_b200/csrc/unet.cu (layers, padded parameter layout, 2 x 2 average pooling, nearest
upsampling, skip concatenations, ReLU, an L1 loss), its forward and backward passes in float64 numpy, written from the
layer definitions alone. Only tests use it: to check the device's outputs and gradients, and (by finite differences)
to check its own gradients.
"""
from __future__ import annotations

import numpy as np

# (cin padded to 32, cout, relu), in the device's order
LAYERS = [(32, 32, 1), (32, 32, 1), (32, 64, 1), (64, 64, 1), (64, 96, 1), (96, 96, 1), (96, 128, 1), (128, 128, 1),
          (224, 96, 1), (96, 96, 1), (160, 64, 1), (64, 64, 1), (96, 32, 1), (32, 32, 1), (32, 3, 0)]
NAMES = ["e0a", "e0b", "e1a", "e1b", "e2a", "e2b", "e3a", "e3b", "d2a", "d2b", "d1a", "d1b", "d0a", "d0b", "out"]


def r64(v):
    return (v + 63) // 64 * 64


def unpack(params):
    """The flat parameter vector as {name: (W [9, cin, cout], b [cout])} (logical output channels only)."""
    out, o = {}, 0
    for name, (cin, cout, _) in zip(NAMES, LAYERS):
        cp = r64(cout)
        W = params[o:o + 9 * cin * cp].reshape(9, cin, cp)[:, :, :cout]
        o += 9 * cin * cp
        b = params[o:o + cp][:cout]
        o += cp
        out[name] = (np.asarray(W, np.float64), np.asarray(b, np.float64))
    return out


def pack(grads, like):
    """{name: (dW, db)} back into the flat layout (padding zero)."""
    flat = np.zeros_like(like, dtype=np.float64)
    o = 0
    for name, (cin, cout, _) in zip(NAMES, LAYERS):
        cp = r64(cout)
        dW, db = grads[name]
        blk = np.zeros((9, cin, cp))
        blk[:, :, :cout] = dW
        flat[o:o + 9 * cin * cp] = blk.ravel()
        o += 9 * cin * cp
        flat[o:o + cout] = db
        o += cp
    return flat


def _shift(x, dy, dx):
    """x moved so that out[y, x] = x[y + dy, x + dx] (zero outside)."""
    B, H, W, C = x.shape
    out = np.zeros_like(x)
    ys, ye = max(0, -dy), min(H, H - dy)
    xs, xe = max(0, -dx), min(W, W - dx)
    out[:, ys:ye, xs:xe] = x[:, ys + dy:ye + dy, xs + dx:xe + dx]
    return out


def conv(x, W, b):
    y = np.broadcast_to(b, x.shape[:3] + (W.shape[2],)).copy()
    for t in range(9):
        y += _shift(x, t // 3 - 1, t % 3 - 1) @ W[t]
    return y


def conv_back(x, W, dy):
    dW = np.stack([np.einsum("bhwc,bhwn->cn", _shift(x, t // 3 - 1, t % 3 - 1), dy) for t in range(9)])
    db = dy.sum((0, 1, 2))
    dx = np.zeros_like(x)
    for t in range(9):
        dx += _shift(dy @ W[t].T, -(t // 3 - 1), -(t % 3 - 1))
    return dx, dW, db


def pool(x):
    B, H, W, C = x.shape
    return x.reshape(B, H // 2, 2, W // 2, 2, C).mean((2, 4))


def pool_back(dy):
    return np.repeat(np.repeat(dy, 2, 1), 2, 2) * 0.25


def up(x):
    return np.repeat(np.repeat(x, 2, 1), 2, 2)


def up_back(dy):
    B, H, W, C = dy.shape
    return dy.reshape(B, H // 2, 2, W // 2, 2, C).sum((2, 4))


def bf16_round(a):
    """Values rounded to bfloat16 (to nearest, ties to even), as float64."""
    u = np.asarray(a, np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def forward(p, feats, act=None):
    """feats (B, H, W, k <= 32): the prediction (B, H, W, 3) and the activations the backward pass needs. act: None, or
    a rounding applied where the device stores an activation (each hidden layer's output and each pooling's, as bf16:
    bf16_round), so that the device's outputs can be held to the accumulation's rounding alone."""
    B, H, W, k = feats.shape
    x = np.zeros((B, H, W, 32))
    x[..., :k] = feats
    A = {"in": x}
    relu = lambda v: np.maximum(v, 0.0)
    keep = act if act is not None else (lambda v: v)

    def L(name, inp):
        W_, b_ = p[name]
        pre = conv(inp, W_, b_)
        out = keep(relu(pre)) if name != "out" else pre
        A[name] = out
        return out

    pl = lambda v: keep(pool(v))
    e0 = L("e0b", L("e0a", x))
    e1 = L("e1b", L("e1a", pl(e0)))
    e2 = L("e2b", L("e2a", pl(e1)))
    e3 = L("e3b", L("e3a", pl(e2)))
    A["cat2"] = np.concatenate([up(e3), e2], -1)
    u2 = L("d2b", L("d2a", A["cat2"]))
    A["cat1"] = np.concatenate([up(u2), e1], -1)
    u1 = L("d1b", L("d1a", A["cat1"]))
    A["cat0"] = np.concatenate([up(u1), e0], -1)
    u0 = L("d0b", L("d0a", A["cat0"]))
    pred = L("out", u0)
    return pred, A


def loss_and_grads(p, feats, target):
    """The mean L1 loss and its gradient for every layer: {name: (dW, db)}."""
    pred, A = forward(p, feats)
    d = pred - target
    loss = np.abs(d).mean()
    dpred = np.sign(d) / d.size
    G = {}
    inputs = {"e0a": A["in"], "e0b": A["e0a"], "e1a": pool(A["e0b"]), "e1b": A["e1a"], "e2a": pool(A["e1b"]),
              "e2b": A["e2a"], "e3a": pool(A["e2b"]), "e3b": A["e3a"], "d2a": A["cat2"], "d2b": A["d2a"],
              "d1a": A["cat1"], "d1b": A["d1a"], "d0a": A["cat0"], "d0b": A["d0a"], "out": A["d0b"]}

    def back(name, dy_post):
        dy = dy_post if name == "out" else dy_post * (A[name] > 0)
        dx, dW, db = conv_back(inputs[name], p[name][0], dy)
        G[name] = (dW, db)
        return dx

    du0 = back("out", dpred)
    dcat0 = back("d0a", back("d0b", du0))
    du1, de0 = up_back(dcat0[..., :64]), dcat0[..., 64:]
    dcat1 = back("d1a", back("d1b", du1))
    du2, de1 = up_back(dcat1[..., :96]), dcat1[..., 96:]
    dcat2 = back("d2a", back("d2b", du2))
    de3, de2 = up_back(dcat2[..., :128]), dcat2[..., 128:]
    dp2 = back("e3a", back("e3b", de3))
    dp1 = back("e2a", back("e2b", de2 + pool_back(dp2)))
    dp0 = back("e1a", back("e1b", de1 + pool_back(dp1)))
    back("e0a", back("e0b", de0 + pool_back(dp0)))
    return loss, G, pred
