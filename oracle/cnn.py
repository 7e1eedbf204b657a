"""FP64 numpy oracle of the committor surrogate network.  TEST
INFRASTRUCTURE ONLY: tests compare the CUDA forward pass, loss and gradients
against it.

Network (no reference counterpart; specified for the surrogate): spins (+-1)
-> 4 circularly padded 3x3 convolutions with 32 channels (1->32, 32->32 x3),
each followed by ReLU -> global average pool -> 32->1 linear -> sigmoid.
Loss: binomial cross-entropy against a committor label y in [0, 1], mean
over the batch.

Flat parameter order (float32 on the device, float64 here):
  W1[32][9] b1[32] W2[32][9][32] b2[32] W3[...] b3 W4[...] b4 Wf[32] bf[1]
with tap = (dy+1)*3 + (dx+1) for dy, dx in {-1, 0, 1} (row offset dy,
column offset dx) and W[co][tap][ci].
"""
from __future__ import annotations

import numpy as np

C = 32
TAPS = [(dy, dx) for dy in (-1, 0, 1) for dx in (-1, 0, 1)]
SHAPES = [("W1", (C, 9, 1)), ("b1", (C,)), ("W2", (C, 9, C)), ("b2", (C,)),
          ("W3", (C, 9, C)), ("b3", (C,)), ("W4", (C, 9, C)), ("b4", (C,)),
          ("Wf", (C,)), ("bf", (1,))]
NPARAM = sum(int(np.prod(s)) for _, s in SHAPES)


def unflatten(flat):
    flat = np.asarray(flat, np.float64)
    out, o = {}, 0
    for name, shp in SHAPES:
        n = int(np.prod(shp))
        out[name] = flat[o:o + n].reshape(shp)
        o += n
    return out


def flatten(d):
    return np.concatenate([np.asarray(d[name], np.float64).reshape(-1) for name, _ in SHAPES])


def init_params(seed=0):
    """He-normal convolution weights, small head, zero biases (float32)."""
    rs = np.random.default_rng(seed)
    d = {}
    for name, shp in SHAPES:
        if name.startswith("W") and name != "Wf":
            fan_in = shp[1] * shp[2]
            d[name] = rs.normal(0.0, np.sqrt(2.0 / fan_in), shp)
        elif name == "Wf":
            d[name] = rs.normal(0.0, 0.1, shp)
        else:
            d[name] = np.zeros(shp)
    return flatten(d).astype(np.float32)


def _shift(x, dy, dx):
    """out[:, y, x] = x[:, (y+dy) % L, (x+dx) % L]."""
    return np.roll(x, shift=(-dy, -dx), axis=(1, 2))


def conv(x, W, b):
    out = np.zeros(x.shape[:3] + (W.shape[0],))
    for t, (dy, dx) in enumerate(TAPS):
        out += _shift(x, dy, dx) @ W[:, t, :].T
    return out + b


def _bf16_weights(p):
    q = dict(p)
    for layer in range(1, 5):
        q[f"W{layer}"] = bf16_round(p[f"W{layer}"])
    return q


def forward(params, spins, bf16=False):
    """bf16=True mirrors the device's rounding points: convolution weights and
    stored activations in bfloat16, accumulation and the head in float."""
    p = unflatten(params)
    if bf16:
        p = _bf16_weights(p)
    rnd = bf16_round if bf16 else (lambda v: v)
    a = [np.asarray(spins, np.float64)[..., None]]
    z = []
    for layer in range(1, 5):
        zz = conv(a[-1], p[f"W{layer}"], p[f"b{layer}"])
        z.append(zz)
        a.append(rnd(np.maximum(zz, 0.0)))
    pooled = a[-1].mean(axis=(1, 2))
    zf = pooled @ p["Wf"] + p["bf"][0]
    q = 1.0 / (1.0 + np.exp(-zf))
    return {"a": a, "z": z, "pooled": pooled, "zf": zf, "q": q}


def loss_and_grads(params, spins, labels, bf16=False):
    """bf16=True also rounds each layer's data gradient dZ to bfloat16 (the
    device stores them so) and masks ReLU by the stored activation."""
    p = unflatten(params)
    f = forward(params, spins, bf16=bf16)
    if bf16:
        p = _bf16_weights(p)
    rnd = bf16_round if bf16 else (lambda v: v)
    y = np.asarray(labels, np.float64)
    q = np.clip(f["q"], 1e-12, 1 - 1e-12)
    B = y.size
    loss = float(np.mean(-(y * np.log(q) + (1 - y) * np.log(1 - q))))
    g = {}
    dzf = (f["q"] - y) / B
    g["Wf"] = f["pooled"].T @ dzf
    g["bf"] = np.array([dzf.sum()])
    Npix = f["a"][-1].shape[1] * f["a"][-1].shape[2]
    da = np.broadcast_to((dzf[:, None] * p["Wf"][None, :])[:, None, None, :] / Npix,
                         f["a"][-1].shape).copy()
    for layer in range(4, 0, -1):
        mask = (f["a"][layer] > 0) if bf16 else (f["z"][layer - 1] > 0)
        dz = rnd(da * mask)
        x = f["a"][layer - 1]
        W = p[f"W{layer}"]
        gW = np.zeros_like(W)
        dx = np.zeros_like(x)
        for t, (dy, dxo) in enumerate(TAPS):
            xs = _shift(x, dy, dxo)
            gW[:, t, :] = np.tensordot(dz, xs, axes=([0, 1, 2], [0, 1, 2]))
            dx += _shift(dz, -dy, -dxo) @ W[:, t, :]
        g[f"W{layer}"] = gW
        g[f"b{layer}"] = dz.sum(axis=(0, 1, 2))
        da = dx
    return loss, flatten(g), f["q"]


def bf16_round(x):
    """Round-to-nearest-even to bfloat16, returned as float64."""
    a = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    rounded = ((a + 0x7FFF + ((a >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return rounded.view(np.float32).astype(np.float64)
