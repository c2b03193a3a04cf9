"""Test infrastructure only: the CPU oracle of the learned proposal's network.

The learned proposal has no counterpart in the reference (it is the new part of the
hot path), so this numpy model is the checker of the device kernels in
pyopenlpt_b200/csrc/mlp.cu and gemm.cu: the same layer sequence, the same bf16
rounding points (inputs, hidden weights and activations, and the backward
dZ operands of the weight gradients), f32 accumulation, and the same loss.
``fd_check`` pins the analytic gradients of the model itself against central finite
differences (with bf16 rounding switched off).

Parameter layout (flat f32): W1[256][n_in], b1[256], W2[256][256], b2, W3[256][256],
b3, W4[4][256], b4[4], with n_in = 121 C + 2 C + 1 for C cameras (493 for 4; the
functions take n_in from the flat size).  Nothing in the product imports this module.
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf

IN, HID, OUT = 493, 256, 4


def n_in(n_cam: int) -> int:
    return 121 * n_cam + 2 * n_cam + 1


def shapes(n_in_: int = IN):
    return [("W1", (HID, n_in_)), ("b1", (HID,)), ("W2", (HID, HID)), ("b2", (HID,)),
            ("W3", (HID, HID)), ("b3", (HID,)), ("W4", (OUT, HID)), ("b4", (OUT,))]


SHAPES = shapes(IN)
N_PARAMS = sum(int(np.prod(s)) for _, s in SHAPES)
_REST = N_PARAMS - HID * IN


def shapes_of(flat) -> list:
    """The layer shapes of a flat parameter array (its first layer's width from its size)."""
    return shapes((len(flat) - _REST) // HID)


def unpack(flat: np.ndarray) -> dict:
    out, off = {}, 0
    for name, shp in shapes_of(flat):
        k = int(np.prod(shp))
        out[name] = flat[off:off + k].reshape(shp).astype(np.float32)
        off += k
    return out


def pack(p: dict) -> np.ndarray:
    return np.concatenate([p[name].ravel() for name, _ in shapes(p["W1"].shape[1])]).astype(
        np.float32)


def bf16(a: np.ndarray) -> np.ndarray:
    """Round f32 to the nearest bf16 (ties to even), returned as f32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32)
    return np.where(np.isnan(a), a, out)


def bf16_bits(a: np.ndarray) -> np.ndarray:
    return (bf16(a).view(np.uint32) >> 16).astype(np.uint16)


def gelu(x):
    return 0.5 * x * (1.0 + erf(x / np.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + erf(x / np.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / np.sqrt(2.0 * np.pi)


def forward(flat: np.ndarray, x: np.ndarray, rounding: bool = True):
    """Network outputs (n x 4) and the intermediates the backward pass needs.  With
    rounding: f32 with the device's bf16 rounding points; without: float64."""
    dt = np.float32 if rounding else np.float64
    r = bf16 if rounding else (lambda a: np.asarray(a, dt))
    p = {k: v.astype(dt) for k, v in unpack(np.asarray(flat, np.float64)).items()}
    if not rounding:  # unpack rounds to f32; take the float64 values
        off = 0
        for name, shp in shapes_of(flat):
            k = int(np.prod(shp))
            p[name] = np.asarray(flat[off:off + k], np.float64).reshape(shp)
            off += k
    xb = r(x.astype(dt))
    W1, W2, W3 = r(p["W1"]), r(p["W2"]), r(p["W3"])
    z1 = (xb @ W1.T + p["b1"]).astype(dt)
    h1 = r(gelu(z1))
    z2 = (h1 @ W2.T + p["b2"]).astype(dt)
    h2 = r(gelu(z2))
    z3 = (h2 @ W3.T + p["b3"]).astype(dt)
    h3 = r(gelu(z3))
    o = (h3 @ p["W4"].T + p["b4"]).astype(dt)
    return o, dict(xb=xb, W1=W1, W2=W2, W3=W3, z1=z1, h1=h1, z2=z2, h2=h2, z3=z3, h3=h3, p=p)


def loss_and_dout(o: np.ndarray, t: np.ndarray, ghost_weight: float):
    n = len(o)
    y = t[:, 3]
    pos = 1.0 - y
    e = o[:, :3] - t[:, :3]
    z = o[:, 3].astype(np.float64)
    bce = np.maximum(z, 0) - z * y + np.log1p(np.exp(-np.abs(z)))
    loss = float(np.mean(pos * np.sum(e * e, axis=1) / 3.0 + ghost_weight * bce))
    dout = np.empty_like(o)
    dout[:, :3] = pos[:, None] * (2.0 / 3.0) * e / n
    dout[:, 3] = ghost_weight * (1.0 / (1.0 + np.exp(-z)) - y) / n
    return loss, dout


def backward(flat: np.ndarray, x: np.ndarray, t: np.ndarray, ghost_weight: float = 1.0,
             rounding: bool = True):
    """Mean loss and the flat gradient."""
    r = bf16 if rounding else (lambda a: np.asarray(a, np.float64))
    o, c = forward(flat, x, rounding)
    loss, do = loss_and_dout(o, t, ghost_weight)
    p = c["p"]
    g = {}
    g["W4"] = do.T @ c["h3"]
    g["b4"] = do.sum(0)
    dz3 = (do @ p["W4"]) * gelu_grad(c["z3"])
    g["W3"] = r(dz3).T @ c["h2"]
    g["b3"] = dz3.sum(0)
    dz2 = (r(dz3) @ c["W3"]) * gelu_grad(c["z2"])
    g["W2"] = r(dz2).T @ c["h1"]
    g["b2"] = dz2.sum(0)
    dz1 = (r(dz2) @ c["W2"]) * gelu_grad(c["z1"])
    g["W1"] = r(dz1).T @ c["xb"]
    g["b1"] = dz1.sum(0)
    return loss, np.concatenate([g[name].ravel() for name, _ in shapes_of(flat)])


def adam(flat, grad, m, v, t, lr, b1=0.9, b2=0.999, eps=1e-8):
    m = b1 * m + (1 - b1) * grad
    v = b2 * v + (1 - b2) * grad * grad
    flat = flat - lr * (m / (1 - b1 ** t)) / (np.sqrt(v / (1 - b2 ** t)) + eps)
    return flat.astype(np.float32), m, v


def init(seed: int = 0, n_in_: int = IN) -> np.ndarray:
    rng = np.random.default_rng(seed)
    p = {}
    for name, shp in shapes(n_in_):
        if name.startswith("b"):
            p[name] = np.zeros(shp, np.float32)
        else:
            fan_in = shp[1]
            lim = np.sqrt((1.0 if name == "W4" else 6.0) / fan_in)
            p[name] = rng.uniform(-lim, lim, shp).astype(np.float32)
    return pack(p)


def fd_check(seed: int = 0, n: int = 8, n_probe: int = 40, h: float = 1e-2):
    """Largest relative error of the analytic gradient against central differences
    (float64 evaluation of the f32 model, no bf16 rounding) over random coordinates."""
    rng = np.random.default_rng(seed)
    flat = init(seed).astype(np.float64)
    x = rng.normal(0, 1, (n, IN))
    t = np.concatenate([rng.normal(0, 1, (n, 3)), (rng.random((n, 1)) < 0.3)], axis=1)

    def f(fl):
        o, _ = forward(fl, x, rounding=False)
        return loss_and_dout(o, t, 1.0)[0]

    _, g = backward(flat, x, t, 1.0, rounding=False)
    worst = 0.0
    for i in rng.choice(N_PARAMS, n_probe, replace=False):
        e = np.zeros_like(flat)
        e[i] = h
        num = (f(flat + e) - f(flat - e)) / (2 * h)
        den = max(abs(num), abs(g[i]), 1e-6)
        worst = max(worst, abs(num - g[i]) / den)
    return worst
