"""CPU oracle of the learned chemistry surrogate's network (test
infrastructure only: the product never imports this file).

Restates, in numpy FP64, the forward pass, the mean-squared-error loss and
the backward pass of the MLP 16(12 used) -> 128 -> 128 -> 128 -> 16(10 used)
with GELU that the CUDA kernels train and evaluate.  The network is new (the
reference's "DNN" mode, src/Euler.cpp:773-780, has no model), so the oracle
is pinned by finite differences of its own loss (tests/test_mlp_oracle.py),
not by reference outputs.

With quantize=True the BF16 roundings of the device pipeline are applied at
the same points (inputs, weights, hidden activations, output-layer and
hidden-layer gradients before their GEMMs) and the activation is evaluated in
packed-BF16 arithmetic as on the device (each operation rounded to BF16;
tanh exact, then rounded); everything else is FP64, so the remaining
difference to the device is its FP32 accumulation order and its hardware
tanh.  With quantize=False everything is FP64 with the exact GELU.
"""
from __future__ import annotations

import numpy as np

N_IN, N_OUT, IN_PAD, H, OUT_PAD = 12, 10, 16, 128, 16
LAYOUT = (("W1", (IN_PAD, H)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (H, H)), ("b3", (H,)),
          ("W4", (H, OUT_PAD)), ("b4", (OUT_PAD,)))
NPARAM = sum(int(np.prod(s)) for _, s in LAYOUT)
C_GELU = np.sqrt(2.0 / np.pi)


def unpack(p):
    out, o = {}, 0
    for name, shape in LAYOUT:
        n = int(np.prod(shape))
        out[name] = np.asarray(p[o:o + n], dtype=np.float64).reshape(shape)
        o += n
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], dtype=np.float64).reshape(-1) for name, _ in LAYOUT])


def bf16(x):
    """Round to BF16 (nearest even) and return as float64."""
    a = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32)
    r = ((a >> 16) & 1) + np.uint32(0x7FFF)
    return ((a + r) & np.uint32(0xFFFF0000)).view(np.float32).astype(np.float64)


def gelu(z):
    return 0.5 * z * (1.0 + np.tanh(C_GELU * (z + 0.044715 * z ** 3)))


C1_BF16 = 0.796875        # BF16 of sqrt(2/pi)
C3_BF16 = 0.03564453125   # BF16 of sqrt(2/pi) * 0.044715


def gelu_bf16(z):
    """The device's packed-BF16 GELU: z/2 + z/2 tanh(z (c + c3 z^2))."""
    zb = bf16(z)
    a = bf16(bf16(zb * zb) * C3_BF16 + C1_BF16)
    t = bf16(np.tanh(bf16(zb * a)))
    hz = bf16(zb * 0.5)
    return bf16(hz * t + hz)


def gelu_grad(z):
    t = np.tanh(C_GELU * (z + 0.044715 * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * C_GELU * (1.0 + 3 * 0.044715 * z * z)


def forward(p, X, quantize=True):
    """Network outputs (B, 16) and the cache for backward."""
    q = bf16 if quantize else (lambda a: np.asarray(a, dtype=np.float64))
    w = unpack(p)
    h = q(X)
    cache = {"h0": h}
    for l in (1, 2, 3):
        z = h @ q(w[f"W{l}"]) + w[f"b{l}"]
        h = gelu_bf16(z) if quantize else gelu(z)
        cache[f"z{l}"], cache[f"h{l}"] = z, h
    out = h @ q(w["W4"]) + w["b4"]
    return out, cache


def loss_grad(p, X, Y, quantize=True):
    """Loss sum_r w_r sum_{k<10} (out - y)^2 / (B 10) (w_r = Y[r, 15]) and its
    gradient with respect to the flat parameter vector."""
    q = bf16 if quantize else (lambda a: np.asarray(a, dtype=np.float64))
    B = X.shape[0]
    w = unpack(p)
    out, c = forward(p, X, quantize)
    wt = np.asarray(Y[:, 15], dtype=np.float64)[:, None]
    d = np.zeros_like(out)
    d[:, :N_OUT] = out[:, :N_OUT] - np.asarray(Y[:, :N_OUT], dtype=np.float64)
    scale = 1.0 / (B * N_OUT)
    loss = float(np.sum(wt * d * d) * scale)
    dz = q(2.0 * wt * d * scale)
    g = {"W4": c["h3"].T @ dz, "b4": dz.sum(axis=0)}
    dh = dz @ q(w["W4"]).T
    for l in (3, 2, 1):
        dz = q(dh * gelu_grad(c[f"z{l}"]))
        g[f"W{l}"] = c[f"h{l - 1}"].T @ dz
        g[f"b{l}"] = dz.sum(axis=0)
        if l > 1:
            dh = dz @ q(w[f"W{l}"]).T
    return loss, pack(g), out
