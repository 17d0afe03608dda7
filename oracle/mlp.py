"""numpy restatement of the learned warm-start network -- TEST INFRASTRUCTURE
ONLY (the checker for the tcgen05 forward / backward / Adam kernels of
sap_warp_b200/csrc/sapb_mlp.cu; see oracle/__init__.py).

The network has no counterpart in the reference (its warm start is the
previous step's velocity, sim/solver_sap.py:1441-1451).  `forward` and
`backward` mirror the kernels' rounding points exactly: BF16 weights, BF16
inputs, BF16 hidden activations h = bf16(gelu(z)), BF16 dy for the W4
gradient, BF16 dz = bf16(dh * gelu'(z)) as the operand of the weight and
input gradients; sums are accumulated in float64 here (FP32 on the GPU).
With ``mirror=False`` nothing is rounded except the weights, which is the
network that float64 autograd differentiates.
"""

from __future__ import annotations

import numpy as np

IN, IN_PAD, HID, OUT = 12, 16, 128, 3
_SIZES = [("W1", (HID, IN)), ("b1", (HID,)), ("W2", (HID, HID)), ("b2", (HID,)), ("W3", (HID, HID)),
          ("b3", (HID,)), ("W4", (OUT, HID)), ("b4", (OUT,))]
PARAM_COUNT = sum(int(np.prod(s)) for _, s in _SIZES)

GELU_C = np.sqrt(2.0 / np.pi)
GELU_A = 0.044715


def offsets() -> dict:
    out, o = {}, 0
    for name, shape in _SIZES:
        size = int(np.prod(shape))
        out[name] = (o, shape)
        o += size
    return out


def unpack(params: np.ndarray) -> dict:
    p = np.asarray(params, dtype=np.float32)
    return {k: p[o:o + int(np.prod(s))].reshape(s) for k, (o, s) in offsets().items()}


def pack(parts: dict) -> np.ndarray:
    out = np.zeros(PARAM_COUNT, dtype=np.float32)
    for k, (o, s) in offsets().items():
        out[o:o + int(np.prod(s))] = np.asarray(parts[k], dtype=np.float32).reshape(-1)
    return out


def init_params(seed: int = 0) -> np.ndarray:
    """U(-1/sqrt(fan_in), 1/sqrt(fan_in)) weights and biases; the output layer
    scaled by 0.1 so the untrained network predicts near the target mean."""
    rng = np.random.default_rng(seed)
    parts = {}
    for k, (o, s) in offsets().items():
        fan_in = IN if k in ("W1", "b1") else HID
        bound = 1.0 / np.sqrt(fan_in)
        parts[k] = rng.uniform(-bound, bound, size=s).astype(np.float32)
    parts["W4"] *= 0.1
    parts["b4"] *= 0.1
    return pack(parts)


def bf16(x) -> np.ndarray:
    """Round float32 to the nearest bfloat16 (ties to even), as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).reshape(a.shape)


def bf16_bits(x) -> np.ndarray:
    return (bf16(x).view(np.uint32) >> 16).astype(np.uint16)


def from_bf16_bits(b) -> np.ndarray:
    return (np.asarray(b, dtype=np.uint32) << 16).view(np.float32)


def gelu(z):
    t = np.tanh(GELU_C * (z + GELU_A * z ** 3))
    return 0.5 * z * (1.0 + t)


def gelu_grad(z):
    t = np.tanh(GELU_C * (z + GELU_A * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * GELU_C * (1.0 + 3.0 * GELU_A * z * z)


def _r(x, mirror):
    return bf16(x).astype(np.float64) if mirror else np.asarray(x, dtype=np.float64)


def forward(params: np.ndarray, x: np.ndarray, mirror: bool = True) -> dict:
    """x: (M, 12 or 16) inputs (rounded to BF16 when mirroring)."""
    p = unpack(params)
    W = {k: bf16(p[k]).astype(np.float64) for k in ("W1", "W2", "W3", "W4")}
    b = {k: p[k].astype(np.float64) for k in ("b1", "b2", "b3", "b4")}
    x = _r(np.asarray(x, dtype=np.float32)[:, :IN], mirror)
    z1 = x @ W["W1"].T + b["b1"]
    h1 = _r(gelu(z1), mirror)
    z2 = h1 @ W["W2"].T + b["b2"]
    h2 = _r(gelu(z2), mirror)
    z3 = h2 @ W["W3"].T + b["b3"]
    h3 = _r(gelu(z3), mirror)
    y = h3 @ W["W4"].T + b["b4"]
    return dict(x=x, z1=z1, h1=h1, z2=z2, h2=h2, z3=z3, h3=h3, y=y, W=W)


def backward(params: np.ndarray, x: np.ndarray, target: np.ndarray, mirror: bool = True):
    """(loss = sum of squared errors, gradient of the mean squared error in
    the master layout, forward cache)."""
    f = forward(params, x, mirror)
    W = f["W"]
    M = f["y"].shape[0]
    d = f["y"] - np.asarray(target, dtype=np.float64)
    loss = float((d * d).sum())
    dy = d * (2.0 / (3.0 * M))
    g = {}
    g["W4"] = _r(dy, mirror).T @ f["h3"]
    g["b4"] = dy.sum(0)
    dz3 = _r((dy @ W["W4"]) * gelu_grad(f["z3"]), mirror)
    g["W3"] = dz3.T @ f["h2"]
    g["b3"] = dz3.sum(0)
    dz2 = _r((dz3 @ W["W3"]) * gelu_grad(f["z2"]), mirror)
    g["W2"] = dz2.T @ f["h1"]
    g["b2"] = dz2.sum(0)
    dz1 = _r((dz2 @ W["W2"]) * gelu_grad(f["z1"]), mirror)
    g["W1"] = dz1.T @ f["x"]
    g["b1"] = dz1.sum(0)
    return loss, pack(g), f


def adam(params, grad, m, v, step, lr, beta1=0.9, beta2=0.999, eps=1e-8, weight_decay=0.0):
    """One Adam step with decoupled weight decay, float32 like the kernel."""
    p = np.asarray(params, np.float32).copy()
    g = np.asarray(grad, np.float32)
    m = (np.float32(beta1) * m + np.float32(1 - beta1) * g).astype(np.float32)
    v = (np.float32(beta2) * v + np.float32(1 - beta2) * g * g).astype(np.float32)
    c1 = np.float32(1.0 / (1.0 - beta1 ** step))
    c2 = np.float32(1.0 / (1.0 - beta2 ** step))
    p = p - np.float32(lr) * (m * c1 / (np.sqrt(v * c2) + np.float32(eps)) + np.float32(weight_decay) * p)
    return p.astype(np.float32), m, v
