"""CPU oracle of the radiance-cache MLP — TEST INFRASTRUCTURE ONLY.

FP64 forward, loss and backward of the network in cuda-path-tracer_b200/csrc/pt_mlp.cu, rounding
to BF16 at the points where the GPU stores BF16 (inputs, weights, post-ReLU activations, output
and hidden-layer gradients); the GPU accumulates in FP32 on the tensor cores, this oracle in FP64.
There is no reference counterpart (the reference has no learned component); the encoding and
the loss are the ones pt.h documents.
"""
from __future__ import annotations

import numpy as np

HIDDEN, WIDTH, OUT = 5, 64, 3
MASTER = HIDDEN * WIDTH * WIDTH + WIDTH * OUT

SH = [0.28209479177387814, 0.48860251190291987, 1.0925484305920792, 0.31539156525252005, 0.5462742152960396,
      0.5900435899266435, 2.890611442640554, 0.4570457994644658, 0.3731763325901154, 1.445305721320277]


def bf16(x: np.ndarray) -> np.ndarray:
    """Round to the nearest BF16 (ties to even), returned as float64."""
    f = np.asarray(x, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(master: np.ndarray):
    w = [master[l * 4096:(l + 1) * 4096].reshape(64, 64).astype(np.float64) for l in range(HIDDEN)]
    w.append(master[HIDDEN * 4096:].reshape(64, OUT).astype(np.float64))
    return w


def pack(mats) -> np.ndarray:
    return np.concatenate([m.reshape(-1) for m in mats]).astype(np.float32)


def encode(queries: np.ndarray, lo, hi) -> np.ndarray:
    """queries: structured array with position, direction, normal, albedo (3 each) and roughness."""
    n = len(queries)
    x = np.zeros((n, 64), np.float64)
    pos = queries["position"].astype(np.float32)
    p = (pos - np.float32(lo)) * (np.float32(1.0) / (np.float32(hi) - np.float32(lo)))
    k = 0
    for a in range(3):
        s = np.float32(3.14159265358979) * p[:, a]
        for f in range(6):
            x[:, k] = np.sin(s.astype(np.float64)); x[:, k + 1] = np.cos(s.astype(np.float64))
            k += 2
            s = s * np.float32(2.0)
    d = queries["direction"].astype(np.float64)
    dx, dy, dz = d[:, 0], d[:, 1], d[:, 2]
    xx, yy, zz = dx * dx, dy * dy, dz * dz
    sh = [np.full(n, SH[0]), -SH[1] * dy, SH[1] * dz, -SH[1] * dx, SH[2] * dx * dy, -SH[2] * dy * dz,
          SH[3] * (3 * zz - 1), -SH[2] * dx * dz, SH[4] * (xx - yy), -SH[5] * dy * (3 * xx - yy), SH[6] * dx * dy * dz,
          -SH[7] * dy * (5 * zz - 1), SH[8] * dz * (5 * zz - 3), -SH[7] * dx * (5 * zz - 1), SH[9] * dz * (xx - yy),
          -SH[5] * dx * (xx - 3 * yy)]
    for v in sh:
        x[:, k] = v
        k += 1
    for name in ("normal", "albedo"):
        x[:, k:k + 3] = queries[name]
        k += 3
    x[:, k] = queries["roughness"]
    return x


def forward(master: np.ndarray, x: np.ndarray, keep: bool = False):
    w = [bf16(m) for m in unpack(master)]
    a = bf16(x)
    acts = [a]
    for l in range(HIDDEN):
        a = bf16(np.maximum(a @ w[l], 0.0))
        acts.append(a)
    z = a @ w[HIDDEN]
    y = np.exp(z)
    return (y, acts, w) if keep else y


def loss_and_grad(master: np.ndarray, x: np.ndarray, targets: np.ndarray):
    """Mean relative-L2 loss and its gradient w.r.t. the FP32 masters (flat, PT_CACHE_WEIGHTS)."""
    y, acts, w = forward(master, x, keep=True)
    n = len(x)
    denom = y * y + 0.01
    diff = y - targets
    loss = float((diff * diff / denom).sum() / (n * OUT))
    gz = bf16((1.0 / (n * OUT)) * 2.0 * diff * y / denom)
    grads = [None] * (HIDDEN + 1)
    grads[HIDDEN] = acts[HIDDEN].T @ gz
    dh = gz @ w[HIDDEN].T
    for l in range(HIDDEN - 1, -1, -1):
        dz = bf16(np.where(acts[l + 1] > 0, dh, 0.0))
        grads[l] = acts[l].T @ dz
        if l > 0:
            dh = dz @ w[l].T
    return loss, pack(grads)


def adam(master, m, v, grad, step, lr=1e-2, beta1=0.9, beta2=0.99, eps=1e-8):
    m = beta1 * m + (1 - beta1) * grad
    v = beta2 * v + (1 - beta2) * grad * grad
    mh = m / (1 - beta1 ** step)
    vh = v / (1 - beta2 ** step)
    return master - lr * mh / (np.sqrt(vh) + eps), m, v
