"""FP64 host oracle of the learned sample-interval proposal (TEST INFRASTRUCTURE ONLY).

The proposal has no reference counterpart: this is the project's own CPU statement of the
network the CUDA kernels implement (clear-plenoxels_b200/csrc/proposal.cu), in float64
numpy, used by the tests as the checker of the tensor-core inference, the FP32 training
gradients and the feature encoding.  Nothing in the product imports it.

Network: 32 segments per ray; per segment 48 inputs (33 used) -> 64 -> 64 -> 64 -> 1 with
ReLU; parameters in one flat block [W1 (64x48), b1, W2 (64x64), b2, W3 (64x64), b3, w4 (64),
b4]; loss: mean binary cross-entropy with logits against label = segment weight > tau.
"""
from __future__ import annotations

import numpy as np

SEG = 32
N_IN = 48
N_FEAT = 33
HID = 64
O_W1 = 0
O_B1 = O_W1 + HID * N_IN
O_W2 = O_B1 + HID
O_B2 = O_W2 + HID * HID
O_W3 = O_B2 + HID
O_B3 = O_W3 + HID * HID
O_W4 = O_B3 + HID
O_B4 = O_W4 + HID
N_PARAMS = O_B4 + 1


def unpack(p):
    p = np.asarray(p, np.float64)
    return (p[O_W1:O_B1].reshape(HID, N_IN), p[O_B1:O_W2], p[O_W2:O_B2].reshape(HID, HID), p[O_B2:O_W3],
            p[O_W3:O_B3].reshape(HID, HID), p[O_B3:O_W4], p[O_W4:O_B4], p[O_B4])


def features(ox, oy, oz, dx, dy, dz, near, far, dims, dtype=np.float64):
    """[n_rays, 32, 48] inputs: midpoint in [-1, 1] box coordinates, sin/cos of pi 2^k x
    (k = 0..3), ray direction, origin in box coordinates / 4; zeros after 33."""
    o = np.stack([ox, oy, oz], 1).astype(dtype)
    d = np.stack([dx, dy, dz], 1).astype(dtype)
    near = np.asarray(near, dtype)
    far = np.asarray(far, dtype)
    n = o.shape[0]
    sc = np.array([2.0 / (dims[0] - 1), 2.0 / (dims[1] - 1), 2.0 / (dims[2] - 1)], dtype)
    s = np.arange(SEG, dtype=dtype)
    t = near[:, None] + (s[None, :] + 0.5) * (far - near)[:, None] / SEG
    p = o[:, None, :] + t[:, :, None] * d[:, None, :]
    x = p * sc - 1.0
    f = np.zeros((n, SEG, N_IN), dtype)
    f[:, :, 0:3] = x
    for k in range(4):
        w = np.pi * (2.0 ** k) * x
        for ax in range(3):
            f[:, :, 3 + 6 * k + 2 * ax] = np.sin(w[:, :, ax])
            f[:, :, 4 + 6 * k + 2 * ax] = np.cos(w[:, :, ax])
    f[:, :, 27:30] = d[:, None, :]
    f[:, :, 30:33] = ((o * sc - 1.0) * 0.25)[:, None, :]
    return f


def forward(params, x, bf16=False):
    """Logits of inputs x [..., 48].  bf16=True rounds the weights and every layer's input to
    bfloat16 as the tensor-core path does (accumulation stays wide)."""
    W1, b1, W2, b2, W3, b3, w4, b4 = unpack(params)
    r = bf16_round if bf16 else (lambda a: a)
    h1 = np.maximum(r(x) @ r(W1).T + b1, 0.0)
    h2 = np.maximum(r(h1) @ r(W2).T + b2, 0.0)
    h3 = np.maximum(r(h2) @ r(W3).T + b3, 0.0)
    return h3 @ w4 + b4


def loss_and_grad(params, x, y):
    """Mean binary cross-entropy with logits over all points and its gradient [N_PARAMS]."""
    W1, b1, W2, b2, W3, b3, w4, b4 = unpack(params)
    x = x.reshape(-1, N_IN)
    y = np.asarray(y, np.float64).reshape(-1)
    z1 = x @ W1.T + b1
    h1 = np.maximum(z1, 0)
    z2 = h1 @ W2.T + b2
    h2 = np.maximum(z2, 0)
    z3 = h2 @ W3.T + b3
    h3 = np.maximum(z3, 0)
    z = h3 @ w4 + b4
    n = x.shape[0]
    loss = np.mean(np.maximum(z, 0) - y * z + np.log1p(np.exp(-np.abs(z))))
    dz = (1.0 / (1.0 + np.exp(-z)) - y) / n
    g = np.zeros(N_PARAMS)
    g[O_W4:O_B4] = h3.T @ dz
    g[O_B4] = dz.sum()
    d3 = np.outer(dz, w4) * (z3 > 0)
    g[O_W3:O_B3] = (d3.T @ h2).reshape(-1)
    g[O_B3:O_W4] = d3.sum(0)
    d2 = (d3 @ W3) * (z2 > 0)
    g[O_W2:O_B2] = (d2.T @ h1).reshape(-1)
    g[O_B2:O_W3] = d2.sum(0)
    d1 = (d2 @ W2) * (z1 > 0)
    g[O_W1:O_B1] = (d1.T @ x).reshape(-1)
    g[O_B1:O_W2] = d1.sum(0)
    return loss, g


def bf16_round(a):
    """Round to bfloat16 (nearest, ties to even) and back, elementwise."""
    f = np.asarray(a, np.float32)
    b = f.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) >> 16
    return (b.astype(np.uint32) << 16).view(np.float32).astype(np.float64)
