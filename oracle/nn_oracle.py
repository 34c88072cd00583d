"""CPU FP64 restatement of the learned face-flux correction network and its
loss gradient -- test infrastructure only: the GPU tests compare the tensor-core
kernels (dev_field_efvm_b200/csrc/efvm_nn.cu) with it.

It rounds to BF16 exactly where the GPU kernels hand BF16 operands to the
tensor cores (the stencil features, the weights, the hidden activations, the
output gradient and the hidden-layer gradients) and does everything else in
float64, so the remaining differences are the GPU's FP32 accumulation order.
The network has no counterpart in the reference; this file follows the kernels'
definition of it.
"""
from __future__ import annotations

import numpy as np

IN, K1, H, NOUT = 100, 112, 32, 4
P_W1 = 0
P_W2 = P_W1 + H * K1
P_W3 = P_W2 + H * H
P_B1 = P_W3 + NOUT * H
P_B2 = P_B1 + H
P_B3 = P_B2 + H
P_COUNT = P_B3 + NOUT


def bf16(x) -> np.ndarray:
    """Round float32 values to bfloat16 (round to nearest even), returned as float64."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    b = a.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) >> 16 << 16
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p: np.ndarray):
    w1 = p[P_W1:P_W2].reshape(H, K1).copy()
    w1[:, IN:] = 0.0
    return (w1, p[P_W2:P_W3].reshape(H, H), p[P_W3:P_B1].reshape(NOUT, H), p[P_B1:P_B2], p[P_B2:P_B3],
            p[P_B3:P_COUNT])


def features(states: np.ndarray, gamma: float = 1.4) -> np.ndarray:
    """[batch, 2, ny, nx, K1] stencil features (BF16-rounded) of every face:
    orientation 0 = the x face on the left of a cell, 1 = the y face below it."""
    B, _, ny, nx = states.shape
    r, mx, my, E = (states[:, v] for v in range(4))
    u, v = mx / r, my / r
    p = (gamma - 1.0) * (E - 0.5 * r * (u * u + v * v))
    w = [np.float32(r), np.float32(u), np.float32(v), np.float32(p)]
    X = np.zeros((B, 2, ny, nx, K1))
    for orient in range(2):
        for c in range(-2, 3):
            for a in range(-3, 2):
                # value at cell (i + a, j + c) for x faces, (i + c, j + a) for y faces
                sx, sy = (a, c) if orient == 0 else (c, a)
                sh = [np.roll(q, shift=(-sy, -sx), axis=(1, 2)) for q in w]
                un, ut = (sh[1], sh[2]) if orient == 0 else (sh[2], sh[1])
                f = [sh[0] - np.float32(1.0), un, ut, sh[3] - np.float32(1.0)]
                k0 = ((c + 2) * 5 + (a + 3)) * 4
                for q in range(4):
                    X[:, orient, :, :, k0 + q] = bf16(f[q])
    return X


def forward(p: np.ndarray, states: np.ndarray, out_scale: float, gamma: float = 1.4):
    """Corrections [batch, 2, 4, ny, nx] (grid frame) and the activations."""
    w1, w2, w3, b1, b2, b3 = unpack(p)
    W1, W2, W3 = bf16(w1), bf16(w2), bf16(w3)
    X = features(states, gamma)
    h1 = bf16(np.maximum(X @ W1.T + b1, 0.0))
    h2 = bf16(np.maximum(h1 @ W2.T + b2, 0.0))
    y = (h2 @ W3.T + b3) * out_scale  # [B, 2, ny, nx, 4] face frame
    g = y.copy()
    g[:, 1, ..., 1], g[:, 1, ..., 2] = y[:, 1, ..., 2], y[:, 1, ..., 1]
    corr = np.moveaxis(g, -1, 2).astype(np.float32).astype(np.float64)
    return corr, (X, h1, h2, W1, W2, W3)


def loss_grad(p, states, resid, dx, dy, w, out_scale, gamma=1.4):
    """Loss sum_v w_v mean(e_v^2) with e = resid + div(corr), and its gradient."""
    corr, (X, h1, h2, W1, W2, W3) = forward(p, states, out_scale, gamma)
    B, _, _, ny, nx = corr.shape
    cx, cy = corr[:, 0], corr[:, 1]  # [B, 4, ny, nx]
    div = (np.roll(cx, -1, axis=3) - cx) / dx + (np.roll(cy, -1, axis=2) - cy) / dy
    e = resid + div
    wv = np.asarray(w, dtype=np.float64)[None, :, None, None]
    total = B * nx * ny
    loss = float(np.sum(wv * e * e) / total)
    s = 2.0 / total
    gx = (s * wv * (np.roll(e, 1, axis=3) - e) / dx).astype(np.float32).astype(np.float64)
    gy = (s * wv * (np.roll(e, 1, axis=2) - e) / dy).astype(np.float32).astype(np.float64)
    dcorr = np.stack([gx, gy], axis=1)  # [B, 2, 4, ny, nx] grid frame
    g = np.moveaxis(dcorr, 2, -1).copy()  # [B, 2, ny, nx, 4]
    g[:, 1, ..., 1], g[:, 1, ..., 2] = dcorr[:, 1, 2], dcorr[:, 1, 1]
    dyv = bf16((g * np.float32(out_scale)).astype(np.float32))
    Xf, h1f, h2f, dyf = (a.reshape(-1, a.shape[-1]) for a in (X, h1, h2, dyv))
    dW3 = dyf.T @ h2f
    db3 = dyf.sum(axis=0)
    dz2 = bf16(np.where(h2f > 0, dyf @ W3, 0.0).astype(np.float32))
    dW2 = dz2.T @ h1f
    db2 = dz2.sum(axis=0)
    dz1 = bf16(np.where(h1f > 0, dz2 @ W2, 0.0).astype(np.float32))
    dW1 = dz1.T @ Xf
    db1 = dz1.sum(axis=0)
    grad = np.zeros(P_COUNT)
    grad[P_W1:P_W2] = dW1.reshape(-1)
    grad[P_W2:P_W3] = dW2.reshape(-1)
    grad[P_W3:P_B1] = dW3.reshape(-1)
    grad[P_B1:P_B2] = db1
    grad[P_B2:P_B3] = db2
    grad[P_B3:P_COUNT] = db3
    return loss, grad, corr
