"""CPU oracle of the learned warm start (numpy, FP64).

TEST INFRASTRUCTURE ONLY: ``tests/`` use it to check the device kernels of
the warm-start network (forward activations, loss, gradients); the product
path never imports it.

The network has no counterpart in the reference (it is the learned part of
the B200 path): a 3-layer 3x3 convolutional network on the reconstruction
grid,

    h1 = relu(conv(x, W1) + b1)      x:  [H, W, 2]  input features
    h2 = relu(conv(h1, W2) + b2)     h:  [H, W, C]
    out = conv(h2, W3) + b3          out: [H, W, 1] predicted log prior

with zero padding 1, weights W[l] of shape [3, 3, Cin, Cout] (tap dy, tap
dx, input channel, output channel) and the loss mean((out - target)^2).
Features (``features``): f0 = log(|A^H y|^2 / mean|A^H y|^2 + 1e-3) and
f1 = mean of f0 over the grid (a sparsity / SNR summary), constant over the
grid.
The device keeps activations and the weights it multiplies in BF16 and
accumulates in FP32; this oracle runs FP64 on the same (BF16-rounded)
weights when asked, so the comparison isolates accumulation error.
"""

from __future__ import annotations

import numpy as np


def bf16_round(a: np.ndarray) -> np.ndarray:
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    f = np.asarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    r = ((u + 0x7FFF + lsb) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def features(bp: np.ndarray, grid) -> np.ndarray:
    """bp: complex [B, N] backprojection A^H y -> [B, H, W, 2] float64."""
    b = bp.shape[0]
    e = np.abs(bp.astype(np.complex128)) ** 2
    mean = np.maximum(e.mean(axis=1, keepdims=True), 1e-30)
    f0 = np.log(e / mean + 1e-3)
    f1 = np.broadcast_to(f0.mean(axis=1, keepdims=True), e.shape)
    return np.stack([f0, f1], axis=-1).reshape(b, grid[0], grid[1], 2)


def conv3x3(x: np.ndarray, w: np.ndarray, b: np.ndarray) -> np.ndarray:
    """x [B, H, W, Ci], w [3, 3, Ci, Co], b [Co] -> [B, H, W, Co], zero padding 1."""
    bsz, h, wd, _ = x.shape
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (0, 0)))
    out = np.zeros((bsz, h, wd, w.shape[3]))
    for dy in range(3):
        for dx in range(3):
            out += xp[:, dy:dy + h, dx:dx + wd, :] @ w[dy, dx]
    return out + b


def conv3x3_backward(x, w, dout):
    """Gradients of conv3x3 w.r.t. x, w and b for upstream gradient dout."""
    bsz, h, wd, _ = x.shape
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (0, 0)))
    dxp = np.zeros_like(xp)
    dw = np.zeros_like(w)
    for dy in range(3):
        for dx in range(3):
            patch = xp[:, dy:dy + h, dx:dx + wd, :]
            dw[dy, dx] = np.einsum("bhwi,bhwo->io", patch, dout)
            dxp[:, dy:dy + h, dx:dx + wd, :] += dout @ w[dy, dx].T
    db = dout.sum(axis=(0, 1, 2))
    return dxp[:, 1:-1, 1:-1, :], dw, db


def forward(params, x):
    """params: dict W1,b1,W2,b2,W3,b3.  Returns (out [B,H,W], cache)."""
    a1 = conv3x3(x, params["W1"], params["b1"])
    h1 = np.maximum(a1, 0.0)
    a2 = conv3x3(h1, params["W2"], params["b2"])
    h2 = np.maximum(a2, 0.0)
    out = conv3x3(h2, params["W3"], params["b3"])[..., 0]
    return out, (x, a1, h1, a2, h2)


def loss_and_grads(params, x, target, mask=None):
    """Mean squared error over the (masked) pixels and its gradients."""
    out, (x, a1, h1, a2, h2) = forward(params, x)
    wgt = np.ones_like(out) if mask is None else mask.astype(np.float64)
    count = max(wgt.sum(), 1.0)
    diff = (out - target) * wgt
    loss = float((diff * (out - target)).sum() / count)
    dout = (2.0 * diff / count)[..., None]
    dh2, dW3, db3 = conv3x3_backward(h2, params["W3"], dout)
    da2 = dh2 * (a2 > 0)
    dh1, dW2, db2 = conv3x3_backward(h1, params["W2"], da2)
    da1 = dh1 * (a1 > 0)
    _, dW1, db1 = conv3x3_backward(x, params["W1"], da1)
    return loss, out, {"W1": dW1, "b1": db1, "W2": dW2, "b2": db2, "W3": dW3, "b3": db3}


def init_params(hidden: int = 8, seed: int = 0):
    """He-style initial weights (FP64)."""
    rng = np.random.default_rng(seed)
    def w(ci, co):
        return rng.normal(0.0, np.sqrt(2.0 / (9 * ci)), (3, 3, ci, co))
    return {"W1": w(2, hidden), "b1": np.zeros(hidden), "W2": w(hidden, hidden),
            "b2": np.zeros(hidden), "W3": w(hidden, 1) * 0.1, "b3": np.zeros(1)}
