"""TEST INFRASTRUCTURE ONLY: a CPU (numpy FP32) restatement of the surrogate network's forward pass, loss gradient and
backward pass, rounding to BF16 at the points where the library's kernels do (weights, activations, the heads'
gradient and each layer's dZ), so the GPU gradients can be checked layer by layer. The reference (imalsky/maxichem)
has no learned part; this restates the standard MLP algebra the library's kernels implement: z = a W^T + b, a' =
silu(z), dW = dZ^T a, db = sum dZ, dA = dZ W, dZ' = dA * silu'(z). Only tests import it.
"""

from __future__ import annotations

import numpy as np

FLOAT = np.float32  # the arithmetic of the kernels' sums; the CPU pin of this module sets float64


def bf16(a: np.ndarray) -> np.ndarray:
    """Round FP32 values to BF16 (to nearest, ties to even), returned as FP32."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def silu(z: np.ndarray) -> np.ndarray:
    return z / (1.0 + np.exp(-z))


def dsilu(z: np.ndarray) -> np.ndarray:
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def unpack(p: np.ndarray, shapes: list[tuple[int, int]]) -> list[tuple[np.ndarray, np.ndarray]]:
    out, off = [], 0
    for rows, cols in shapes:
        w = p[off : off + rows * cols].reshape(rows, cols)
        off += rows * cols
        out.append((w, p[off : off + rows]))
        off += rows
    return out


def forward(feat: np.ndarray, layers: list[tuple[np.ndarray, np.ndarray]]) -> tuple[np.ndarray, list, list]:
    """pred, the activations a_0 .. a_L (BF16 values) and the pre-activations z_0 .. z_{L-1} (FP32)."""
    a = [bf16(feat)]
    z = []
    for w, b in layers[:-1]:
        zz = a[-1] @ bf16(w).T + b
        z.append(zz.astype(FLOAT))
        a.append(bf16(silu(zz)))
    w, b = layers[-1]
    return (a[-1] @ bf16(w).T + b).astype(FLOAT), a, z


def loss_grad(pred: np.ndarray, tgt: np.ndarray, wts: np.ndarray, heads: int, nt: int,
              delta: float = 0.0) -> tuple[np.ndarray, float]:
    """The heads' gradient (BF16 values, padding columns 0) and the weighted loss: the mean square error (delta 0) or
    the Huber loss of width delta (quadratic within it, linear beyond)."""
    M = pred.shape[0]
    d = np.zeros_like(pred)
    loss = 0.0
    scale = 1.0 / (M * heads * nt)
    for h in range(heads):
        diff = pred[:, h * nt : (h + 1) * nt] - tgt
        w = wts[:, h : h + 1]
        if delta > 0:
            clipped = np.clip(diff, -delta, delta)
            value = np.where(np.abs(diff) > delta, delta * (2.0 * np.abs(diff) - delta), diff * diff)
        else:
            clipped, value = diff, diff * diff
        d[:, h * nt : (h + 1) * nt] = 2.0 * w * clipped * scale
        loss += float((w * value).sum()) * scale
    return bf16(d), loss


def backward(dpred: np.ndarray, layers, a: list, z: list) -> list[tuple[np.ndarray, np.ndarray]]:
    """(dW_l, db_l) for every layer, the library's order of rounding: dZ in BF16, sums in FP32."""
    grads = [None] * len(layers)
    dz = dpred
    for l in range(len(layers) - 1, -1, -1):
        grads[l] = ((dz.T @ a[l]).astype(FLOAT), dz.sum(0).astype(FLOAT))
        if l > 0:
            da = dz @ bf16(layers[l][0])
            dz = bf16(da * dsilu(z[l - 1]))
    return grads
