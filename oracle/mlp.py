"""FP64 restatement of the surrogate MLP's forward and backward (test oracle).

Test infrastructure: only tests/ use this module, as the checker.  It mirrors
the rounding points of the GPU kernels: weights and layer inputs are BF16,
products accumulate exactly (FP64 here, FP32 in tensor memory), hidden
activations are rounded to BF16 after SiLU, and the output gradient is rounded
to BF16 before it enters a matrix product.
"""

from __future__ import annotations

import numpy as np
import torch


def bf16(x):
    return torch.as_tensor(np.asarray(x, np.float32)).to(torch.bfloat16).to(torch.float64).numpy()


def silu(z):
    return z / (1.0 + np.exp(-z))


def forward(W, b, X):
    """W, b: lists of FP32 arrays (out, in) and (out,); X: (B, in) already BF16-valued."""
    H = bf16(X)
    acts, pres = [H], []
    L = len(W)
    for l in range(L):
        Z = H @ bf16(W[l]).T + b[l]
        pres.append(Z)
        if l < L - 1:
            H = bf16(silu(Z))
            acts.append(H)
    return Z, acts, pres


def backward(W, acts, pres, dY):
    L = len(W)
    gW, gb = [None] * L, [None] * L
    dZ = np.asarray(dY, np.float64)
    for l in range(L - 1, -1, -1):
        d16 = bf16(dZ)
        gW[l] = d16.T @ acts[l]
        gb[l] = dZ.sum(axis=0)
        if l > 0:
            dH = d16 @ bf16(W[l])
            z = pres[l - 1]
            s = 1.0 / (1.0 + np.exp(-z))
            dZ = dH * (s * (1.0 + z * (1.0 - s)))
    return gW, gb
