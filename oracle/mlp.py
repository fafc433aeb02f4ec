"""CPU oracle of the warm-start MLP (test infrastructure only).

Float64 restatement of the forward and backward passes of
``fenics_nonlinear_energies_b200.warmstart.NodalMLP``, rounding to bfloat16
(round-to-nearest-even) at exactly the points where the kernels store BF16:
the layer inputs, the weights and the pre-activation gradients fed to the
GEMMs.  Everything else is float64, so the comparison isolates the kernels'
FP32 accumulation.
"""

from __future__ import annotations

import numpy as np


def bf16_round(x):
    """Round float32 values to the nearest bfloat16 (ties to even), returned as float64."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def silu(z):
    return z / (1.0 + np.exp(-z))


def silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(W, b, X):
    """Returns the output and the (input_bf16, Z) pairs of every layer."""
    h = bf16_round(X)
    saved = []
    L = len(W)
    for l in range(L):
        Wl = bf16_round(W[l])
        Z = h @ Wl.T + b[l]
        saved.append((h, Z))
        if l < L - 1:
            h = bf16_round(silu(Z))
        else:
            h = Z
    return h, saved


def backward(W, saved, dY):
    L = len(W)
    gW, gb = [None] * L, [None] * L
    dH = np.asarray(dY, dtype=np.float64)
    for l in reversed(range(L)):
        h, Z = saved[l]
        dZ = dH if l == L - 1 else dH * silu_grad(Z)
        dZ16 = bf16_round(dZ)
        gW[l] = dZ16.T @ h
        gb[l] = dZ.sum(axis=0)
        if l > 0:
            dH = dZ16 @ bf16_round(W[l])
    return gW, gb
