"""Float64 restatement of the surrogate network (test oracle; only tests and the
benchmark's checker import it).

The learned surrogate has no counterpart in the reference, so this oracle is the
same network written with plain torch float64 CPU operations and autograd: the
truncated 2D DFT as explicit cos/sin sums over the kept modes, the per-mode complex
channel mixing, GELU (tanh form), pooled head. It checks the bf16 kernels' forward
values and gradients (parameters and input density).
"""
from __future__ import annotations

import math

import numpy as np
import torch


def bases(n: int, modes: int):
    ky = np.concatenate([np.arange(modes), np.arange(n - modes, n)])
    kx = np.arange(modes)
    KY, KX = [a.ravel() for a in np.meshgrid(ky, kx, indexing="ij")]
    y, x = [a.ravel() for a in np.meshgrid(np.arange(n), np.arange(n), indexing="ij")]
    th = 2 * np.pi * (np.outer(y, KY) + np.outer(x, KX)) / n  # [P][K]
    w = np.where(KX == 0, 1.0, 2.0) / (n * n)
    return torch.as_tensor(np.cos(th)), torch.as_tensor(np.sin(th)), torch.as_tensor(w)


def gelu(v):
    return 0.5 * v * (1.0 + torch.tanh(math.sqrt(2.0 / math.pi) * (v + 0.044715 * v ** 3)))


def forward(params: dict, rho: torch.Tensor, n: int, modes: int, layers: int):
    """params: name -> float64 tensor (W0 [C,3], b0, W1.., b1.., R1.. [K,C,C,2], Q1, q1, Q2, q2)."""
    cos, sin, w = bases(n, modes)
    B = rho.shape[0]
    P = n * n
    c = (torch.arange(n, dtype=torch.float64) + 0.5) / n
    X = torch.stack([rho.reshape(B, P), c[None, :].expand(n, n).reshape(1, P).expand(B, P),
                     c[:, None].expand(n, n).reshape(1, P).expand(B, P)], dim=1)  # [B][3][P]
    V = torch.einsum("cj,bjp->bcp", params["W0"], X) + params["b0"][None, :, None]
    for l in range(1, layers + 1):
        ur = torch.einsum("bcp,pk->bck", V, cos)
        ui = -torch.einsum("bcp,pk->bck", V, sin)
        R = params[f"R{l}"]
        orr = torch.einsum("bck,kco->bok", ur, R[..., 0]) - torch.einsum("bck,kco->bok", ui, R[..., 1])
        oi = torch.einsum("bck,kco->bok", ur, R[..., 1]) + torch.einsum("bck,kco->bok", ui, R[..., 0])
        S = torch.einsum("bok,pk->bop", orr * w, cos) - torch.einsum("bok,pk->bop", oi * w, sin)
        Vn = torch.einsum("oc,bcp->bop", params[f"W{l}"], V) + params[f"b{l}"][None, :, None] + S
        V = gelu(Vn) if l < layers else Vn
    H = gelu(torch.einsum("hc,bcp->bhp", params["Q1"], V) + params["q1"][None, :, None])
    pooled = H.mean(dim=2)
    return pooled @ params["Q2"].T + params["q2"][None, :]
