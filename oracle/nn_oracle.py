"""CPU oracle of the learned range-kernel surrogate network -- TEST INFRASTRUCTURE ONLY.

The network has no counterpart in the reference; this FP64 NumPy restatement defines it and
checks the tensor-core training kernels (forward values and every gradient).  Activations are
rounded to bfloat16 at exactly the points where the CUDA path stores them in bf16, so the only
remaining differences are fp32-vs-fp64 accumulation.

Network (per sample: a 9^3 patch, channels-last):
  x0 [9,9,9,4]   density / 2 and a one-hot isotope (18F, 68Ga, 82Rb)
  a1 = relu(conv3(x0, W1) + b1)  [7,7,7,32]   W: [cout][kz][ky][kx][cin]
  a2 = relu(conv3(a1, W2) + b2)  [5,5,5,32]
  a3 = relu(conv3(a2, W3) + b3)  [3,3,3,32]
  a4 = relu(conv3(a3, W4) + b4)  [32]
  y  = a4 . Wh^T + bh            [2048] = 128 directions x 16 radial bins
Loss: mean over B x 2048 of (y - t)^2.
"""
from __future__ import annotations

import numpy as np

C = 32
OUT = 2048


def bf16(x):
    """Round float values to bfloat16 (round to nearest even), returned as float64."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def conv3_valid(x, w):
    """x [B,S,S,S,Cin], w [Cout,3,3,3,Cin] -> [B,S-2,S-2,S-2,Cout] (cross-correlation)."""
    B, S = x.shape[0], x.shape[1]
    So = S - 2
    out = np.zeros((B, So, So, So, w.shape[0]))
    for kz in range(3):
        for ky in range(3):
            for kx in range(3):
                out += np.einsum("bzyxc,oc->bzyxo", x[:, kz:kz + So, ky:ky + So, kx:kx + So, :], w[:, kz, ky, kx, :])
    return out


def conv3_valid_dx(dy, w, S):
    """Gradient of conv3_valid with respect to its input of size S."""
    B, So = dy.shape[0], dy.shape[1]
    dx = np.zeros((B, S, S, S, w.shape[-1]))
    for kz in range(3):
        for ky in range(3):
            for kx in range(3):
                dx[:, kz:kz + So, ky:ky + So, kx:kx + So, :] += np.einsum("bzyxo,oc->bzyxc", dy, w[:, kz, ky, kx, :])
    return dx


def conv3_valid_dw(x, dy):
    So = dy.shape[1]
    dw = np.zeros((dy.shape[-1], 3, 3, 3, x.shape[-1]))
    for kz in range(3):
        for ky in range(3):
            for kx in range(3):
                dw[:, kz, ky, kx, :] = np.einsum("bzyxo,bzyxc->oc", dy, x[:, kz:kz + So, ky:ky + So, kx:kx + So, :])
    return dw


class Net:
    """Parameters as float64 arrays in the layouts the CUDA network uses."""

    def __init__(self, params: dict):
        self.p = {k: np.asarray(v, dtype=np.float64) for k, v in params.items()}

    def forward(self, x0):
        p = self.p
        W = [bf16(p[f"w{i}"]) for i in range(1, 5)]
        acts = [bf16(x0)]
        for i in range(4):
            z = conv3_valid(acts[-1], W[i]) + p[f"b{i + 1}"]
            acts.append(bf16(np.maximum(z, 0.0)))
        a4 = acts[-1].reshape(len(x0), C)
        y = a4 @ bf16(p["wh"]).T + p["bh"]
        return y, acts

    def loss_and_grads(self, x0, target):
        p = self.p
        B = len(x0)
        y, acts = self.forward(x0)
        loss = float(np.mean((y - target) ** 2))
        dy = bf16(2.0 * (y - target) / (B * OUT))
        a4 = acts[4].reshape(B, C)
        g = {"wh": dy.T @ a4, "bh": dy.sum(0)}
        dz = bf16((dy @ bf16(p["wh"])) * (a4 > 0)).reshape(B, 1, 1, 1, C)
        for i in range(4, 0, -1):
            x = acts[i - 1]
            g[f"w{i}"] = conv3_valid_dw(x, dz)
            g[f"b{i}"] = dz.sum(axis=(0, 1, 2, 3))
            if i > 1:
                dx = conv3_valid_dx(dz, bf16(p[f"w{i}"]), x.shape[1])
                dz = bf16(dx * (x > 0))
        return loss, g
