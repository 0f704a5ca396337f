"""CPU oracle of the learned range-kernel surrogate network -- TEST INFRASTRUCTURE ONLY.

The network has no counterpart in the reference; this FP64 NumPy restatement defines it and
checks the tensor-core training kernels (forward values and every gradient).  Activations are
rounded to bfloat16 at exactly the points where the CUDA path stores them in bf16, so the only
remaining differences are fp32-vs-fp64 accumulation.

Network (per sample: a 21^3 patch, channels-last; conv3 with dilation d reads taps d apart):
  x0 [21,21,21,8]   density / 2, inside-the-volume flag, one-hot isotope (18F, 68Ga, 82Rb), 3 zeros
  a1 = relu(conv3(x0, W1, d=1) + b1)  [19,19,19,32]   W: [cout][kz][ky][kx][cin]
  a2 = relu(conv3(a1, W2, d=2) + b2)  [15,15,15,32]
  a3 = relu(conv3(a2, W3, d=3) + b3)  [9,9,9,32]
  a4 = relu(conv3(a3, W4, d=4) + b4)  [32]
  y  = a4 . Wh^T + bh                 [2048] = 128 directions x 16 radial bins
Loss: mean over B x 2048 of (y - t)^2, with outputs whose target is negative counted as zero.
"""
from __future__ import annotations

import numpy as np

C = 32
OUT = 2048
DIL = (1, 2, 3, 4)
SIDE = 1 + 2 * sum(DIL)


def bf16(x):
    """Round float values to bfloat16 (round to nearest even), returned as float64."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def conv3_valid(x, w, d=1):
    """x [B,S,S,S,Cin], w [Cout,3,3,3,Cin] -> [B,S-2d,S-2d,S-2d,Cout] (cross-correlation, taps d apart)."""
    B, S = x.shape[0], x.shape[1]
    So = S - 2 * d
    out = np.zeros((B, So, So, So, w.shape[0]))
    for kz in range(3):
        for ky in range(3):
            for kx in range(3):
                z, y, xx = kz * d, ky * d, kx * d
                out += np.einsum("bzyxc,oc->bzyxo", x[:, z:z + So, y:y + So, xx:xx + So, :], w[:, kz, ky, kx, :])
    return out


def conv3_valid_dx(dy, w, S, d=1):
    """Gradient of conv3_valid with respect to its input of size S."""
    B, So = dy.shape[0], dy.shape[1]
    dx = np.zeros((B, S, S, S, w.shape[-1]))
    for kz in range(3):
        for ky in range(3):
            for kx in range(3):
                z, y, xx = kz * d, ky * d, kx * d
                dx[:, z:z + So, y:y + So, xx:xx + So, :] += np.einsum("bzyxo,oc->bzyxc", dy, w[:, kz, ky, kx, :])
    return dx


def conv3_valid_dw(x, dy, d=1):
    So = dy.shape[1]
    dw = np.zeros((dy.shape[-1], 3, 3, 3, x.shape[-1]))
    for kz in range(3):
        for ky in range(3):
            for kx in range(3):
                z, y, xx = kz * d, ky * d, kx * d
                dw[:, kz, ky, kx, :] = np.einsum("bzyxo,bzyxc->oc", dy, x[:, z:z + So, y:y + So, xx:xx + So, :])
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
            z = conv3_valid(acts[-1], W[i], DIL[i]) + p[f"b{i + 1}"]
            acts.append(bf16(np.maximum(z, 0.0)))
        a4 = acts[-1].reshape(len(x0), C)
        y = a4 @ bf16(p["wh"]).T + p["bh"]
        return y, acts

    def loss_and_grads(self, x0, target):
        p = self.p
        B = len(x0)
        y, acts = self.forward(x0)
        diff = np.where(target < 0, 0.0, y - target)  # negative targets are masked
        loss = float(np.mean(diff ** 2))
        dy = bf16(2.0 * diff / (B * OUT))
        a4 = acts[4].reshape(B, C)
        g = {"wh": dy.T @ a4, "bh": dy.sum(0)}
        dz = bf16((dy @ bf16(p["wh"])) * (a4 > 0)).reshape(B, 1, 1, 1, C)
        for i in range(4, 0, -1):
            x = acts[i - 1]
            g[f"w{i}"] = conv3_valid_dw(x, dz, DIL[i - 1])
            g[f"b{i}"] = dz.sum(axis=(0, 1, 2, 3))
            if i > 1:
                dx = conv3_valid_dx(dz, bf16(p[f"w{i}"]), x.shape[1], DIL[i - 1])
                dz = bf16(dx * (x > 0))
        return loss, g
