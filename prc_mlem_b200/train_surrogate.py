"""Trains the learned range-kernel surrogate on the GPU and writes its weights.

    python -m prc_mlem_b200.train_surrogate [--volumes 4096] [--epochs 15] [--out PATH]

Training set: random 48^3 volumes at 0.8 mm, each air plus a seeded union of 3-10 ellipsoids
with densities from {0.0012, 0.26, 1.0, 1.4, 1.85} and 0, 2 or 5 % Gaussian density jitter (by
turns, per chunk of 256 volumes); 32 tissue voxels per volume and isotope (18F, 68Ga, 82Rb);
targets are the plain ray tracer's far-field kernels (128 rays, 16 radial bins), masked where
a surrogate field keeps exact weights or stores nothing.  The network trains with the library's bf16 tensor-core kernels and Adam
(lr 3e-4, cosine decay to 0).  Prints one JSON line with the loss history and the validation
MSE of the network and of the density-blind mean kernel (both over the unmasked targets).
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--volumes", type=int, default=4096)
    ap.add_argument("--per-volume", type=int, default=32)
    ap.add_argument("--epochs", type=int, default=15)
    ap.add_argument("--batch", type=int, default=256)
    ap.add_argument("--lr", type=float, default=3e-4)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--out", default=None)
    args = ap.parse_args()
    import torch
    from . import surrogate as sg

    t0 = time.perf_counter()
    x, t = sg.make_dataset(args.volumes, args.per_volume, seed=args.seed)
    xv, tv = sg.make_dataset(max(64, args.volumes // 32), args.per_volume, seed=args.seed + 1000)
    torch.cuda.synchronize()
    t_data = time.perf_counter() - t0
    net = sg.Network(sg.init_params(args.seed))
    t0 = time.perf_counter()
    history = sg.train(net, x, t, epochs=args.epochs, batch=args.batch, lr=args.lr, seed=args.seed)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    keep = (tv >= 0).float()
    val = net.evaluate(xv, tv) * float(keep.numel() / keep.sum())  # per unmasked target
    used = (t >= 0).float()
    mean = (t.clamp(min=0) * used).sum(0, keepdim=True) / used.sum(0, keepdim=True).clamp(min=1)
    blind = float((((tv - mean) * keep) ** 2).sum() / keep.sum())
    out = args.out or str(sg.PARAMS_PATH)
    np.save(out, net.params())
    print(json.dumps({"samples": int(x.shape[0]), "data_s": round(t_data, 2), "train_s": round(t_train, 2),
                      "loss": [round(v, 5) for v in history], "val_mse": val, "blind_val_mse": blind,
                      "weights": out}))


if __name__ == "__main__":
    main()
