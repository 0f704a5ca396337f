"""The learned range-kernel surrogate: training data, training and the trained network.

A 3D CNN (four 3x3x3 convolutions of 32 channels with dilations 1, 2, 3 and 4 on a 21^3
density patch, an inside-the-volume flag and a one-hot isotope, and a linear head) predicts,
for every tissue voxel, its far-field range kernel as 128 ray directions x 16 radial bins of
deposit coefficients.  The targets come from the plain ray tracer (include/prc_surrogate.h:
prc_nn_make_samples) on random ellipsoid phantoms, masked (-1) where a surrogate field never
uses the network's output; the network trains on the GPU with the library's own bf16
tensor-core forward and backward kernels and Adam.  `Projector(..., surrogate=net)` then
builds the surrogate coefficient field by whole-volume inference, with the tracer as judge and
fallback.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

from . import _check, lib

ISOTOPES = ("18F", "68Ga", "82Rb")
DENSITIES = (0.0012, 0.26, 1.0, 1.4, 1.85)
TARGET_SCALE = 10.0   # targets are trained as 10 x the deposit coefficients
# Relative density jitter of the training volumes, by turns: noiseless phantoms and noisy
# (CT-like) maps both occur in use, and a network that only saw 5 % noise reads a noiseless map
# with a bias (its rectified noise features vanish there).
JITTERS = (0.0, 0.02, 0.05)
SIDE = 48             # training volumes: 48^3 voxels of 0.8 mm
SPACING = 0.8
PARAMS_PATH = Path(__file__).resolve().parent / "data" / "surrogate_params.npy"
IN_CHANNELS = 8       # density / 2, inside-the-volume flag, one-hot isotope, 3 zeros
SHAPES = [("w1", (32, 3, 3, 3, IN_CHANNELS)), ("b1", (32,)), ("w2", (32, 3, 3, 3, 32)), ("b2", (32,)),
          ("w3", (32, 3, 3, 3, 32)), ("b3", (32,)), ("w4", (32, 3, 3, 3, 32)), ("b4", (32,)),
          ("wh", (2048, 32)), ("bh", (2048,))]


def init_params(seed: int = 0) -> np.ndarray:
    """He-initialised weights and small positive biases (every ReLU starts alive), flattened in
    the library's parameter order."""
    rng = np.random.default_rng(seed)
    parts = []
    for name, shape in SHAPES:
        if name.startswith("w"):
            fan_in = int(np.prod(shape[1:]))
            parts.append(rng.normal(0.0, np.sqrt(2.0 / fan_in), shape).ravel())
        else:
            parts.append(np.full(shape, 0.05 if name != "bh" else 0.0).ravel())
    return np.concatenate(parts).astype(np.float32)


def ellipsoids(n_vol: int, seed: int, side: int = SIDE) -> np.ndarray:
    """[n_vol][10][8] parameters: each volume a union of 3-10 ellipsoids (centre, radii in
    voxels, density from DENSITIES, used flag), painted in order over air."""
    rng = np.random.default_rng(seed)
    e = np.zeros((n_vol, 10, 8), np.float32)
    for v in range(n_vol):
        k = rng.integers(3, 11)
        for j in range(k):
            big = j == 0
            e[v, j, 0:3] = rng.uniform(0.2 * side, 0.8 * side, 3) if big else rng.uniform(0, side, 3)
            e[v, j, 3:6] = rng.uniform(0.3 * side, 0.6 * side, 3) if big else rng.uniform(2.0, 0.35 * side, 3)
            e[v, j, 6] = 1.0 if big else rng.choice(DENSITIES)
            e[v, j, 7] = 1.0
    return e


class Network:
    """The CNN on the device (prc_nn_*): fp32 master weights, bf16 tensor-core copies, Adam."""

    def __init__(self, params: np.ndarray | None = None, max_batch: int = 512):
        h = ctypes.c_void_p()
        _check(lib().prc_nn_create(max_batch, ctypes.byref(h)))
        self._h = h
        self.max_batch = max_batch
        self.set_params(init_params() if params is None else params)

    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None):
            lib().prc_nn_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, params: np.ndarray) -> None:
        params = np.ascontiguousarray(params, np.float32)
        assert params.size == lib().prc_nn_param_count()
        _check(lib().prc_nn_set_params(self._h, params.ctypes.data))

    def params(self) -> np.ndarray:
        out = np.zeros(lib().prc_nn_param_count(), np.float32)
        _check(lib().prc_nn_get(self._h, 0, out.ctypes.data))
        return out

    def train_step(self, x, t, lr: float) -> float:
        """One forward + backward + Adam step on a batch (torch CUDA tensors); returns the MSE."""
        b = x.shape[0]
        _check(lib().prc_nn_forward(self._h, x.data_ptr(), b, None, None))
        loss = ctypes.c_double()
        _check(lib().prc_nn_backward(self._h, t.data_ptr(), b, lr, ctypes.byref(loss), None))
        return loss.value

    def predict(self, x):
        import torch
        y = torch.empty(x.shape[0], 2048, dtype=torch.float32, device="cuda")
        _check(lib().prc_nn_forward(self._h, x.data_ptr(), x.shape[0], y.data_ptr(), None))
        return y

    def evaluate(self, x, t, batch: int = 512) -> float:
        """MSE over a data set (masked targets count as zero error) without updating the weights."""
        total = 0.0
        for i in range(0, x.shape[0], batch):
            xb, tb = x[i:i + batch], t[i:i + batch]
            _check(lib().prc_nn_forward(self._h, xb.data_ptr(), xb.shape[0], None, None))
            loss = ctypes.c_double()
            _check(lib().prc_nn_backward(self._h, tb.data_ptr(), xb.shape[0], 0.0, ctypes.byref(loss), None))
            total += loss.value * xb.shape[0]
        return total / x.shape[0]


def patch_side() -> int:
    """Side of the network's input patch (21)."""
    return int(lib().prc_nn_patch_side())


def make_dataset(n_vol: int, per_vol: int = 32, seed: int = 1, isotopes=ISOTOPES, chunk: int = 256,
                 jitters=JITTERS):
    """(patches [N][21][21][21][8] bf16, targets [N][2048] fp32, -1 where masked) on the GPU for
    every isotope; successive chunks of volumes take their density jitter from `jitters` in
    turn."""
    import torch
    side = patch_side()
    xs, ts = [], []
    for ii, iso in enumerate(isotopes):
        for c0 in range(0, n_vol, chunk):
            nv = min(chunk, n_vol - c0)
            ell = ellipsoids(nv, seed * 1000003 + ii * 7919 + c0)
            x = torch.empty(nv * per_vol, side, side, side, IN_CHANNELS, dtype=torch.bfloat16, device="cuda")
            t = torch.empty(nv * per_vol, 2048, dtype=torch.float32, device="cuda")
            chunk_no = c0 // chunk
            _check(lib().prc_nn_make_samples(iso.encode(), nv, SIDE, SPACING, ell.ctypes.data,
                                             seed * 7 + ii * 131 + c0, per_vol, x.data_ptr(), t.data_ptr(),
                                             TARGET_SCALE, jitters[chunk_no % len(jitters)], None))
            xs.append(x)
            ts.append(t)
    if len(xs) == 1:
        return xs[0], ts[0]
    out = torch.empty((sum(len(x) for x in xs),) + tuple(xs[0].shape[1:]), dtype=xs[0].dtype, device="cuda")
    i = 0
    for x in xs:  # one copy at a time: the patches are large
        out[i:i + len(x)] = x
        i += len(x)
    del xs
    return out, torch.cat(ts)


def train(net: Network, x, t, epochs: int = 4, batch: int = 256, lr: float = 3e-4, seed: int = 0, log=None,
          cosine: bool = True):
    """Adam over shuffled mini-batches, the step size decaying from lr to 0 on a half cosine over
    the run (cosine=False: constant); returns the per-epoch mean training loss."""
    import math
    import torch
    g = torch.Generator(device="cuda").manual_seed(seed)
    n = x.shape[0]
    steps = max(1, epochs * (n // batch))
    step = 0
    history = []
    for ep in range(epochs):
        perm = torch.randperm(n, device="cuda", generator=g)
        total, count = 0.0, 0
        for i in range(0, n - batch + 1, batch):
            idx = perm[i:i + batch]
            rate = lr * 0.5 * (1.0 + math.cos(math.pi * step / steps)) if cosine else lr
            step += 1
            loss = net.train_step(x[idx].contiguous(), t[idx].contiguous(), rate)
            total += loss
            count += 1
        history.append(total / max(count, 1))
        if log:
            log(f"epoch {ep}: loss {history[-1]:.5f}")
    return history


def load_trained(max_batch: int = 512) -> Network | None:
    """The network with the committed trained weights, or None when they are absent."""
    if not PARAMS_PATH.is_file():
        return None
    return Network(np.load(PARAMS_PATH), max_batch=max_batch)
