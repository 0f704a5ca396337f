#!/usr/bin/env python3
"""Reference-based NRMSE, 3D SSIM, uptake and local-range metrics, scored on the GPU.

The interface of the reference's scorer, tools/evaluate.py: ``load``, ``Evaluator(truth,
mask, data_range, background, hot_mask)`` whose call returns the same metric dictionary
(tools/evaluate.py:105-154), ``COLUMNS``, ``format_table`` and the same command line.  The
masks are fixed by the truth and built once on the host with the reference's definitions
(tools/evaluate.py:48-103); each reconstruction is then reduced on the device by
``libprc_b200.so`` (``prc_eval_sums``): one pass for every sum and three separable Gaussian
passes for SSIM.  A reconstruction may be a NumPy array or a CUDA tensor (float32 or float64).

SSIM follows Wang et al. (2004) as the reference configures it: Gaussian window sigma 1.5
truncated at 3.5 sigma (11 voxels), population covariances, K1 = 0.01, K2 = 0.03, the mean
over voxels at least 5 from every face of the dilated-body box.  The reference computes it
with scikit-image, which is not available to check against here; the mean over that interior
does not depend on how the filter extends the box.

Usage: python -m prc_mlem_b200.evaluate --truth TRUTH.raw --shape NZ NY NX name=image.raw [...]
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
from pathlib import Path

import numpy as np
from scipy import ndimage as ndi

from . import PrcError, lib

CLASS_BODY, CLASS_HOT, CLASS_BACKGROUND, CLASS_EDGE, CLASS_HALO, CLASS_ROI = 1, 2, 4, 8, 16, 32
(D2, T2, D2_BODY, T2_BODY, ABS_BODY, N_BODY, F, T, D2_ROI, N_ROI, F_HOT, T_HOT, F_BG, F2_BG, N_BG, RING2, OVER2,
 UNDER2, N_EDGE, D2_EDGE, T2_EDGE, F_HALO, N_HALO, NONFINITE, SSIM_SUM) = range(25)
NUM_SUMS = SSIM_SUM + 6
SSIM_WINDOW = 11


def load(path, shape):
    """A headerless little-endian float32 volume of shape (NZ, NY, NX); the file must hold
    exactly that many values (the loader contract of tools/evaluate.py:23-33)."""
    dims = tuple(int(d) for d in shape)
    if len(dims) != 3 or min(dims) <= 0:
        raise ValueError("shape must contain three positive dimensions (NZ NY NX)")
    want = 4 * math.prod(dims)
    raw = Path(path).read_bytes()
    if len(raw) != want:
        raise ValueError(f"{path}: expected {want} bytes, got {len(raw)}")
    return np.frombuffer(raw, dtype="<f4").reshape(dims).astype(np.float32)


def _ratio_sqrt(num, den):
    return float(np.sqrt(num / den)) if den > 0 else None


def _finite_volume_like(a, shape, what):
    """`a` as an array of `shape` with only finite values, else ValueError."""
    a = np.asarray(a)
    if a.shape != shape or not np.isfinite(a).all():
        raise ValueError(f"{what} must be finite and have the truth shape")
    return a


def _bounding_box(mask):
    """Slices of the smallest box holding every set voxel of a non-empty 3D mask."""
    box = []
    for axis in range(3):
        hit = np.flatnonzero(mask.any(axis=tuple(a for a in range(3) if a != axis)))
        box.append(slice(int(hit[0]), int(hit[-1]) + 1))
    return tuple(box)


def _class_volume(truth, body, hot, bg):
    """The per-voxel class byte of the scorer's regions, built in one pass over the masks of
    tools/evaluate.py:93-103 (their definitions are the metrics' meaning):
      body        tissue (the mask, or truth > 0);
      hot         the high-uptake regions;
      background  background-level tissue (|t - bg| < 1e-6 bg) eroded 4 times by a 3x3x3 cube;
      edge        voxels whose 5x5x5 neighbourhood of the truth is not constant;
      halo        background tissue 2-3 voxels outside a hot region and 4 voxels inside the skin;
      roi         the bounding box of the body dilated 4 times (PSNR and SSIM are taken there).
    Returns (classes uint8, 5x5x5 minimum, 5x5x5 maximum, roi slices)."""
    level = (np.abs(truth.astype(np.float64) - bg) < 1e-6 * bg) & body
    lo = ndi.minimum_filter(truth, size=5, mode="nearest").astype(np.float64)
    hi = ndi.maximum_filter(truth, size=5, mode="nearest").astype(np.float64)
    near_hot = ndi.binary_dilation(hot)  # 1 step; the halo's outer limit grows it 2 steps more
    shell = ndi.binary_dilation(near_hot, iterations=2) & ~near_hot
    classes = np.zeros(truth.shape, np.uint8)
    for bit, region in ((CLASS_BODY, body), (CLASS_HOT, hot),
                        (CLASS_BACKGROUND, ndi.binary_erosion(level, structure=np.ones((3, 3, 3)), iterations=4)),
                        (CLASS_EDGE, hi > lo),
                        (CLASS_HALO, shell & level & ndi.binary_erosion(body, iterations=4))):
        classes[region] |= bit
    roi = _bounding_box(ndi.binary_dilation(body, iterations=4))
    classes[roi] |= CLASS_ROI
    return classes, lo, hi, roi


class Evaluator:
    """Scores reconstructions against one truth (the Evaluator of tools/evaluate.py:47-154:
    same arguments, same checks and messages, same metric dictionary)."""

    def __init__(self, truth, mask=None, data_range=None, background=None, hot_mask=None):
        truth = np.asarray(truth)
        if truth.ndim != 3 or not np.isfinite(truth).all() or (truth < 0).any():
            raise ValueError("truth must be a finite, nonnegative 3D activity volume")
        if not (truth > 0).any():
            raise ValueError("truth must contain positive activity")
        shape = truth.shape
        body = truth > 0
        if mask is not None:
            body = _finite_volume_like(mask, shape, "mask") > 0
            if not body.any():
                raise ValueError("mask must contain tissue voxels")
        rng = float(truth.max()) if data_range is None else float(data_range)
        if not (np.isfinite(rng) and rng > 0):
            raise ValueError("data_range must be finite and positive")
        if background is None:  # the most frequent positive tissue value (the smallest on a tie)
            values, counts = np.unique(truth[body & (truth > 0)], return_counts=True)
            if values.size == 0:
                raise ValueError("mask must include positive truth activity, or supply background")
            background = values[counts == counts.max()][0]
        bg = float(background)
        if not (np.isfinite(bg) and bg > 0):
            raise ValueError("background must be finite and positive")
        if hot_mask is None:
            hot = (truth > 1.5 * bg) & body
            hot_definition = "truth > 1.5 * background (high-uptake regions; not necessarily lesions)"
        else:
            hot = _finite_volume_like(hot_mask, shape, "hot_mask") > 0
            if (hot & ~(body & (truth > 0))).any():
                raise ValueError("hot_mask must lie inside tissue with positive truth activity")
            hot_definition = "explicit hot mask; connected positive components define lesions"
        labels, n_hot = ndi.label(hot)
        self.body, self.hot, self.hot_labels, self.n_hot = body, hot, labels, n_hot
        self.data_range, self.bg, self.shape = rng, bg, shape
        self.metric_settings = {
            "data_range": rng, "background": bg,
            "tissue_mask": "truth > 0" if mask is None else "explicit mask",
            "hot_regions": hot_definition, "hot_region_count": int(n_hot),
            "hot_region_voxels": int(np.count_nonzero(hot)),
            "ssim_window": "3D Gaussian sigma 1.5, 11 voxels",
        }
        classes, lo, hi, self.roi = _class_volume(truth, body, hot, bg)
        self._box = tuple(r.stop - r.start for r in self.roi)
        corners = np.array([[r.start, r.stop] for r in self.roi], dtype=np.int32).ravel()
        t = np.ascontiguousarray(truth, dtype=np.float64)
        lab = np.ascontiguousarray(labels, dtype=np.int32)
        handle = ctypes.c_void_p()
        rc = lib().prc_eval_create(*shape, t.ctypes.data, classes.ctypes.data, lab.ctypes.data if n_hot else None,
                                   int(n_hot), lo.ctypes.data, hi.ctypes.data, corners.ctypes.data, rng,
                                   ctypes.byref(handle))
        if rc != 0:
            raise PrcError(rc, lib().prc_last_error().decode())
        self._handle = handle

    def close(self) -> None:
        if getattr(self, "_handle", None):
            lib().prc_eval_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def sums(self, f) -> np.ndarray:
        """The device's FP64 sums for reconstruction f (NumPy array or CUDA tensor)."""
        import torch
        if isinstance(f, torch.Tensor):
            d = f.detach()
            if tuple(d.shape) != self.shape:
                raise ValueError("reconstruction must be finite and have the truth shape")
            if d.dtype not in (torch.float32, torch.float64):
                d = d.to(torch.float64)
            d = d.cuda().contiguous()
        else:
            a = np.asarray(f)
            if a.shape != self.shape:
                raise ValueError("reconstruction must be finite and have the truth shape")
            a = np.ascontiguousarray(a, dtype=np.float32 if a.dtype == np.float32 else np.float64)
            d = torch.from_numpy(a).cuda()
        out = np.zeros(NUM_SUMS + 2 * self.n_hot, dtype=np.float64)
        fn = lib().prc_eval_sums if d.dtype == torch.float32 else lib().prc_eval_sums_f64
        stream = torch.cuda.current_stream(d.device).cuda_stream
        rc = fn(self._handle, d.data_ptr(), out.ctypes.data, stream)
        if rc != 0:
            raise PrcError(rc, lib().prc_last_error().decode())
        return out

    def __call__(self, f):
        s = self.sums(f)
        if s[NONFINITE] > 0:
            raise ValueError("reconstruction must be finite and have the truth shape")
        n = float(np.prod(self.shape))
        bg = self.bg
        out = {}
        out["nrmse"] = _ratio_sqrt(s[D2], s[T2])
        out["nrmse_tissue"] = _ratio_sqrt(s[D2_BODY], s[T2_BODY])
        out["mse"] = float(s[D2] / n)
        out["mae_tissue"] = float(s[ABS_BODY] / s[N_BODY]) if s[N_BODY] else None
        out["count_bias"] = float(s[F] / s[T] - 1.0)
        rmse_roi = np.sqrt(s[D2_ROI] / s[N_ROI])
        out["psnr"] = float(20.0 * np.log10(self.data_range / rmse_roi)) if rmse_roi > 0 else None
        out.update(ssim=None, ssim_tissue=None, ssim_edge=None)
        if min(self._box) >= SSIM_WINDOW:
            out["ssim"] = float(s[SSIM_SUM] / s[SSIM_SUM + 1])
            out["ssim_tissue"] = float(s[SSIM_SUM + 2] / s[SSIM_SUM + 3]) if s[SSIM_SUM + 3] else None
            out["ssim_edge"] = float(s[SSIM_SUM + 4] / s[SSIM_SUM + 5]) if s[SSIM_SUM + 5] else None
        out["rc_hot"] = out["rc_min"] = None
        if self.n_hot:
            out["rc_hot"] = float(s[F_HOT] / s[T_HOT])
            per = s[NUM_SUMS::2] / s[NUM_SUMS + 1::2]
            out["rc_min"] = float(np.min(per))
        if s[N_BG]:
            mean = s[F_BG] / s[N_BG]
            var = max(s[F2_BG] / s[N_BG] - mean * mean, 0.0)
            out["bg_bias"] = float(mean / bg - 1.0)
            out["bg_cov"] = float(np.sqrt(var) / mean) if mean > 0 else None
        else:
            out["bg_bias"] = out["bg_cov"] = None
        if s[N_EDGE]:
            out["ring"] = float(np.sqrt(s[RING2] / s[N_EDGE]) / bg)
            out["overshoot"] = float(np.sqrt(s[OVER2] / s[N_EDGE]) / bg)
            out["undershoot"] = float(np.sqrt(s[UNDER2] / s[N_EDGE]) / bg)
        else:
            out["ring"] = out["overshoot"] = out["undershoot"] = None
        out["edge_nrmse"] = _ratio_sqrt(s[D2_EDGE], s[T2_EDGE])
        out["halo"] = float(1.0 - (s[F_HALO] / s[N_HALO]) / bg) if s[N_HALO] else None
        return out


COLUMNS = ["nrmse", "ssim", "ssim_tissue", "ssim_edge", "edge_nrmse", "rc_hot", "rc_min", "bg_cov", "ring", "halo"]


def format_table(rows):
    """Markdown table: one row per (name, metrics), the COLUMNS to 4 decimals, a dash where a
    score is unavailable (the table of tools/evaluate.py:160-171)."""
    def cell(v):
        return "—" if v is None else f"{v:.4f}"
    table = [f"| image | {' | '.join(COLUMNS)} |", "|---|" + "---:|" * len(COLUMNS)]
    table += [f"| {name} | {' | '.join(cell(m.get(c)) for c in COLUMNS)} |" for name, m in rows]
    return "\n".join(table)


# the command line of tools/evaluate.py:174-197: flag, options
_FLAGS = (("--truth", dict(required=True)),
          ("--shape", dict(type=int, nargs=3, required=True, metavar=("NZ", "NY", "NX"))),
          ("--json", dict(help="write metrics to this JSON file")),
          ("--mask", dict(help="float32 tissue mask (positive = tissue), including cold regions")),
          ("--hot-mask", dict(help="float32 true hot-lesion mask (positive = lesion); recommended for smooth uptake")),
          ("--data-range", dict(type=float, help="fixed reference intensity range for SSIM/PSNR")),
          ("--background", dict(type=float, help="known background level for phantom metrics")),
          ("images", dict(nargs="+", help="name=path.raw")))


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    for flag, kw in _FLAGS:
        ap.add_argument(flag, **kw)
    a = ap.parse_args(argv)

    def optional(path):
        return None if not path else load(path, a.shape)

    ev = Evaluator(load(a.truth, a.shape), mask=optional(a.mask), data_range=a.data_range,
                   background=a.background, hot_mask=optional(a.hot_mask))
    scored = {}
    for item in a.images:
        name, _, path = item.rpartition("=")
        scored[name] = ev(load(path, a.shape))
    print(format_table(scored.items()))
    print("Hot-region definition: " + ev.metric_settings["hot_regions"])
    if a.json:
        Path(a.json).write_text(json.dumps(scored, indent=2, allow_nan=False))


if __name__ == "__main__":
    main()
