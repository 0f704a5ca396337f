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
    """A headerless float32 volume of the given (NZ, NY, NX) shape (tools/evaluate.py:23-33)."""
    if len(shape) != 3 or any(s <= 0 for s in shape):
        raise ValueError("shape must contain three positive dimensions (NZ NY NX)")
    expected_bytes = int(np.prod(shape)) * np.dtype(np.float32).itemsize
    actual_bytes = Path(path).stat().st_size
    if actual_bytes != expected_bytes:
        raise ValueError(f"{path}: expected {expected_bytes} bytes, got {actual_bytes}")
    values = np.fromfile(path, dtype=np.float32)
    if values.size != int(np.prod(shape)):
        raise ValueError(f"{path}: expected {int(np.prod(shape))} float32 values, got {values.size}")
    return values.reshape(shape)


def _ratio_sqrt(num, den):
    return float(np.sqrt(num / den)) if den > 0 else None


class Evaluator:
    """Scores reconstructions against one truth (tools/evaluate.py:47-154)."""

    def __init__(self, truth, mask=None, data_range=None, background=None, hot_mask=None):
        truth = np.asarray(truth)
        if truth.ndim != 3 or not np.all(np.isfinite(truth)) or np.any(truth < 0):
            raise ValueError("truth must be a finite, nonnegative 3D activity volume")
        if not np.any(truth > 0):
            raise ValueError("truth must contain positive activity")
        t = truth.astype(np.float64)
        if mask is None:
            body = truth > 0
        else:
            mask = np.asarray(mask)
            if mask.shape != truth.shape or not np.all(np.isfinite(mask)):
                raise ValueError("mask must be finite and have the truth shape")
            body = mask > 0
            if not np.any(body):
                raise ValueError("mask must contain tissue voxels")
        self.body = body
        self.data_range = float(truth.max() if data_range is None else data_range)
        if not np.isfinite(self.data_range) or self.data_range <= 0:
            raise ValueError("data_range must be finite and positive")
        if background is None:
            values, counts = np.unique(truth[body & (truth > 0)], return_counts=True)
            if not values.size:
                raise ValueError("mask must include positive truth activity, or supply background")
            background = values[np.argmax(counts)]
        self.bg = float(background)
        if not np.isfinite(self.bg) or self.bg <= 0:
            raise ValueError("background must be finite and positive")
        if hot_mask is None:
            hot = (truth > 1.5 * self.bg) & body
            hot_definition = "truth > 1.5 * background (high-uptake regions; not necessarily lesions)"
        else:
            hot_mask = np.asarray(hot_mask)
            if hot_mask.shape != truth.shape or not np.all(np.isfinite(hot_mask)):
                raise ValueError("hot_mask must be finite and have the truth shape")
            hot = hot_mask > 0
            if np.any(hot & (~body | (truth <= 0))):
                raise ValueError("hot_mask must lie inside tissue with positive truth activity")
            hot_definition = "explicit hot mask; connected positive components define lesions"
        self.hot = hot
        self.hot_labels, self.n_hot = ndi.label(hot)
        self.metric_settings = {
            "data_range": self.data_range, "background": self.bg,
            "tissue_mask": "explicit mask" if mask is not None else "truth > 0",
            "hot_regions": hot_definition, "hot_region_count": int(self.n_hot),
            "hot_region_voxels": int(hot.sum()),
            "ssim_window": "3D Gaussian sigma 1.5, 11 voxels",
        }
        self.roi = ndi.find_objects(ndi.binary_dilation(body, iterations=4), max_label=1)[0]
        is_background = (np.abs(t - self.bg) < 1e-6 * self.bg) & body
        bg_interior = ndi.binary_erosion(is_background, structure=np.ones((3, 3, 3)), iterations=4)
        lo = ndi.minimum_filter(truth, size=5, mode="nearest").astype(np.float64)
        hi = ndi.maximum_filter(truth, size=5, mode="nearest").astype(np.float64)
        edge_band = hi > lo
        hot_shell = ndi.binary_dilation(hot, iterations=3) & ~ndi.binary_dilation(hot, iterations=1)
        skin_core = ndi.binary_erosion(body, iterations=4)
        halo_shell = hot_shell & skin_core & is_background
        self.t, self.lo, self.hi = t, lo, hi
        self.bg_interior, self.edge_band, self.halo_shell = bg_interior, edge_band, halo_shell
        classes = (body * CLASS_BODY | hot * CLASS_HOT | bg_interior * CLASS_BACKGROUND | edge_band * CLASS_EDGE
                   | halo_shell * CLASS_HALO).astype(np.uint8)
        classes[self.roi] |= CLASS_ROI
        self.shape = truth.shape
        self._box = tuple(s.stop - s.start for s in self.roi)
        roi = np.array([self.roi[0].start, self.roi[0].stop, self.roi[1].start, self.roi[1].stop,
                        self.roi[2].start, self.roi[2].stop], dtype=np.int32)
        labels = np.ascontiguousarray(self.hot_labels, dtype=np.int32)
        t = np.ascontiguousarray(t)
        handle = ctypes.c_void_p()
        nz, ny, nx = truth.shape
        rc = lib().prc_eval_create(nz, ny, nx, t.ctypes.data, classes.ctypes.data,
                                   labels.ctypes.data if self.n_hot else None, int(self.n_hot),
                                   lo.ctypes.data, hi.ctypes.data, roi.ctypes.data, self.data_range,
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
    """Markdown table of the COLUMNS of each (name, metrics) row (tools/evaluate.py:160-171)."""
    head = "| image | " + " | ".join(COLUMNS) + " |"
    sep = "|---|" + "---:|" * len(COLUMNS)
    lines = [head, sep]
    for name, m in rows:
        cells = ["—" if m.get(c) is None else f"{m.get(c):.4f}" for c in COLUMNS]
        lines.append(f"| {name} | " + " | ".join(cells) + " |")
    return "\n".join(lines)


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--truth", required=True)
    ap.add_argument("--shape", type=int, nargs=3, required=True, metavar=("NZ", "NY", "NX"))
    ap.add_argument("--json", help="write metrics to this JSON file")
    ap.add_argument("--mask", help="float32 tissue mask (positive = tissue), including cold regions")
    ap.add_argument("--hot-mask", help="float32 true hot-lesion mask (positive = lesion); recommended for smooth uptake")
    ap.add_argument("--data-range", type=float, help="fixed reference intensity range for SSIM/PSNR")
    ap.add_argument("--background", type=float, help="known background level for phantom metrics")
    ap.add_argument("images", nargs="+", help="name=path.raw")
    args = ap.parse_args(argv)
    ev = Evaluator(load(args.truth, args.shape),
                   mask=load(args.mask, args.shape) if args.mask else None,
                   data_range=args.data_range, background=args.background,
                   hot_mask=load(args.hot_mask, args.shape) if args.hot_mask else None)
    rows = []
    for item in args.images:
        name, path = item.rsplit("=", 1)
        rows.append((name, ev(load(path, args.shape))))
    print(format_table(rows))
    print("Hot-region definition: " + ev.metric_settings["hot_regions"])
    if args.json:
        with open(args.json, "w") as fh:
            json.dump({name: m for name, m in rows}, fh, indent=2, allow_nan=False)


if __name__ == "__main__":
    main()
