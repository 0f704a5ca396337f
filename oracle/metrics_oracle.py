"""CPU restatement of the reference's image-quality scorer -- TEST INFRASTRUCTURE ONLY.

Follows tools/evaluate.py of the reference: the masks of Evaluator.__init__ (:48-103) and the
metric formulas of Evaluator.__call__ (:105-154), in NumPy float64 with scipy.ndimage.  The
reference computes SSIM with scikit-image (structural_similarity, :125-127), which is not
installed here; ``ssim_map`` restates the published method (Wang et al. 2004) with the same
settings -- Gaussian window sigma 1.5 truncated at 3.5 sigma, population covariances,
K1 = 0.01, K2 = 0.03 -- so SSIM parity with the reference is unpinned.  The non-SSIM metrics
are pinned to the reference's own code by tests/golden/make_metrics_golden.py.
Only tests/ use this module; the device scorer (prc_mlem_b200.evaluate) is checked against it.
"""
from __future__ import annotations

import numpy as np
from scipy import ndimage as ndi

K1, K2, SIGMA, TRUNCATE = 0.01, 0.03, 1.5, 3.5


def ssim_map(x, y, data_range):
    """SSIM map of x (reference image) and y, and the half-width of the window."""
    x = np.asarray(x, np.float64)
    y = np.asarray(y, np.float64)
    filt = lambda a: ndi.gaussian_filter(a, sigma=SIGMA, truncate=TRUNCATE, mode="reflect")
    ux, uy = filt(x), filt(y)
    vx, vy, vxy = filt(x * x) - ux * ux, filt(y * y) - uy * uy, filt(x * y) - ux * uy
    c1, c2 = (K1 * data_range) ** 2, (K2 * data_range) ** 2
    s = ((2 * ux * uy + c1) * (2 * vxy + c2)) / ((ux * ux + uy * uy + c1) * (vx + vy + c2))
    return s, int(TRUNCATE * SIGMA + 0.5)


def _rel(diff, truth):
    norm = float(np.sum(truth ** 2))
    return float(np.sqrt(np.sum(diff ** 2) / norm)) if norm > 0 else None


def _mean(v):
    return float(v.mean()) if v.size else None


class Evaluator:
    """tools/evaluate.py:47-154 with SSIM restated (see the module notes)."""

    def __init__(self, truth, mask=None, data_range=None, background=None, hot_mask=None):
        truth = np.asarray(truth)
        if truth.ndim != 3 or not np.all(np.isfinite(truth)) or np.any(truth < 0):
            raise ValueError("truth must be a finite, nonnegative 3D activity volume")
        if not np.any(truth > 0):
            raise ValueError("truth must contain positive activity")
        self.t = truth.astype(np.float64)
        body = truth > 0 if mask is None else np.asarray(mask) > 0
        if mask is not None and not np.any(body):
            raise ValueError("mask must contain tissue voxels")
        self.body = body
        self.data_range = float(truth.max() if data_range is None else data_range)
        if background is None:
            values, counts = np.unique(truth[body & (truth > 0)], return_counts=True)
            background = values[np.argmax(counts)]
        self.bg = float(background)
        self.hot = (truth > 1.5 * self.bg) & body if hot_mask is None else np.asarray(hot_mask) > 0
        self.hot_labels, self.n_hot = ndi.label(self.hot)
        self.roi = ndi.find_objects(ndi.binary_dilation(body, iterations=4), max_label=1)[0]
        is_background = (np.abs(self.t - self.bg) < 1e-6 * self.bg) & body
        self.bg_interior = ndi.binary_erosion(is_background, structure=np.ones((3, 3, 3)), iterations=4)
        self.lo = ndi.minimum_filter(truth, size=5, mode="nearest").astype(np.float64)
        self.hi = ndi.maximum_filter(truth, size=5, mode="nearest").astype(np.float64)
        self.edge_band = self.hi > self.lo
        hot_shell = ndi.binary_dilation(self.hot, iterations=3) & ~ndi.binary_dilation(self.hot, iterations=1)
        skin_core = ndi.binary_erosion(body, iterations=4)
        self.halo_shell = hot_shell & skin_core & is_background

    def __call__(self, f):
        f = np.asarray(f, dtype=np.float64)
        if f.shape != self.t.shape or not np.all(np.isfinite(f)):
            raise ValueError("reconstruction must be finite and have the truth shape")
        t = self.t
        diff = f - t
        out = {"nrmse": _rel(diff, t), "nrmse_tissue": _rel(diff[self.body], t[self.body]),
               "mse": float(np.mean(diff ** 2)), "mae_tissue": _mean(np.abs(diff[self.body])),
               "count_bias": float(f.sum() / t.sum() - 1.0)}
        fr, tr = f[self.roi], t[self.roi]
        rmse_roi = np.sqrt(((fr - tr) ** 2).mean())
        out["psnr"] = float(20.0 * np.log10(self.data_range / rmse_roi)) if rmse_roi > 0 else None
        out.update(ssim=None, ssim_tissue=None, ssim_edge=None)
        if min(tr.shape) >= 11:
            smap, pad = ssim_map(tr, fr, self.data_range)
            valid = (slice(pad, -pad),) * 3
            smap = smap[valid]
            out["ssim"] = float(smap.mean())
            out["ssim_tissue"] = _mean(smap[self.body[self.roi][valid]])
            out["ssim_edge"] = _mean(smap[self.edge_band[self.roi][valid]])
        out["rc_hot"] = out["rc_min"] = None
        if self.n_hot:
            out["rc_hot"] = float(f[self.hot].mean() / t[self.hot].mean())
            labels = range(1, self.n_hot + 1)
            per = ndi.mean(f, self.hot_labels, labels) / ndi.mean(t, self.hot_labels, labels)
            out["rc_min"] = float(np.min(per))
        bgv = f[self.bg_interior]
        out["bg_bias"] = float(bgv.mean() / self.bg - 1.0) if bgv.size else None
        out["bg_cov"] = float(bgv.std() / bgv.mean()) if bgv.size and bgv.mean() > 0 else None
        over = np.maximum(f - self.hi, 0.0)[self.edge_band]
        under = np.maximum(self.lo - f, 0.0)[self.edge_band]
        out["ring"] = float(np.sqrt(np.mean((over + under) ** 2)) / self.bg) if over.size else None
        out["overshoot"] = float(np.sqrt(np.mean(over ** 2)) / self.bg) if over.size else None
        out["undershoot"] = float(np.sqrt(np.mean(under ** 2)) / self.bg) if under.size else None
        out["edge_nrmse"] = _rel(diff[self.edge_band], t[self.edge_band])
        halo = _mean(f[self.halo_shell])
        out["halo"] = 1.0 - halo / self.bg if halo is not None else None
        return out
