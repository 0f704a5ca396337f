"""Seeded inputs of the image-metric parity cases (shared by make_metrics_golden.py and the
tests, so the golden file holds only the reference's outputs)."""
import numpy as np
from scipy import ndimage as ndi


def cube_phantom():
    """The 35^3 metrics phantom of the reference's tests/test_metrics.py:18-22."""
    truth = np.zeros((35, 35, 35), dtype=np.float32)
    truth[4:31, 4:31, 4:31] = 1
    truth[13:22, 13:22, 13:22] = 4
    return truth


def torso_crop():
    """A 40x48x56 crop of a seeded torso-like volume: water body with lungs and hot lesions."""
    rng = np.random.default_rng(21)
    z, y, x = np.mgrid[0:40, 0:48, 0:56].astype(np.float32)
    truth = np.zeros((40, 48, 56), np.float32)
    body = ((x - 28) / 25) ** 2 + ((y - 24) / 20) ** 2 <= 1
    truth[body] = 1.0
    for cx in (18, 38):
        truth[((x - cx) / 7) ** 2 + ((y - 24) / 10) ** 2 + ((z - 20) / 14) ** 2 <= 1] = 0.3
    for _ in range(5):
        c = rng.uniform([8, 12, 12], [32, 36, 44])
        r = rng.uniform(1.5, 4.0)
        truth[(z - c[0]) ** 2 + (y - c[1]) ** 2 + (x - c[2]) ** 2 <= r * r] = rng.uniform(3, 8)
    return truth


def cases():
    """(name, truth, evaluator keywords, {candidate name: candidate}) of every parity case."""
    out = []
    t = cube_phantom()
    rng = np.random.default_rng(4)
    ring = t.copy()
    ring[13:15, 13:22, 13:22] += 0.5
    ring[11:13, 13:22, 13:22] = -0.2
    out.append(("cube", t, {}, {
        "identity": t,
        "gauss07": ndi.gaussian_filter(t.astype(np.float64), sigma=0.7),
        "uniform3": ndi.uniform_filter(t, size=3),
        "ring": ring,
        "noisy": t + rng.normal(0, 0.2, t.shape) * (t > 0),
    }))
    lesions = t == 4
    t2 = t.copy()
    t2[5:9, 5:9, 5:9] = 2
    c2 = t2.copy()
    c2[5:9, 5:9, 5:9] = 1
    out.append(("cube_hot_mask", t2, {"background": 1, "hot_mask": lesions}, {"bright_bg": c2,
                                                                           "gauss08": ndi.gaussian_filter(t2, 0.8)}))
    t3 = t.copy()
    body = t3 > 0
    t3[8:12, 8:12, 8:12] = 0
    c3 = t3.copy()
    c3[8:12, 8:12, 8:12] = 1
    out.append(("cube_cold_mask", t3, {"mask": body}, {"filled": c3}))
    tc = torso_crop()
    rng = np.random.default_rng(9)
    blur = ndi.gaussian_filter(tc.astype(np.float64), 1.2)
    out.append(("torso_crop", tc, {}, {
        "blurred": blur,
        "blurred_noisy": np.maximum(blur + rng.normal(0, 0.05, tc.shape), 0.0),
        "sharpened": np.maximum(tc + 0.5 * (tc - blur), 0.0),
    }))
    return out
