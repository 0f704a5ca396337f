"""Device image-quality metrics (prc_eval_* through prc_mlem_b200.evaluate) against the CPU
oracle, and the behaviour the reference's tests/test_metrics.py asks of its scorer."""
import json
import math
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np
import pytest
import torch
from scipy import ndimage as ndi

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "tests" / "golden"))
import metrics_cases  # noqa: E402
from oracle import metrics_oracle  # noqa: E402
from prc_mlem_b200 import evaluate, phantoms  # noqa: E402

pytestmark = pytest.mark.gpu
TOL = 1e-9  # FP64 sums in a different order than NumPy's


def same(a, b, tol=TOL):
    assert set(a) == set(b)
    for k in b:
        if b[k] is None or a[k] is None:
            assert a[k] is None and b[k] is None, k
        else:
            assert math.isclose(a[k], b[k], rel_tol=tol, abs_tol=tol), (k, a[k], b[k])


@pytest.mark.parametrize("case", [c[0] for c in metrics_cases.cases()])
def test_device_matches_oracle(case):
    name, truth, kw, candidates = next(c for c in metrics_cases.cases() if c[0] == case)
    dev, ref = evaluate.Evaluator(truth, **kw), metrics_oracle.Evaluator(truth, **kw)
    for f in candidates.values():
        same(dev(f), ref(f))
        same(dev(torch.from_numpy(np.asarray(f, np.float64)).cuda()), ref(f))


def test_clinical_volume_matches_oracle():
    rho, truth, sp = phantoms.torso_phantom()
    blur = ndi.gaussian_filter(truth, 1.5).astype(np.float32)
    dev, ref = evaluate.Evaluator(truth), metrics_oracle.Evaluator(truth)
    got = dev(torch.from_numpy(blur).cuda())
    same(got, ref(blur))
    assert got["rc_hot"] < 1 and got["ssim"] < 1


def test_identity_and_strict_json():
    truth = metrics_cases.cube_phantom()
    m = evaluate.Evaluator(truth)(truth)
    for key in ("nrmse", "nrmse_tissue", "mse", "mae_tissue", "edge_nrmse", "ring", "overshoot",
                "undershoot", "bg_bias", "bg_cov", "halo", "count_bias"):
        assert m[key] == 0, key
    for key in ("ssim", "ssim_tissue", "ssim_edge", "rc_hot", "rc_min"):
        assert abs(m[key] - 1) < 1e-12, key
    assert m["psnr"] is None
    json.dumps(m, allow_nan=False)


def test_blur_and_local_range_violations_are_distinct():
    truth = metrics_cases.cube_phantom()
    ev = evaluate.Evaluator(truth)
    blur = ev(ndi.uniform_filter(truth, size=3))
    assert blur["edge_nrmse"] > 0.05 and blur["ring"] < 1e-7
    ring = truth.copy()
    ring[13:15, 13:22, 13:22] += 0.5
    ring[11:13, 13:22, 13:22] = -0.2
    m = ev(ring)
    assert m["overshoot"] > 0 and m["undershoot"] > 0
    assert abs(m["ring"] ** 2 - (m["overshoot"] ** 2 + m["undershoot"] ** 2)) < 1e-12


def test_scale_invariant_scores():
    truth = metrics_cases.cube_phantom()
    candidate = ndi.gaussian_filter(truth, 0.8)
    a = evaluate.Evaluator(truth)(candidate)
    for scale in (1e-4, 20, 1e4):
        b = evaluate.Evaluator(truth.astype(np.float64) * scale)(candidate.astype(np.float64) * scale)
        for key in ("nrmse", "ssim", "ssim_tissue", "ssim_edge", "ring", "halo", "edge_nrmse", "bg_bias",
                    "bg_cov", "rc_hot", "rc_min"):
            assert math.isclose(a[key], b[key], abs_tol=1e-9), (scale, key)


def test_missing_scores_and_small_volumes():
    flat = np.ones((15, 15, 15), dtype=np.float32)
    m = evaluate.Evaluator(flat)(flat)
    for key in ("rc_hot", "rc_min", "ring", "halo", "edge_nrmse", "ssim_edge"):
        assert m[key] is None, key
    assert m["ssim"] == 1
    assert "—" in evaluate.format_table([("constant", m)])
    thin = np.ones((5, 15, 15), dtype=np.float32)
    m = evaluate.Evaluator(thin)(thin)
    assert m["ssim"] is None and m["nrmse"] == 0


def test_mask_and_hot_mask():
    truth = metrics_cases.cube_phantom()
    body = truth > 0
    cold = truth.copy()
    cold[8:12, 8:12, 8:12] = 0
    filled = cold.copy()
    filled[8:12, 8:12, 8:12] = 1
    assert evaluate.Evaluator(cold)(filled)["nrmse_tissue"] == 0
    assert evaluate.Evaluator(cold, mask=body)(filled)["nrmse_tissue"] > 0
    lesions = truth == 4
    bright = truth.copy()
    bright[5:9, 5:9, 5:9] = 2
    dim = bright.copy()
    dim[5:9, 5:9, 5:9] = 1
    threshold = evaluate.Evaluator(bright, background=1)
    explicit = evaluate.Evaluator(bright, background=1, hot_mask=lesions)
    assert threshold(dim)["rc_hot"] < 1
    assert explicit(dim)["rc_hot"] == 1 and explicit(dim)["rc_min"] == 1
    assert explicit.metric_settings["hot_region_count"] == 1 and threshold.metric_settings["hot_region_count"] == 2


def test_invalid_reconstructions_are_rejected():
    truth = metrics_cases.cube_phantom()
    ev = evaluate.Evaluator(truth)
    bad = truth.copy()
    bad[0, 0, 0] = np.nan
    for value in (bad, truth[:, :, :-1], torch.from_numpy(bad).cuda()):
        with pytest.raises(ValueError):
            ev(value)
    assert ev(truth)["nrmse"] == 0  # the evaluator stays usable


def test_cli_writes_flat_json():
    with tempfile.TemporaryDirectory() as tmp:
        data = Path(tmp)
        truth = metrics_cases.cube_phantom()
        truth.tofile(data / "truth.raw")
        (truth > 1.5).astype(np.float32).tofile(data / "hot.raw")
        proc = subprocess.run([sys.executable, "-m", "prc_mlem_b200.evaluate", "--truth", str(data / "truth.raw"),
                               "--shape", "35", "35", "35", "--hot-mask", str(data / "hot.raw"), "--background", "1",
                               "--json", str(data / "metrics.json"), f"identity={data / 'truth.raw'}"],
                              capture_output=True, text=True, cwd=ROOT)
        assert proc.returncode == 0, proc.stderr
        report = json.loads((data / "metrics.json").read_text())
        assert set(report) == {"identity"} and report["identity"]["rc_hot"] == 1
        assert "explicit hot mask" in proc.stdout
