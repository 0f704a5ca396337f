"""Golden metric values from the reference's own scorer, tools/evaluate.py.

Run with the reference checkout as the argument or in PRC_REFERENCE_DIR:
    python tests/golden/make_metrics_golden.py path/to/PRC_MLEM
It imports the reference's Evaluator with scikit-image replaced by a stand-in SSIM (the
oracle's restatement; scikit-image is not installed here), runs every case of
metrics_cases.py and writes tests/golden/metrics_golden.json.  The non-SSIM metrics pin the
oracle to the reference's code; the SSIM entries only record the stand-in.
"""
import json
import os
import sys
import types
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(HERE))
from oracle.metrics_oracle import ssim_map  # noqa: E402
import metrics_cases  # noqa: E402


def structural_similarity(im1, im2, data_range=None, gaussian_weights=False, sigma=1.5,
                          use_sample_covariance=True, full=False):
    assert gaussian_weights and sigma == 1.5 and not use_sample_covariance
    s, pad = ssim_map(im1, im2, data_range)
    mssim = float(s[(slice(pad, -pad),) * 3].mean())
    return (mssim, s) if full else mssim


def main():
    skimage = types.ModuleType("skimage")
    metrics = types.ModuleType("skimage.metrics")
    metrics.structural_similarity = structural_similarity
    skimage.metrics = metrics
    sys.modules["skimage"], sys.modules["skimage.metrics"] = skimage, metrics
    ref_dir = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PRC_REFERENCE_DIR")
    if not ref_dir:
        raise SystemExit("give the reference checkout as the argument or in PRC_REFERENCE_DIR")
    sys.path.insert(0, str(Path(ref_dir) / "tools"))
    import evaluate as ref  # the reference's tools/evaluate.py
    golden = {}
    for name, truth, kw, candidates in metrics_cases.cases():
        ev = ref.Evaluator(truth, **kw)
        golden[name] = {"settings": ev.metric_settings,
                        "metrics": {c: ev(f) for c, f in candidates.items()}}
    (HERE / "metrics_golden.json").write_text(json.dumps(golden, indent=1, allow_nan=False))
    print("wrote", HERE / "metrics_golden.json")


if __name__ == "__main__":
    main()
