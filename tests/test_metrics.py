"""Image-quality metrics: the CPU oracle pinned to the reference's scorer (tools/evaluate.py,
run on the seeded cases of tests/golden/metrics_cases.py by make_metrics_golden.py), and the
host side of the device evaluator (raw loading, table, argument validation) -- no GPU needed."""
import json
import math
import sys
import tempfile
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "tests" / "golden"))
import metrics_cases  # noqa: E402
from oracle import metrics_oracle  # noqa: E402
from prc_mlem_b200 import evaluate  # noqa: E402

GOLDEN = json.loads((ROOT / "tests" / "golden" / "metrics_golden.json").read_text())
TOL = 1e-12


def close(a, b, tol=TOL):
    if a is None or b is None:
        return a is None and b is None
    return math.isclose(a, b, rel_tol=tol, abs_tol=tol)


@pytest.mark.parametrize("case", [c[0] for c in metrics_cases.cases()])
def test_oracle_matches_reference_scorer(case):
    name, truth, kw, candidates = next(c for c in metrics_cases.cases() if c[0] == case)
    ev = metrics_oracle.Evaluator(truth, **kw)
    assert ev.n_hot == GOLDEN[name]["settings"]["hot_region_count"]
    for cname, f in candidates.items():
        got, want = ev(f), GOLDEN[name]["metrics"][cname]
        assert set(got) == set(want)
        for key in want:
            assert close(got[key], want[key]), (cname, key, got[key], want[key])


def test_oracle_identity_is_exact():
    t = metrics_cases.cube_phantom()
    m = metrics_oracle.Evaluator(t)(t)
    for key in ("nrmse", "nrmse_tissue", "mse", "edge_nrmse", "ring", "bg_bias", "bg_cov", "halo", "count_bias"):
        assert m[key] == 0, key
    for key in ("ssim", "ssim_tissue", "ssim_edge", "rc_hot", "rc_min"):
        assert abs(m[key] - 1) < 1e-12, key


def test_raw_size_is_checked():
    with tempfile.TemporaryDirectory() as tmp:
        path = Path(tmp) / "bad.raw"
        np.zeros(7, dtype=np.float32).tofile(path)
        with pytest.raises(ValueError, match="expected 32 bytes, got 28"):
            evaluate.load(path, (2, 2, 2))
        path.write_bytes(np.ones(8, dtype=np.float32).tobytes() + b"x")
        with pytest.raises(ValueError, match="expected 32 bytes, got 33"):
            evaluate.load(path, (2, 2, 2))
        with pytest.raises(ValueError, match="three positive"):
            evaluate.load(path, (2, 2))


def test_table_marks_missing_scores():
    metric = dict.fromkeys(evaluate.COLUMNS, None)
    metric["nrmse"] = 0.5
    table = evaluate.format_table([("x", metric)])
    assert "| x | 0.5000 | —" in table and table.count("—") == len(evaluate.COLUMNS) - 1


def test_invalid_truth_and_masks_are_rejected_before_the_device():
    truth = metrics_cases.cube_phantom()
    bad = truth.copy()
    bad[0, 0, 0] = np.nan
    for value in (bad, -truth, np.zeros_like(truth), np.ones((3, 3))):
        with pytest.raises(ValueError):
            evaluate.Evaluator(value)
    for kwargs in ({"data_range": 0}, {"data_range": np.nan}, {"background": -1},
                   {"mask": np.zeros_like(truth)}, {"mask": np.ones((3, 3, 3))}):
        with pytest.raises(ValueError):
            evaluate.Evaluator(truth, **kwargs)
    lesions = truth == 4
    stray = lesions.copy()
    stray[0, 0, 0] = True
    with pytest.raises(ValueError, match="inside tissue"):
        evaluate.Evaluator(truth, hot_mask=stray)
    with pytest.raises(ValueError, match="truth shape"):
        evaluate.Evaluator(truth, hot_mask=lesions[:, :, :-1])
