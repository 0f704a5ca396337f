"""bench.py keeps its contract: one JSON line per arm with the keys the measurement needs, on a
small torso (48 x 64 x 64) so that the run takes seconds."""
import json
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]
SMALL = ["--grid", "48", "64", "64", "--steps", "3", "--warmup", "3"]


def run(*args):
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), *SMALL, *args], capture_output=True, text=True,
                       timeout=900, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    return json.loads(lines[0])


_lines = {}


def ours():
    if "ours" not in _lines:
        _lines["ours"] = run("--no-forms", "--no-oracle-check", "--no-batch")
    return _lines["ours"]


def test_our_arm_line():
    d = ours()
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
                "vs_baseline", "dtype", "data", "config", "e2e", "roofline", "cpu_baseline", "gpu_launches", "clocks"):
        assert key in d, key
    assert d["n_gpus"] == 1 and d["steps"] == 3 and d["warmup"] == 3 and d["value"] > 0
    assert "workload" in d["config"]
    assert set(d["e2e"]) >= {"value", "unit", "h2d_bytes_per_step", "d2h_bytes_per_step"}
    assert d["e2e"]["h2d_bytes_per_step"] == d["e2e"]["d2h_bytes_per_step"] == 48 * 64 * 64 * 4
    r = d["roofline"]
    assert r["bound"] == "hbm" and r["unit"] == "GB/s" and r["achieved"] > 0 and r["peak"] > 0
    assert abs(r["frac"] - r["achieved"] / r["peak"]) < 1e-3
    assert r["launches_timed"] == 2 * 3 * 6
    it = r["iteration"]
    assert it["algorithmic_bytes"] == 74 * 48 * 64 * 64 + 2 * r["algorithmic_bytes"]
    assert 0 < it["compulsory_bytes"] < it["algorithmic_bytes"] and 0 < it["achieved"]
    assert abs(it["frac"] - it["achieved"] / r["peak"]) < 1e-3
    c = d["cpu_baseline"]
    assert c["kind"] == "port" and c["cores"] >= 1 and c["value"] > 0 and c["sample"]
    assert c["reference_quadrature"]["seconds"] > 0 and c["reference_quadrature"]["cores"] == 1
    assert c["small_configuration_fp64"]["seconds"] > 0
    # projections, ratio, update and finish per iteration, plus the initialisation, per step
    assert d["gpu_launches"] >= 3 * (3 + 5 * 6)
    assert r["dram_frac"] is None or 0 < r["dram_frac"] < 1.5
    assert d["details"]["n_active"] > 0
    assert {"sm_mhz", "sm_max_mhz", "reasons"} <= set(d["clocks"])
    assert d["image_quality"]["corrected"]["nrmse"] < d["image_quality"]["measured"]["nrmse"]


def test_our_arm_parity_and_time_to_image():
    from oracle import ref_exe
    d = ours()
    if not ref_exe.available():
        pytest.skip("oracle/_ref/prc not built")
    p = d["parity_vs_prc_cu"]
    assert p["forward_fp32_field"] < 1e-5 and p["adjoint_fp32_field"] < 1e-5
    assert p["corrected"]["fp32_field"] < 1e-5
    t = d["time_to_image"]
    assert t["fp32_field"]["seconds"] > 0 and t["prc_cu"]["seconds"] > 0


def test_reference_arm_line():
    d = run("--impl", "reference", "--steps", "3", "--warmup", "3")
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "EM iters/s"
    assert d["cpu_baseline"]["value"] == d["value"] and d["cpu_baseline"]["kind"] == "port"
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["config"] == ours()["config"]  # both arms name the same workload
    assert d["cpu_baseline"]["setup_s"] > 0
    from oracle import ref_exe
    if ref_exe.available():
        assert d["data"] == ours()["data"]  # the same recipe: prc.cu's blur, the counter-based sampler
        assert d["reference_gpu"]["value"] > 0 and d["reference_gpu"]["job"]["seconds"] > 0
