"""The fixed byte accounting bench.py reports its rooflines against."""
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

import bench  # noqa: E402

# 128x128x159 68Ga torso: voxels, tissue sources and deposits per projection counted on the device
N, N_ACTIVE, V = 128 * 128 * 159, 1_098_372, 2_271_204_018


def test_projection_bytes_match_the_fp32_line():
    acct = bench.algorithmic_bytes(N, N_ACTIVE, V)
    assert acct["projection"] == 18_182_812_608  # 12 B per source + 8 B per deposit


def test_iteration_adds_the_elementwise_chain_to_two_projections():
    acct = bench.algorithmic_bytes(N, N_ACTIVE, V)
    assert acct["iteration"] == 74 * N + 2 * acct["projection"]
    assert 36e9 < acct["iteration"] < 37e9


def test_bf16_counts_the_stored_dtype():
    fp32 = bench.algorithmic_bytes(N, N_ACTIVE, V, weight_bytes=4)
    bf16 = bench.algorithmic_bytes(N, N_ACTIVE, V, weight_bytes=2)
    assert fp32["projection"] - bf16["projection"] == 2 * V
    assert bf16["compulsory"] == fp32["compulsory"]


def test_compulsory_figure_is_about_a_fifth_of_a_gigabyte():
    acct = bench.algorithmic_bytes(N, N_ACTIVE, V)
    assert acct["compulsory"] == 74 * N + 24 * N_ACTIVE
    assert 0.2e9 < acct["compulsory"] < 0.25e9


def test_empty_volume():
    assert bench.algorithmic_bytes(0, 0, 0) == {"projection": 0, "iteration": 0, "compulsory": 0}


def test_reference_quadrature_leg_times_the_restated_cpu_path():
    q = bench.reference_quadrature(repeats=1)
    assert q["seconds"] > 0 and q["cores"] == 1 and q["kind"] == "port"
    assert "68Ga" in q["case"] and "half-width 6" in q["case"]


def test_small_configuration_fp64_runs_the_three_modes():
    r = bench.small_configuration_fp64(2)
    assert r["seconds"] > 0 and r["cores"] == 2 and r["kind"] == "port"
    assert "32x32x24" in r["case"] and "4 RL iterations" in r["case"]


def test_reference_arm_samples_are_bounded():
    """1-8 s of projection time per step, shared so that the default 63 runs stay short."""
    for runs in (1, 5, 13, 63, 1000):
        per = max(1.0, min(8.0, bench.REFERENCE_ARM_SECONDS / runs))
        assert 1.0 <= per <= 8.0
        assert runs * per <= max(bench.REFERENCE_ARM_SECONDS, runs * 1.0)
