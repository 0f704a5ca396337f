"""Command-line contract of `prc` without a GPU: the reference's CommandLineTests
(tests/test_solver.py:25-124) run against this engine's executable with every GPU hidden.
Validation must reject bad input before the first CUDA call."""
import os
import struct
import subprocess
import tempfile
from pathlib import Path

import pytest

from prc_mlem_b200 import CLI_PATH


def write_raw(path, values):
    path.write_bytes(struct.pack(f"={len(values)}f", *values))


@pytest.fixture
def files():
    with tempfile.TemporaryDirectory() as d:
        d = Path(d)
        density, image, output = d / "density.raw", d / "input.raw", d / "output.raw"
        write_raw(density, [1.0] * 8)
        write_raw(image, [0.0] * 8)
        yield density, image, output


def run_prc(files, *options, geometry=None):
    density, image, output = files
    args = geometry or ["68Ga", "2", "2", "2", "1", "1", "1"]
    return subprocess.run([str(CLI_PATH), *args, "--density", str(density), "--input", str(image),
                           "--output", str(output), *options],
                          env={**os.environ, "CUDA_VISIBLE_DEVICES": ""}, text=True, capture_output=True, timeout=30)


def assert_rejected(result, message, files):
    assert result.returncode != 0, result.stdout
    assert message in result.stderr
    assert "CUDA error" not in result.stderr
    assert not files[2].exists()


def test_binary_exists():
    assert CLI_PATH.is_file(), "build with make -C prc_mlem_b200/csrc"


@pytest.mark.parametrize("option", ["--help", "-h"])
def test_help_succeeds_without_gpu(option):
    r = subprocess.run([str(CLI_PATH), option], env={**os.environ, "CUDA_VISIBLE_DEVICES": ""},
                       text=True, capture_output=True, timeout=30)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "Usage:" in r.stdout
    assert r.stderr == ""
    for iso in ("11C", "13N", "15O", "18F", "64Cu", "68Ga", "82Rb", "124I"):
        assert iso in r.stdout


@pytest.mark.parametrize("option,value", [
    ("--beta", "garbage"), ("--beta", "nan"), ("--gamma", "inf"), ("--rays", "128x"), ("--rays", "2147483648"),
    ("--iterations", "2.5"), ("--beta", "1e999")])
def test_invalid_numeric_options(files, option, value):
    assert_rejected(run_prc(files, option, value), "Invalid", files)


@pytest.mark.parametrize("option,value", [
    ("--support-rho", "-1"), ("--air-cap-mm", "0"), ("--save-every", "-1"), ("--iterations", "2147483647"),
    ("--rays", "2147483647"), ("--rays", "1"), ("--rays", "3"), ("--rays", "129"), ("--mode", "sideways"),
    ("--cache", "sometimes")])
def test_invalid_bounds(files, option, value):
    assert_rejected(run_prc(files, option, value), "Invalid", files)


@pytest.mark.parametrize("geometry", [
    ["68Ga", "2x", "2", "2", "1", "1", "1"], ["68Ga", "2", "2", "2", "nan", "1", "1"],
    ["68Ga", "0", "2", "2", "1", "1", "1"], ["68Ga", "2", "2", "2", "1", "-1", "1"]])
def test_invalid_geometry(files, geometry):
    assert_rejected(run_prc(files, geometry=geometry), "Invalid", files)


def test_index_overflow(files):
    assert_rejected(run_prc(files, geometry=["68Ga", "65536", "65536", "1", "1", "1", "1"]), "INT_MAX", files)


@pytest.mark.parametrize("size", [7, 9])
def test_raw_size_must_match_exactly(files, size):
    write_raw(files[1], [0.0] * size)
    assert_rejected(run_prc(files), "Expected exactly", files)


def test_raw_size_odd_bytes(files):
    files[1].write_bytes(b"\x00" * 33)
    assert_rejected(run_prc(files), "Expected exactly", files)


def test_missing_file(files):
    files[0].unlink()
    assert_rejected(run_prc(files), "Expected exactly", files)


@pytest.mark.parametrize("which", [0, 1])
@pytest.mark.parametrize("value", [float("nan"), float("inf"), float("-inf")])
def test_nonfinite_raw_values(files, which, value):
    write_raw(files[1], [1.0] * 8)
    write_raw(files[which], [value] + [1.0] * 7)
    assert_rejected(run_prc(files), "Non-finite", files)


@pytest.mark.parametrize("mode", ["correct", "forward", "adjoint"])
def test_zero_activity_is_rejected_without_gpu(files, mode):
    assert_rejected(run_prc(files, "--mode", mode), "No activity", files)


def test_empty_support_is_rejected_without_gpu(files):
    write_raw(files[0], [0.0] * 8)
    write_raw(files[1], [3.0] * 8)
    assert_rejected(run_prc(files), "No activity", files)


def test_unknown_option_and_missing_value(files):
    r = run_prc(files, "--frobnicate")
    assert_rejected(r, "Unknown option", files)
    assert "Usage:" in r.stderr
    assert_rejected(run_prc(files, "--beta"), "Missing value", files)


def test_unknown_isotope(files):
    r = run_prc(files, geometry=["99Zz", "2", "2", "2", "1", "1", "1"])
    assert r.returncode != 0
    assert "Usage:" in r.stderr
    assert not files[2].exists()


def test_too_few_arguments():
    r = subprocess.run([str(CLI_PATH), "68Ga", "2"], env={**os.environ, "CUDA_VISIBLE_DEVICES": ""},
                       text=True, capture_output=True, timeout=30)
    assert r.returncode != 0
    assert "Usage:" in r.stderr
