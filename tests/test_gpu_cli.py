"""The `prc` executable end to end on a B200 (tests/test_solver.py:141-361 run through the CLI):
outputs match the reference executable's, and the failure paths behave like prc.cu's."""
import subprocess
import tempfile
from pathlib import Path

import numpy as np
import pytest

from conftest import rel_l2
from prc_mlem_b200 import CLI_PATH

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def workdir(fixture72):
    with tempfile.TemporaryDirectory(prefix="prc_cli_") as d:
        d = Path(d)
        rho, x, y, shape, sp = fixture72
        rho.tofile(d / "density.raw")
        x.tofile(d / "x.raw")
        y.tofile(d / "y.raw")
        yield d


def run(workdir, image, mode, *options, out="out.raw"):
    cmd = [str(CLI_PATH), "68Ga", "16", "14", "12", "1.1", "1.6", "2.3", "--input", str(workdir / image),
           "--density", str(workdir / "density.raw"), "--output", str(workdir / out), "--mode", mode,
           "--rays", "32", *options]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    return np.fromfile(workdir / out, np.float32).reshape(12, 14, 16)


@pytest.mark.parametrize("extra", [(), ("--cache", "source"), ("--cache", "near"), ("--no-cache-near",)],
                         ids=["full", "source", "near", "none"])
def test_cli_matches_reference_binary(workdir, ref_golden, extra):
    assert rel_l2(run(workdir, "x.raw", "forward", *extra), ref_golden["fixture_fwd_68Ga"]) < 1e-5
    assert rel_l2(run(workdir, "y.raw", "adjoint", *extra), ref_golden["fixture_adj_68Ga"]) < 1e-5
    out = run(workdir, "x.raw", "correct", "--iterations", "3", "--beta", "0.1", *extra)
    assert rel_l2(out, ref_golden["fixture_em_b0.1_it3"]) < 1e-5


def test_cli_bf16_weights(workdir, ref_golden):
    out = run(workdir, "x.raw", "correct", "--iterations", "6", "--beta", "0.03", "--bf16-weights")
    assert rel_l2(out, ref_golden["fixture_em_b0.03_it6"]) < 1e-2


def test_buffered_output_write_failure_is_reported(tmp_path):
    if not Path("/dev/full").exists():
        pytest.skip("/dev/full is unavailable")
    np.ones(8, np.float32).tofile(tmp_path / "in.raw")
    np.ones(8, np.float32).tofile(tmp_path / "rho.raw")
    r = subprocess.run([str(CLI_PATH), "68Ga", "2", "2", "2", "1", "1", "1", "--mode", "forward", "--input",
                        str(tmp_path / "in.raw"), "--density", str(tmp_path / "rho.raw"), "--output", "/dev/full",
                        "--rays", "32"], capture_output=True, text=True, timeout=120)
    assert r.returncode != 0
    assert "Cannot write /dev/full" in r.stderr


def test_overflowing_update_fails_without_writing_output(tmp_path):
    np.full(8, 1e20, np.float32).tofile(tmp_path / "in.raw")
    np.ones(8, np.float32).tofile(tmp_path / "rho.raw")
    out = tmp_path / "out.raw"
    r = subprocess.run([str(CLI_PATH), "68Ga", "2", "2", "2", "1", "1", "1", "--input", str(tmp_path / "in.raw"),
                        "--density", str(tmp_path / "rho.raw"), "--output", str(out), "--iterations", "1",
                        "--no-accel", "--rays", "32"], capture_output=True, text=True, timeout=120)
    assert r.returncode != 0
    assert "Non-finite output" in r.stderr
    assert not out.exists()


def test_checkpoint_and_reprojection_names_in_dotted_directory(workdir, fixture72):
    rho, x, y, shape, sp = fixture72
    dotted = workdir / "dir.with.dots"
    dotted.mkdir()
    cmd = [str(CLI_PATH), "68Ga", "16", "14", "12", "1.1", "1.6", "2.3", "--input", str(workdir / "x.raw"),
           "--density", str(workdir / "density.raw"), "--output", str(dotted / "output"), "--rays", "32",
           "--iterations", "3", "--save-every", "1", "--reproject"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    for name in ["output", "output_it001", "output_it002", "output_REPROJ"]:
        assert (dotted / name).stat().st_size == x.nbytes
    final = np.fromfile(dotted / "output", np.float32).reshape(shape)
    reproj = np.fromfile(dotted / "output_REPROJ", np.float32)
    assert abs(reproj.sum(dtype=np.float64) / final.sum(dtype=np.float64) - 1) < 3e-6


def test_checkpoint_write_failure_stops_the_run(workdir):
    """--save-every writes checkpoints from a helper thread while the GPU iterates; a failed
    checkpoint write still ends the run with the reference's message and no final output."""
    missing = workdir / "no_such_dir" / "output"
    cmd = [str(CLI_PATH), "68Ga", "16", "14", "12", "1.1", "1.6", "2.3", "--input", str(workdir / "x.raw"),
           "--density", str(workdir / "density.raw"), "--output", str(missing), "--rays", "32",
           "--iterations", "3", "--save-every", "1"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=120)
    assert r.returncode != 0
    assert r.stderr.count("Cannot write") == 1 and "output_it001" in r.stderr
    assert not missing.exists()
