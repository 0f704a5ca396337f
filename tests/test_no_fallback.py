"""The product path has no CPU fallback: without its shared library, or without a CUDA device,
the Python binding raises instead of computing anything on the host."""
import numpy as np
import pytest
import torch

import prc_mlem_b200 as pm


def test_missing_library_raises(monkeypatch, tmp_path):
    monkeypatch.setattr(pm, "LIB_PATH", tmp_path / "libprc_b200.so")
    monkeypatch.setattr(pm, "_lib_handle", None)
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        pm.lib()
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        pm.Projector("18F", np.ones((4, 4, 4), np.float32), (2.0, 2.0, 2.0))


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the behaviour without a CUDA device")
def test_without_a_device_the_projector_reports_an_error():
    with pytest.raises(pm.PrcError):
        pm.Projector("18F", np.ones((4, 4, 4), np.float32), (2.0, 2.0, 2.0))


def test_host_side_validation_runs_before_any_device_call():
    with pytest.raises(ValueError):
        pm.Projector("18F", np.ones((4, 4), np.float32), (2.0, 2.0, 2.0))
