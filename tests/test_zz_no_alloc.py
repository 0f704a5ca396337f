"""prc_sum_static: the FP64 volume sum for callers that cannot allocate device memory where
they need it (services that reserve all GPU memory at start-up, hot paths that must not pay
cudaMalloc's synchronisation, operators inside another framework's allocator).  It keeps its
scratch in a static device array, so this test checks, through the C ABI, that the calls after
the first one on a device leave free device memory unchanged (the first may load the array's
module under CUDA's lazy loading), that two calls in a row agree with the handle-based prc_sum
on the same data, that the size limit is enforced, and that an empty input gives zero.  This
file is collected last, so a run that stops at the first failure has already run every other
test."""
import ctypes

import numpy as np
import pytest
import torch

import prc_mlem_b200 as pm

pytestmark = pytest.mark.gpu
REL_TOL = 1e-12  # both sums accumulate in FP64; only the order of additions differs


def static_sum(d_x, n=None):
    out = torch.full((1,), -1.0, dtype=torch.float64, device=d_x.device)
    rc = pm.lib().prc_sum_static(d_x.data_ptr(), d_x.numel() if n is None else n, out.data_ptr(), None)
    assert rc == pm.PRC_OK, pm.lib().prc_last_error().decode()
    torch.cuda.synchronize()
    return float(out.item())


def test_calls_after_the_first_allocate_no_device_memory(record_property):
    x = torch.rand(1 << 20, dtype=torch.float32, device="cuda")
    out = torch.zeros(4, dtype=torch.float64, device="cuda")  # every buffer exists before measuring
    expect = x.double().sum().item()
    torch.cuda.synchronize()

    def call():
        rc = pm.lib().prc_sum_static(x.data_ptr(), x.numel(), out.data_ptr(), None)
        assert rc == pm.PRC_OK, pm.lib().prc_last_error().decode()
        torch.cuda.synchronize()

    free0, _ = torch.cuda.mem_get_info()
    call()  # warm-up: under lazy module loading this is what loads the static array
    free1, _ = torch.cuda.mem_get_info()
    record_property("first_call_device_bytes", free0 - free1)
    assert free0 - free1 <= 16 << 20  # at most the module image, never a volume-sized buffer
    for _ in range(8):
        call()
    free2, _ = torch.cuda.mem_get_info()
    assert free2 == free1, f"later calls changed free device memory by {free1 - free2} bytes"
    assert abs(out[0].item() - expect) <= 1e-9 * expect


def test_two_calls_in_a_row_match_prc_sum():
    rng = np.random.default_rng(5)
    shape = (40, 36, 34)
    rho = np.where(rng.random(shape) < 0.8, 1.0, 0.001).astype(np.float32)
    with pm.Projector("18F", rho, (2.0, 2.0, 2.0), rays=2, cache=pm.PRC_CACHE_NONE) as P:
        for seed in (1, 2):  # the second call reuses the array the first one left behind
            x = np.random.default_rng(seed).uniform(0.0, 5.0, shape).astype(np.float32)
            d_x = torch.from_numpy(x).cuda()
            expect = P.sum(d_x)
            got = static_sum(d_x)
            assert abs(got - expect) <= REL_TOL * abs(expect)
            assert abs(got - x.sum(dtype=np.float64)) <= 1e-9 * abs(expect)


def test_large_volume_uses_many_blocks():
    n = 128 * 128 * 159
    x = torch.rand(n, dtype=torch.float32, device="cuda")
    expect = x.double().sum().item()
    for _ in range(2):
        assert abs(static_sum(x) - expect) <= 1e-9 * expect


def test_limit_and_empty_input():
    x = torch.ones(16, dtype=torch.float32, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = pm.lib().prc_sum_static(x.data_ptr(), (1 << 28) + 1, out.data_ptr(), None)
    assert rc == 8  # PRC_ERR_LIMIT, rejected before any work is enqueued
    assert b"static scratch limit" in pm.lib().prc_last_error()
    assert static_sum(x, n=0) == 0.0
    assert pm.lib().prc_sum_static(None, 4, out.data_ptr(), None) == 1
