"""Projector parity on a B200: the CUDA engine against the reference executable's own outputs
(tests/golden/ref_outputs.npz, prc.cu built for sm_100a) and the FP64 CPU oracle, in every
cache mode and weight precision.  fp32 and 24-bit-weight forms must match the reference within
1e-5 relative L2; bf16-stored weights within 2e-3.  The adjoint identity and count conservation hold to 3e-6
(tests/test_solver.py:180-214)."""
import numpy as np
import pytest
import torch

import prc_mlem_b200 as pm
from conftest import GOLDEN, rel_l2

pytestmark = pytest.mark.gpu
ISOTOPES = ("11C", "13N", "15O", "18F", "64Cu", "68Ga", "82Rb", "124I")
MODES = [(pm.PRC_CACHE_FULL, pm.PRC_PRECISION_FP32), (pm.PRC_CACHE_SOURCE_MAJOR, pm.PRC_PRECISION_FP32),
         (pm.PRC_CACHE_NEAR, pm.PRC_PRECISION_FP32), (pm.PRC_CACHE_NONE, pm.PRC_PRECISION_FP32),
         (pm.PRC_CACHE_FULL, pm.PRC_PRECISION_BF16), (pm.PRC_CACHE_SOURCE_MAJOR, pm.PRC_PRECISION_BF16),
         (pm.PRC_CACHE_NEAR, pm.PRC_PRECISION_BF16), (pm.PRC_CACHE_FULL, pm.PRC_PRECISION_FP24),
         (pm.PRC_CACHE_SOURCE_MAJOR, pm.PRC_PRECISION_FP24)]
MODE_IDS = ["full-fp32", "source-fp32", "near-fp32", "none-fp32", "full-bf16", "source-bf16", "near-bf16",
            "full-fp24", "source-fp24"]


def tol(prec):
    """fp32 and the 24-bit field (weights within 2^-17 relative) at the reference's 1e-5."""
    return 1e-5 if prec in (pm.PRC_PRECISION_FP32, pm.PRC_PRECISION_FP24) else 2e-3


_cache = {}


def projector(fixture72, iso="68Ga", cache=pm.PRC_CACHE_FULL, prec=pm.PRC_PRECISION_FP32, rays=32, exact=False):
    key = (iso, cache, prec, rays, exact)
    if key not in _cache:
        rho, x, y, shape, sp = fixture72
        _cache[key] = pm.Projector(iso, rho, sp, rays=rays, cache=cache, precision=prec, exact_range=exact)
    return _cache[key]


@pytest.mark.parametrize("iso", ISOTOPES)
def test_forward_adjoint_match_reference_binary(fixture72, ref_golden, oracle_mod, iso):
    rho, x, y, shape, sp = fixture72
    P = projector(fixture72, iso)
    mode, source_entries, target_entries = P.cache_mode
    assert mode == pm.PRC_CACHE_FULL and source_entries > 0 and target_entries > 0
    ax, aty = P.forward_host(x), P.adjoint_host(y)
    assert rel_l2(ax, ref_golden[f"fixture_fwd_{iso}"]) < 1e-5
    assert rel_l2(aty, ref_golden[f"fixture_adj_{iso}"]) < 1e-5
    O = oracle_mod.Problem(iso, rho, sp, rays=32, precision=64).normalize()
    assert rel_l2(ax, O.forward(x)) < 1e-5  # error against the FP64 oracle
    assert rel_l2(aty, O.adjoint(y)) < 1e-5


@pytest.mark.parametrize("mode", MODES, ids=MODE_IDS)
def test_cache_modes_match_reference_binary(fixture72, ref_golden, mode):
    rho, x, y, shape, sp = fixture72
    P = projector(fixture72, "68Ga", *mode)
    assert P.cache_mode[0] == mode[0]  # no fall-back at this size
    assert rel_l2(P.forward_host(x), ref_golden["fixture_fwd_68Ga"]) < tol(mode[1])
    assert rel_l2(P.adjoint_host(y), ref_golden["fixture_adj_68Ga"]) < tol(mode[1])


@pytest.mark.parametrize("mode", MODES, ids=MODE_IDS)
def test_adjoint_identity_conservation_and_support(fixture72, mode):
    rho, x, y, shape, sp = fixture72
    P = projector(fixture72, "68Ga", *mode)
    ax, aty = P.forward_host(x), P.adjoint_host(y)
    lhs = np.sum(ax.astype(np.float64) * y)
    rhs = np.sum(x.astype(np.float64) * aty)
    assert abs(lhs / rhs - 1) < 3e-6
    assert abs(ax.sum(dtype=np.float64) / x.sum(dtype=np.float64) - 1) < 3e-6
    assert np.all(ax[~P.support] == 0)
    one = P.adjoint_host(np.ones(shape, np.float32))
    np.testing.assert_allclose(one[P.support], 1, rtol=3e-6, atol=3e-6)
    assert np.all(one[~P.support] == 0)


def test_more_rays_and_exact_range(fixture72, ref_golden):
    rho, x, y, shape, sp = fixture72
    assert rel_l2(projector(fixture72, rays=128).forward_host(x), ref_golden["fixture_fwd_128_68Ga"]) < 1e-5
    P = projector(fixture72, exact=True)
    assert rel_l2(P.forward_host(x), ref_golden["fixture_fwd_exact_68Ga"]) < 1e-5
    assert rel_l2(P.adjoint_host(np.ones(shape, np.float32)), ref_golden["fixture_adj_one_68Ga"]) < 1e-5


@pytest.mark.parametrize("iso", ISOTOPES)
def test_range_table_matches_exact(fixture72, iso):
    """tests/test_solver.py:201-214: table and analytic survival agree to rtol 1e-5 / atol 2e-7."""
    rho, x, y, shape, sp = fixture72
    T, E = projector(fixture72, iso), projector(fixture72, iso, exact=True)
    np.testing.assert_allclose(T.forward_host(x), E.forward_host(x), rtol=1e-5, atol=2e-7)
    np.testing.assert_allclose(T.adjoint_host(y), E.adjoint_host(y), rtol=1e-5, atol=2e-7)


@pytest.mark.parametrize("size", [4.0, 2.0])
def test_water_kernel_matches_reference_quadrature(size):
    g = np.load(GOLDEN / "water_kernel.npz")
    half = int(g[f"half_{size:g}mm"])
    exact = g[f"kernel_{size:g}mm"]
    n, c = 2 * half + 5, half + 2
    delta = np.zeros((n, n, n), np.float32)
    delta[c, c, c] = 1
    with pm.Projector("68Ga", np.ones((n, n, n), np.float32), (size,) * 3, rays=128) as P:
        k = P.forward_host(delta)[c - half:c + half + 1, c - half:c + half + 1, c - half:c + half + 1]
    k = k.astype(np.float64)
    blur = exact.copy()
    blur[half, half, half] -= 1
    assert np.linalg.norm(k - exact) / np.linalg.norm(blur) < 0.01
    for axis in np.indices(k.shape) - half:
        assert abs((k * axis).sum()) < 1e-6


def test_deposit_count_matches_oracle(fixture72, oracle_mod):
    rho, x, y, shape, sp = fixture72
    for iso in ("68Ga", "82Rb"):
        O = oracle_mod.Problem(iso, rho, sp, rays=32, precision=32).normalize()
        assert projector(fixture72, iso).count_deposits() == O.count_deposits()


def test_small_phantom_matches_reference_binary(ref_golden):
    from prc_mlem_b200 import phantoms
    rho, truth, sp = phantoms.small_phantom(seed=1)
    with pm.Projector("18F", rho, sp, rays=32) as P:
        assert rel_l2(P.forward_host(truth), ref_golden["small_fwd"]) < 1e-5
        assert rel_l2(P.adjoint_host(truth), ref_golden["small_adj"]) < 1e-5


def test_device_and_host_forms_agree_and_adjoint_leaves_non_tissue(fixture72):
    rho, x, y, shape, sp = fixture72
    P = projector(fixture72)
    d_x = torch.from_numpy(x).cuda()
    d_out = torch.full_like(d_x, 7.0)
    P.forward(d_x, d_out)
    P.synchronize()
    np.testing.assert_allclose(d_out.cpu().numpy(), P.forward_host(x), rtol=1e-6, atol=1e-9)
    d_out.fill_(7.0)
    P.adjoint(torch.from_numpy(y).cuda(), d_out)
    P.synchronize()
    out = d_out.cpu().numpy()
    assert np.all(out[~P.support] == 7.0)  # Projector::adjoint writes tissue voxels only
    np.testing.assert_allclose(out[P.support], P.adjoint_host(y)[P.support], rtol=1e-6)


def test_sum_is_fp64(fixture72):
    rho, x, y, shape, sp = fixture72
    P = projector(fixture72)
    d = torch.from_numpy(x).cuda()
    assert abs(P.sum(d) - x.sum(dtype=np.float64)) < 1e-9 * x.sum(dtype=np.float64)


def test_bounded_wait_reports_and_the_context_survives(fixture72):
    """A field-stream wait that nothing completes gives up after its bound, raises the error
    flag, and the handle keeps working (the failure is reported on the host, no GPU fault)."""
    rho, x, y, shape, sp = fixture72
    with pm.Projector("68Ga", rho, sp, rays=32) as P:
        rc = pm.lib().prc_wait_selftest(P._h, 2000)
        assert rc == 5  # PRC_ERR_CUDA
        assert b"bounded wait" in pm.lib().prc_last_error()
        P.synchronize()  # the flag was cleared when reported
        assert rel_l2(P.forward_host(x), projector(fixture72).forward_host(x)) < 1e-6
