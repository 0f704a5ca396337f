"""Mixed precision on the long-range isotopes (the 82Rb / 124I configuration): bf16 stored
weights with fp32 accumulation and FP64 sums, checked against the FP64 oracle on a 48^3 crop of
the torso (corrected image and forward/adjoint identity, beside the fp32 form), and on the full
200^3 grid, where the size-independent invariants (identity, count conservation) must hold."""
import numpy as np
import pytest
import torch

import prc_mlem_b200 as pm
from conftest import nrmse
from prc_mlem_b200 import phantoms

pytestmark = pytest.mark.gpu
RAYS = 64
ITERS, BETA, GAMMA = 6, 0.03, 20.0
_crop = {}


def torso_crop():
    """48^3 voxels at 0.776 x 0.776 x 0.795 mm around both lungs, the spine and the body centre."""
    if not _crop:
        rho, truth, sp = phantoms.torso_phantom()
        sl = (slice(80, 128), slice(40, 88), slice(40, 88))
        _crop["v"] = (np.ascontiguousarray(rho[sl]), np.ascontiguousarray(truth[sl]), sp)
    return _crop["v"]


def identity_residual(P, shape, rho, seed=5):
    rng = np.random.default_rng(seed)
    x = np.where(np.maximum(rho, 1e-3) >= 0.05, rng.random(shape), 0.0).astype(np.float32)
    y = rng.random(shape).astype(np.float32)
    ax, aty = P.forward_host(x).astype(np.float64), P.adjoint_host(y).astype(np.float64)
    lhs, rhs = float(np.sum(ax * y)), float(np.sum(x.astype(np.float64) * aty))
    return abs(lhs - rhs) / abs(lhs), abs(ax.sum() / x.sum(dtype=np.float64) - 1)


@pytest.mark.parametrize("iso", ["82Rb", "124I"])
def test_long_range_forms_against_fp64_oracle(iso, oracle_mod):
    rho, truth, sp = torso_crop()
    with pm.Projector(iso, rho, sp, rays=RAYS) as P32:
        g = P32.forward_host(truth)
        out32 = P32.correct_host(g, ITERS, BETA, GAMMA, True)
        ident32, cons32 = identity_residual(P32, rho.shape, rho)
    with pm.Projector(iso, rho, sp, rays=RAYS, precision=pm.PRC_PRECISION_BF16) as P16:
        assert P16.cache_mode[0] == pm.PRC_CACHE_FULL
        out16 = P16.correct_host(g, ITERS, BETA, GAMMA, True)
        ident16, cons16 = identity_residual(P16, rho.shape, rho)
    ref = oracle_mod.Problem(iso, rho, sp, rays=RAYS, precision=64).correct(g, ITERS, BETA, GAMMA, True)
    assert nrmse(out32, ref) < 1e-4   # the plain method
    assert nrmse(out16, ref) < 1e-2   # mixed precision: the 1 % gate
    assert ident32 < 1e-6 and ident16 < 1e-6
    assert cons32 < 3e-6 and cons16 < 3e-6


def test_full_grid_200_cubed_82rb_bf16():
    rho, truth, _ = phantoms.torso_phantom(shape=(200, 200, 200))
    sp = (0.776, 0.776, 0.776)
    with pm.Projector("82Rb", rho, sp, rays=128, precision=pm.PRC_PRECISION_BF16) as P:
        mode, src_entries, tgt_entries = P.cache_mode
        assert mode in (pm.PRC_CACHE_FULL, pm.PRC_CACHE_SOURCE_MAJOR) and src_entries > 0
        ident, cons = identity_residual(P, rho.shape, rho)
        assert ident < 1e-6 and cons < 3e-6
        g = P.forward_host(truth)
        d_g = torch.from_numpy(g).cuda()
        d_out = torch.empty_like(d_g)
        P.correct(d_g, d_out, 2, BETA, GAMMA, True)
        P.synchronize()  # the run is asynchronous on the engine's stream
        out = d_out.cpu().numpy()
        assert np.all(np.isfinite(out))
        measured = np.where(np.maximum(rho, 1e-3) >= 0.05, g, 0.0).sum(dtype=np.float64)
        assert abs(out.sum(dtype=np.float64) / measured - 1) < 1e-5  # counts kept on the support
