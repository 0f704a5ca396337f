"""Source tiles of the stored field change no result: every tile shape, in both stored
precisions, projects and corrects like the reference executable (fp32 within 1e-5 relative L2
of prc.cu's outputs on the seed-72 fixture of tests/test_solver.py:143-157) and keeps the
forward/adjoint identity."""
import numpy as np
import pytest

import prc_mlem_b200 as pm
from conftest import nrmse, rel_l2

pytestmark = pytest.mark.gpu
TILES = [pm.PRC_TILE_8x2x2, pm.PRC_TILE_16x2x1, pm.PRC_TILE_32x1x1, pm.PRC_TILE_4x4x2, pm.PRC_TILE_16x1x2]


@pytest.mark.parametrize("tile", TILES, ids=[f"{x}x{y}x{z}" for x, y, z in (pm.TILE_SHAPES[t] for t in TILES)])
def test_tile_shapes_match_reference_binary(fixture72, ref_golden, tile):
    rho, x, y, shape, sp = fixture72
    with pm.Projector("68Ga", rho, sp, rays=32, tile=tile) as P:
        assert P.tile == tile and P.cache_mode[0] == pm.PRC_CACHE_FULL
        assert rel_l2(P.forward_host(x), ref_golden["fixture_fwd_68Ga"]) < 1e-5
        assert rel_l2(P.adjoint_host(y), ref_golden["fixture_adj_68Ga"]) < 1e-5
        out = P.correct_host(x, 6, 0.03, 20.0, True)
        assert rel_l2(out, ref_golden["fixture_em_b0.03_it6"]) < 1e-5


@pytest.mark.parametrize("tile", TILES)
def test_bf16_tiles_keep_identity_and_accuracy(fixture72, oracle_mod, tile):
    rho, x, y, shape, sp = fixture72
    with pm.Projector("68Ga", rho, sp, rays=32, tile=tile, precision=pm.PRC_PRECISION_BF16) as P:
        ax, aty = P.forward_host(x).astype(np.float64), P.adjoint_host(y).astype(np.float64)
        lhs, rhs = float(np.sum(ax * y)), float(np.sum(x.astype(np.float64) * aty))
        assert abs(lhs - rhs) / abs(lhs) < 3e-6
        fp64 = oracle_mod.Problem("68Ga", rho, sp, rays=32, precision=64).correct(x, 6, 0.03, 20.0, True)
        assert nrmse(P.correct_host(x, 6, 0.03, 20.0, True), fp64) < 1e-2


def test_automatic_tile_is_a_concrete_shape(fixture72):
    rho, x, y, shape, sp = fixture72
    with pm.Projector("68Ga", rho, sp, rays=32) as P:
        assert P.tile in TILES


def test_tuned_tile_is_remembered_for_the_configuration():
    from prc_mlem_b200 import phantoms
    rho, truth, sp = phantoms.torso_phantom(shape=(40, 48, 48))
    tile = pm.tune_tile("18F", rho, sp, rays=64)
    assert tile in (pm.PRC_TILE_8x2x2, pm.PRC_TILE_16x2x1, pm.PRC_TILE_32x1x1)
    assert pm.tune_tile("18F", rho, sp, rays=64) == tile  # remembered, not re-timed
    with pm.Projector("18F", rho, sp, rays=64) as P:
        assert P.tile == tile
