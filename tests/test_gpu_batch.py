"""Batched frames on a B200: frames of different grids, isotopes and projector forms corrected
in one launch per MAP-EM phase (a captured CUDA graph) give the same images as each frame
corrected alone."""
import numpy as np
import pytest
import torch

import prc_mlem_b200 as pm
from conftest import rel_l2
from prc_mlem_b200 import phantoms

pytestmark = pytest.mark.gpu


def frame_set():
    out = []
    for k, (shape, iso) in enumerate([((24, 32, 32), "18F"), ((20, 40, 36), "68Ga"), ((30, 28, 28), "11C"),
                                      ((16, 48, 40), "15O")]):
        rho, truth, _ = phantoms.torso_phantom(seed=10 + k, shape=shape)
        out.append((iso, rho, (2.0, 2.0, 2.0), truth))
    return out


@pytest.mark.parametrize("cache,prec", [(pm.PRC_CACHE_FULL, pm.PRC_PRECISION_FP32), (pm.PRC_CACHE_NEAR, pm.PRC_PRECISION_FP32),
                                        (pm.PRC_CACHE_FULL, pm.PRC_PRECISION_FP24)], ids=["field", "traced", "field-fp24"])
def test_batched_correction_matches_each_frame_alone(cache, prec):
    frames = frame_set()
    batch = pm.Batch([(iso, rho, sp) for iso, rho, sp, _ in frames], rays=32, cache=cache, precision=prec)
    assert batch.warps in (2, 4, 8)
    gs, outs, refs = [], [], []
    for iso, rho, sp, truth in frames:
        with pm.Projector(iso, rho, sp, rays=32, cache=cache, precision=prec) as P:
            g = phantoms.poisson_counts(P.forward_host(truth), 1e5, seed=3)
            refs.append(P.correct_host(g, 5, 0.03, 20.0, True))
        gs.append(torch.from_numpy(g).cuda())
        outs.append(torch.full_like(gs[-1], float("nan")))
    for _ in range(2):  # the second run replays the captured graph
        batch.correct(gs, outs, 5, 0.03, 20.0, True)
        batch.synchronize()
        for out, ref in zip(outs, refs):
            assert rel_l2(out.cpu().numpy(), ref) < 1e-5
    # new parameters: a new schedule is captured
    batch.correct(gs, outs, 3, 0.0, 20.0, False)
    batch.synchronize()
    for (iso, rho, sp, truth), g, out in zip(frames, gs, outs):
        with pm.Projector(iso, rho, sp, rays=32, cache=cache, precision=prec) as P:
            ref = P.correct_host(g.cpu().numpy(), 3, 0.0, 20.0, False)
        assert rel_l2(out.cpu().numpy(), ref) < 1e-5
    batch.close()
