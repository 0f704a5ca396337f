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


@pytest.mark.parametrize("prec", [pm.PRC_PRECISION_FP32, pm.PRC_PRECISION_BF16], ids=["fp32", "bf16"])
def test_frames_of_one_study_share_one_projector(prec):
    """Frames that pass the same density array with the same grid and isotope (the frames of one
    dynamic study) share one projector: the later frames hold no stored field of their own, the
    batched projections take them four (then two) at a time through one pass of the field, and
    every frame's image equals the frame corrected alone."""
    rho, truth, _ = phantoms.torso_phantom(seed=21, shape=(24, 40, 36))
    rho2, truth2, _ = phantoms.torso_phantom(seed=22, shape=(20, 32, 32))
    sp = (2.0, 2.0, 2.0)
    frames = [("68Ga", rho, sp, truth, 1e5), ("68Ga", rho, sp, truth, 3e5), ("18F", rho2, sp, truth2, 1e5),
              ("68Ga", rho, sp, 2.0 * truth, 2e5)] + [("68Ga", rho, sp, truth, 1e5 * k) for k in (4, 5, 6)]
    batch = pm.Batch([(iso, r, s) for iso, r, s, _, _ in frames], rays=32, precision=prec)
    owner = batch.device_bytes(0)
    for i in (1, 3, 4, 5, 6):
        assert batch.cache_mode(i)[0] == pm.PRC_CACHE_FULL
        assert batch.device_bytes(i) < owner / 4, (batch.device_bytes(i), owner)
    gs, outs, refs = [], [], []
    for k, (iso, r, s, t, counts) in enumerate(frames):
        with pm.Projector(iso, r, s, rays=32, precision=prec) as P:
            g = phantoms.poisson_counts(P.forward_host(t), counts, seed=30 + k)
            refs.append(P.correct_host(g, 5, 0.03, 20.0, True))
        gs.append(torch.from_numpy(g).cuda())
        outs.append(torch.full_like(gs[-1], float("nan")))
    for _ in range(2):
        batch.correct(gs, outs, 5, 0.03, 20.0, True)
        batch.synchronize()
        for out, ref in zip(outs, refs):
            assert rel_l2(out.cpu().numpy(), ref) < 1e-5
    batch.close()
