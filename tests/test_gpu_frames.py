"""Frames that share one projector (prc_forward_frames, prc_adjoint_frames, prc_em_run_frames).

The frames of a dynamic study share the density map, isotope and grid, so they share the
operator A; the reference corrects one volume per run of prc.cu (main(), prc.cu:659-711).  With
the stored field one pass projects up to four frames: the stream of weights, their template
offsets and predicates are read once and serve every frame's gather.  Each frame keeps the
single-volume accumulation order and the single-volume MAP-EM kernels, so its result must equal
the single-volume entry point's on the same input BIT FOR BIT in every stored-weight format and
for frame counts that make groups of four, three and two interleaved frames and of one frame
(which takes the single-volume kernels).  The forms without both majors of the
field run the frames one by one (their forward scatters with atomics, so they agree to rounding).
One case is also pinned to the reference executable's own MAP-EM output."""
import ctypes

import numpy as np
import pytest
import torch

import prc_mlem_b200 as pm
from conftest import rel_l2
from prc_mlem_b200 import phantoms

pytestmark = pytest.mark.gpu
FORMS = {"fp32": pm.PRC_PRECISION_FP32, "fp24": pm.PRC_PRECISION_FP24, "bf16": pm.PRC_PRECISION_BF16}
_projectors = {}


@pytest.fixture(scope="module")
def torso():
    rho, truth, spacing = phantoms.torso_phantom(seed=3, shape=(24, 64, 64))
    return rho, truth, spacing


def projector(torso, prec, cache=pm.PRC_CACHE_FULL):
    key = (prec, cache)
    if key not in _projectors:
        rho, _, spacing = torso
        _projectors[key] = pm.Projector("68Ga", rho, spacing, rays=32, cache=cache, precision=prec)
    return _projectors[key]


def frames(shape, n, seed=0):
    """n different activity volumes (device tensors): smooth blobs plus noise, one per frame."""
    rng = np.random.default_rng(seed)
    z, y, x = np.meshgrid(*[np.linspace(-1, 1, k) for k in shape], indexing="ij")
    out = []
    for i in range(n):
        c = rng.uniform(-0.5, 0.5, 3)
        blob = np.exp(-((z - c[0]) ** 2 + (y - c[1]) ** 2 + (x - c[2]) ** 2) / rng.uniform(0.05, 0.4))
        vol = (1000.0 * (i + 1) * blob + rng.uniform(0.0, 50.0, shape)).astype(np.float32)
        out.append(torch.from_numpy(vol).cuda())
    return out


def assert_identical(got, expect, what):
    diff = (got - expect).abs().max().item()
    assert torch.equal(got, expect), f"{what}: max abs difference {diff:.3e}"


@pytest.mark.parametrize("form", sorted(FORMS))
def test_projections_equal_single_volume(torso, form):
    P = projector(torso, FORMS[form])
    assert P.cache_mode[0] == pm.PRC_CACHE_FULL
    ins = frames(P.shape, 9, seed=1)  # two interleaved groups of four, then one frame alone
    fwd = [torch.full_like(x, -7.0) for x in ins]
    P.forward_frames(ins, fwd)
    adj = [torch.full_like(x, -7.0) for x in ins]  # the adjoint leaves off-tissue voxels untouched
    P.adjoint_frames(ins, adj)
    P.synchronize()
    for i, x in enumerate(ins):
        f1 = torch.full_like(x, -7.0)
        P.forward(x, f1)
        a1 = torch.full_like(x, -7.0)
        P.adjoint(x, a1)
        P.synchronize()
        assert_identical(fwd[i], f1, f"{form} forward, frame {i}")
        assert_identical(adj[i], a1, f"{form} adjoint, frame {i}")
    assert not torch.equal(fwd[0], fwd[1])


@pytest.mark.parametrize("form", sorted(FORMS))
@pytest.mark.parametrize("n,iters,beta,accel", [(5, 6, 0.03, True), (2, 3, 0.1, False), (3, 4, 0.0, True)],
                         ids=["5frames_accel", "2frames_plain", "3frames_unregularised"])
def test_map_em_equals_single_volume(torso, form, n, iters, beta, accel):
    P = projector(torso, FORMS[form])
    gs = frames(P.shape, n, seed=n)
    outs = [torch.empty_like(g) for g in gs]
    P.correct_frames(gs, outs, iters, beta, 20.0, accel)
    P.synchronize()
    for i, g in enumerate(gs):
        one = torch.empty_like(g)
        P.correct(g, one, iters, beta, 20.0, accel)
        P.synchronize()
        assert_identical(outs[i], one, f"{form} MAP-EM, frame {i}")
    # a second call reuses the frames' volumes and must not depend on the first
    again = [torch.empty_like(g) for g in gs]
    P.correct_frames(gs, again, iters, beta, 20.0, accel)
    P.synchronize()
    for i in range(n):
        assert_identical(again[i], outs[i], f"{form} MAP-EM repeated, frame {i}")


@pytest.mark.parametrize("cache,prec,exact", [(pm.PRC_CACHE_NEAR, pm.PRC_PRECISION_FP32, False),
                                              (pm.PRC_CACHE_SOURCE_MAJOR, pm.PRC_PRECISION_FP32, False),
                                              (pm.PRC_CACHE_FULL, pm.PRC_PRECISION_BF16_VOLUMES, True)],
                         ids=["near_cache", "source_major", "bf16_volumes"])
def test_forms_without_shared_passes_run_frame_by_frame(torso, cache, prec, exact):
    """Without both majors of the stored field the forward projection scatters with atomics, so
    two runs of the same frame agree to rounding (1e-6 relative L2), not bit for bit; the bf16-
    volume form gathers and must agree exactly."""
    P = projector(torso, prec, cache)

    def check(got, expect, what):
        if exact:
            assert_identical(got, expect, what)
        else:
            assert rel_l2(got.cpu().numpy(), expect.cpu().numpy()) < 1e-6, what

    gs = frames(P.shape, 3, seed=9)
    outs = [torch.empty_like(g) for g in gs]
    P.correct_frames(gs, outs, 3, 0.03, 20.0, True)
    fwd = [torch.empty_like(g) for g in gs]
    P.forward_frames(gs, fwd)
    P.synchronize()
    for i, g in enumerate(gs):
        one, f1 = torch.empty_like(g), torch.empty_like(g)
        P.correct(g, one, 3, 0.03, 20.0, True)
        P.forward(g, f1)
        P.synchronize()
        check(outs[i], one, f"MAP-EM frame {i}")
        check(fwd[i], f1, f"forward frame {i}")


def test_full_size_torso_frames_equal_single_volume():
    """The 128x128x159 68Ga torso at 128 rays (the headline configuration), five frames (a group
    of four and one alone), 6 accelerated MAP-EM iterations: bit-identical to one by one."""
    rho, truth, spacing = phantoms.torso_phantom(seed=2)
    with pm.Projector("68Ga", rho, spacing, rays=128, cache=pm.PRC_CACHE_FULL) as P:
        d_truth = torch.from_numpy(truth).cuda()
        blur = torch.empty_like(d_truth)
        P.forward(d_truth, blur)
        P.synchronize()
        gs = [phantoms.poisson_counts_device(blur, 5e7 * (k + 1), seed=200 + k) for k in range(5)]
        torch.cuda.synchronize()
        outs = [torch.empty_like(d_truth) for _ in gs]
        P.correct_frames(gs, outs, 6, 0.03, 20.0, True)
        P.synchronize()
        for i, g in enumerate(gs):
            one = torch.empty_like(g)
            P.correct(g, one, 6, 0.03, 20.0, True)
            P.synchronize()
            assert_identical(outs[i], one, f"torso frame {i}")


def test_surrogate_field_frames_equal_single_volume():
    """Frames through a surrogate coefficient field (the traced radial bins with exact fallback
    rays): the same shared passes over another template, bit-identical per frame."""
    rho, truth, sp = phantoms.small_phantom(seed=1)
    with pm.Projector("68Ga", rho, sp, surrogate="traced", precision=pm.PRC_PRECISION_BF16) as Q:
        assert Q.cache_mode[0] == pm.PRC_CACHE_FULL
        gs = frames(Q.shape, 4, seed=4)
        outs = [torch.empty_like(g) for g in gs]
        Q.correct_frames(gs, outs, 4, 0.03, 20.0, True)
        Q.synchronize()
        for i, g in enumerate(gs):
            one = torch.empty_like(g)
            Q.correct(g, one, 4, 0.03, 20.0, True)
            Q.synchronize()
            assert_identical(outs[i], one, f"surrogate frame {i}")


def test_fixture_frames_match_reference_binary(fixture72, ref_golden):
    """The seed-72 fixture as frame 1 of 3: its MAP-EM result is prc.cu's within 1e-5."""
    rho, x, y, shape, sp = fixture72
    with pm.Projector("68Ga", rho, sp, rays=32, cache=pm.PRC_CACHE_FULL) as P:
        d_x = torch.from_numpy(x).cuda()
        gs = [2.0 * d_x, d_x, torch.flip(d_x, dims=[0]).contiguous()]
        outs = [torch.empty_like(d_x) for _ in gs]
        for case, (it, beta, accel) in {"em_b0.03_it6": (6, 0.03, True), "em_b0.1_it3": (3, 0.1, True),
                                        "em_b0_it4_plain": (4, 0.0, False)}.items():
            P.correct_frames(gs, outs, it, beta, 20.0, accel)
            P.synchronize()
            assert rel_l2(outs[1].cpu().numpy(), ref_golden[f"fixture_{case}"]) < 1e-5


def test_argument_errors(torso):
    P = projector(torso, pm.PRC_PRECISION_FP32)
    g = torch.ones(P.shape, dtype=torch.float32, device="cuda")
    ptrs = (ctypes.c_void_p * 2)(g.data_ptr(), None)
    outs = (ctypes.c_void_p * 2)(g.data_ptr(), g.data_ptr())
    lib = pm.lib()
    assert lib.prc_em_run_frames(P._h, 0, ptrs, outs, 3, 0.0, 20.0, 1, None) == pm.PRC_ERR_ARGUMENT
    assert lib.prc_em_run_frames(P._h, 2, ptrs, outs, 3, 0.0, 20.0, 1, None) == pm.PRC_ERR_ARGUMENT
    assert b"null frame volume" in lib.prc_last_error()
    assert lib.prc_forward_frames(P._h, 2, ptrs, outs, None) == pm.PRC_ERR_ARGUMENT
    assert lib.prc_adjoint_frames(P._h, 1, None, outs, None) == pm.PRC_ERR_ARGUMENT
    one = (ctypes.c_void_p * 1)(g.data_ptr())
    assert lib.prc_em_run_frames(P._h, 1, one, one, -1, 0.0, 20.0, 1, None) == pm.PRC_ERR_ARGUMENT
    assert lib.prc_em_run_frames(P._h, 1, one, one, 2, float("nan"), 20.0, 1, None) == pm.PRC_ERR_ARGUMENT
