"""The learned range-kernel surrogate on a B200: its tensor-core GEMM engine (tcgen05, bf16
operands, fp32 accumulation in tensor memory) against a float64 reference."""
import ctypes

import numpy as np
import pytest
import torch

import prc_mlem_b200 as pm

pytestmark = pytest.mark.gpu


def lib():
    l = pm.lib()
    l.prc_nn_gemm_bf16.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int] * 3 + [ctypes.c_void_p] * 2
    return l


@pytest.mark.parametrize("M,N,K", [(128, 64, 64), (200, 96, 100), (1000, 32, 864), (33, 2048, 32), (2048, 32, 513)])
def test_tensor_core_gemm_matches_float64(M, N, K):
    g = torch.Generator().manual_seed(M * 7 + N * 3 + K)
    a = torch.randn(M, K, generator=g).to(torch.bfloat16)
    b = torch.randn(N, K, generator=g).to(torch.bfloat16)
    expect = a.double() @ b.double().T
    da, db = a.cuda(), b.cuda()
    c = torch.full((M, N), float("nan"), dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = lib().prc_nn_gemm_bf16(da.data_ptr(), db.data_ptr(), c.data_ptr(), M, N, K, err.data_ptr(), None)
    assert rc == 0, pm.lib().prc_last_error()
    torch.cuda.synchronize()
    assert err.item() == 0
    got = c.double().cpu()
    scale = (a.double().abs() @ b.double().abs().T)
    assert torch.all((got - expect).abs() <= 1e-5 * scale + 1e-6), float(((got - expect).abs() / scale).max())


# ---- the network: forward values and gradients against the FP64 CPU oracle -----------------
def nn_lib():
    l = pm.lib()
    l.prc_nn_create.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
    l.prc_nn_destroy.argtypes = [ctypes.c_void_p]
    l.prc_nn_param_count.restype = ctypes.c_int64
    l.prc_nn_set_params.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    l.prc_nn_get.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
    l.prc_nn_forward.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    l.prc_nn_backward.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_float,
                                  ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]
    return l


SHAPES = [("w1", (32, 3, 3, 3, 8)), ("b1", (32,)), ("w2", (32, 3, 3, 3, 32)), ("b2", (32,)),
          ("w3", (32, 3, 3, 3, 32)), ("b3", (32,)), ("w4", (32, 3, 3, 3, 32)), ("b4", (32,)),
          ("wh", (2048, 32)), ("bh", (2048,))]


def random_params(seed):
    rng = np.random.default_rng(seed)
    p = {}
    for name, shape in SHAPES:
        fan_in = int(np.prod(shape[1:])) if name.startswith("w") else 1
        p[name] = (rng.normal(0, 1.2 / np.sqrt(fan_in), shape) if name.startswith("w")
                   else rng.uniform(0.0, 0.2, shape)).astype(np.float32)
    return p


def flat(p):
    return np.concatenate([p[name].ravel() for name, _ in SHAPES]).astype(np.float32)


def unflat(v):
    out, off = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = v[off:off + n].reshape(shape)
        off += n
    return out


def test_network_forward_and_gradients_match_fp64_oracle():
    from oracle import nn_oracle
    l = nn_lib()
    assert l.prc_nn_param_count() == sum(int(np.prod(s)) for _, s in SHAPES)
    B = 6
    S = nn_oracle.SIDE
    assert l.prc_nn_patch_side() == S
    rng = np.random.default_rng(3)
    x0 = np.zeros((B, S, S, S, 8), np.float32)
    x0[..., 0] = rng.uniform(0, 1, (B, S, S, S))
    x0[..., 1] = rng.uniform(0, 1, (B, S, S, S)) < 0.8
    x0[np.arange(B), ..., 2 + np.arange(B) % 3] = 1.0
    target = rng.normal(0, 1, (B, 2048)).astype(np.float32)
    target[:, 12::16] = -1.0  # masked outputs
    target[1, 16:32] = -1.0
    params = random_params(11)
    h = ctypes.c_void_p()
    assert l.prc_nn_create(64, ctypes.byref(h)) == 0
    try:
        v = flat(params)
        assert l.prc_nn_set_params(h, v.ctypes.data) == 0
        d_x = torch.from_numpy(x0).to(torch.bfloat16).cuda()
        d_y = torch.empty(B, 2048, dtype=torch.float32, device="cuda")
        assert l.prc_nn_forward(h, d_x.data_ptr(), B, d_y.data_ptr(), None) == 0
        assert l.prc_nn_forward(h, d_x.data_ptr(), B, None, None) == 0
        loss = ctypes.c_double()
        d_t = torch.from_numpy(target).cuda()
        assert l.prc_nn_backward(h, d_t.data_ptr(), B, 0.0, ctypes.byref(loss), None) == 0, pm.lib().prc_last_error()
        grads = np.zeros_like(v)
        assert l.prc_nn_get(h, 1, grads.ctypes.data) == 0
    finally:
        l.prc_nn_destroy(h)
    net = nn_oracle.Net(params)
    y_ref, _ = net.forward(x0.astype(np.float64))
    y = d_y.cpu().numpy()
    assert np.linalg.norm(y - y_ref) / np.linalg.norm(y_ref) < 2e-3
    ref_loss, ref_g = net.loss_and_grads(x0.astype(np.float64), target.astype(np.float64))
    assert abs(loss.value - ref_loss) <= 1e-3 * ref_loss
    g = unflat(grads)
    for name, _ in SHAPES:
        err = np.linalg.norm(g[name] - ref_g[name]) / max(np.linalg.norm(ref_g[name]), 1e-30)
        assert err < 2e-2, (name, err)


# ---- training, and the surrogate projector with the tracer as judge and fallback ------------
def test_training_on_the_gpu_reduces_the_loss():
    from prc_mlem_b200 import surrogate as sg
    x, t = sg.make_dataset(n_vol=512, per_vol=32, seed=5)
    xv, tv = sg.make_dataset(n_vol=32, per_vol=32, seed=6)
    net = sg.Network(sg.init_params(1))
    before = net.evaluate(xv, tv)
    hist = sg.train(net, x, t, epochs=3, batch=256, seed=1)
    after = net.evaluate(xv, tv)
    assert hist[-1] < hist[0]
    assert after < 0.5 * before, (before, after)


def test_trained_network_beats_the_density_blind_kernel():
    """The committed weights (python -m prc_mlem_b200.train_surrogate) on fresh volumes: far
    lower error than the best density-blind kernel (the mean of the targets), both over the
    outputs a surrogate field takes from the network (the unmasked targets)."""
    from prc_mlem_b200 import surrogate as sg
    net = sg.load_trained()
    if net is None:
        pytest.skip("no trained weights committed")
    xv, tv = sg.make_dataset(n_vol=64, per_vol=32, seed=4242)
    keep = (tv >= 0).float()
    mean = (tv.clamp(min=0) * keep).sum(0, keepdim=True) / keep.sum(0, keepdim=True).clamp(min=1)
    blind = float((((tv - mean) * keep) ** 2).mean())
    assert net.evaluate(xv, tv) < 0.5 * blind


@pytest.fixture(scope="module")
def small():
    from prc_mlem_b200 import phantoms
    rho, truth, sp = phantoms.small_phantom(seed=1)
    return rho, truth, sp


def test_surrogate_field_is_transpose_consistent_and_conservative(small):
    rho, truth, sp = small
    for fb in (0.0, 0.1):
        with pm.Projector("68Ga", rho, sp, surrogate="traced", fallback_nrmse=fb) as Q:
            x = truth
            y = np.random.default_rng(2).uniform(0.1, 1.0, x.shape).astype(np.float32) * Q.support
            ax, aty = Q.forward_host(x), Q.adjoint_host(y)
            lhs, rhs = np.sum(ax.astype(np.float64) * y), np.sum(x.astype(np.float64) * aty)
            assert abs(lhs / rhs - 1) < 3e-6
            assert abs(ax.sum(dtype=np.float64) / (x * Q.support).sum(dtype=np.float64) - 1) < 3e-6


def test_exact_fallback_where_the_radial_bins_are_coarse(small):
    """The tracer keeps exact weights for the far rays whose positrons travel past the water
    range of the radial bins (through lung or air, where the bins are coarse) and stores the
    water bins of the others: the blur then matches the plain projector closely."""
    rho, truth, sp = small
    with pm.Projector("68Ga", rho, sp) as P:
        ref = P.forward_host(truth)
    with pm.Projector("68Ga", rho, sp, surrogate="traced") as Q:
        mixed = Q.forward_host(truth)
        assert 0 < Q.fallbacks < Q.n_active * 128  # (source, far ray) pairs
    assert np.linalg.norm(mixed - ref) / np.linalg.norm(ref) < 0.01


def test_trained_network_gains_over_the_method_without_it(small):
    """The committed trained network against the same surrogate without a learned kernel (the
    density-blind mean kernel of the training set): lower blur error against the plain
    projector, with every far ray inside the water range predicted (no error judge)."""
    from prc_mlem_b200 import surrogate as sg
    net = sg.load_trained()
    if net is None:
        pytest.skip("no trained weights committed")
    from prc_mlem_b200 import phantoms
    rho, truth, sp = phantoms.torso_phantom(seed=2, shape=(40, 128, 128))  # 0.776 mm, as trained (0.8 mm)
    x, t = sg.make_dataset(n_vol=64, per_vol=32, seed=7)
    blind_params = np.zeros_like(net.params())
    keep = (t >= 0).float()
    blind_params[-2048:] = ((t.clamp(min=0) * keep).sum(0) / keep.sum(0).clamp(min=1)).cpu().numpy()
    blind = sg.Network(blind_params)
    with pm.Projector("68Ga", rho, sp) as P:
        ref = P.forward_host(truth)
    errs = {}
    for name, n in (("learned", net), ("blind", blind)):
        with pm.Projector("68Ga", rho, sp, surrogate=n, target_scale=sg.TARGET_SCALE) as Q:
            errs[name] = np.linalg.norm(Q.forward_host(truth) - ref) / np.linalg.norm(ref)
    assert errs["learned"] < errs["blind"], errs


def test_judge_keeps_rays_cut_by_the_volume_edge_exact():
    """With a network, the tracer also keeps exact every far ray that the volume's edge cuts
    inside the water range (a truncated kernel): on a thin torso slab, whose sources mostly lie
    near a cut face, more (source, ray) pairs stay exact than with the traced coefficients, which
    keep exact only the rays that reach past the water range."""
    from prc_mlem_b200 import phantoms, surrogate as sg
    net = sg.load_trained()
    if net is None:
        pytest.skip("no trained weights committed")
    rho, truth, sp = phantoms.torso_phantom(seed=2, shape=(24, 128, 128))
    with pm.Projector("68Ga", rho, sp, surrogate="traced") as Q:
        beyond_only = Q.fallbacks
    with pm.Projector("68Ga", rho, sp, surrogate=net, target_scale=sg.TARGET_SCALE) as Q:
        with_cut = Q.fallbacks
        total = Q.n_active * 128
    assert beyond_only < with_cut < total
    assert with_cut - beyond_only > 0.05 * total  # most rays toward the two faces 12 voxels away
