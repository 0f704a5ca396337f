"""The CPU oracle (oracle/prc_oracle.c), pinned against the reference itself:
  * golden outputs of the reference executable prc.cu run on a B200 (tests/golden/ref_outputs.npz,
    made by tests/golden/make_ref_golden.py);
  * the reference's own FP64 range quadrature tests/reference.py (tests/golden/*.npz, made by
    tests/golden/make_kernel_golden.py): survival values, table error, homogeneous water kernel;
  * the reference's RDP formula tests (tests/test_rdp.py), applied to the oracle's update.
No GPU is used."""
import math

import numpy as np
import pytest
from scipy.optimize import minimize_scalar

from conftest import GOLDEN, rel_l2

ISOTOPES = ("11C", "13N", "15O", "18F", "64Cu", "68Ga", "82Rb", "124I")
# 99.95 % water-equivalent cutoffs [mm] quoted for the reference model
CUTOFFS = {"11C": 3.77, "13N": 4.98, "15O": 7.81, "18F": 2.12, "64Cu": 2.20, "68Ga": 8.49, "82Rb": 16.16,
           "124I": 9.66}


@pytest.mark.parametrize("iso", ISOTOPES)
def test_isotope_model_and_cutoff(oracle_mod, iso):
    n, br, cutoff = oracle_mod.isotope(iso)
    model = np.load(GOLDEN / "range_model.npz")
    ref = model[f"branches_{iso}"]
    assert n == len(ref)
    # weights fixed so they sum to one in float (prc.cu:577-584)
    assert abs(np.sum(br[:n, 0], dtype=np.float32) - 1) < 1e-6
    np.testing.assert_array_equal(br[:n, 1:], ref[:, 1:])
    assert abs(cutoff - CUTOFFS[iso]) < 0.006


@pytest.mark.parametrize("iso", ISOTOPES)
def test_survival_matches_reference_quadrature(oracle_mod, iso):
    model = np.load(GOLDEN / "range_model.npz")
    r = model["radius"]
    exact = model[f"survival_{iso}"]
    ours = oracle_mod.survival(iso, r)
    # the oracle fixes the weights in float, reference.py in double: ~1e-8
    np.testing.assert_allclose(ours, exact, rtol=0, atol=2e-7)


@pytest.mark.parametrize("iso", ISOTOPES)
def test_float_table_error_bound(oracle_mod, iso):
    """The 4097-entry float table stays within 2e-5 of FP64 survival (tests/test_rdp.py:18-24)."""
    model = np.load(GOLDEN / "range_model.npz")
    assert float(model[f"table_error_{iso}"]) <= 2e-5
    _, _, cutoff = oracle_mod.isotope(iso)
    w = np.concatenate([np.linspace(0, cutoff, 200001), (np.arange(4096) + 0.5) * cutoff / 4096])
    table = oracle_mod.survival(iso, w, f32=True)
    exact = oracle_mod.survival(iso, w)
    assert np.max(np.abs(table - exact)) <= 2e-5


@pytest.mark.parametrize("precision", [64, 32])
@pytest.mark.parametrize("size", [4.0, 2.0])
def test_water_kernel_matches_reference_quadrature(oracle_mod, precision, size):
    """Homogeneous 68Ga water kernel within 1 % of the blur of reference.kernel and with zero
    first moments (tests/test_solver.py:216-243)."""
    g = np.load(GOLDEN / "water_kernel.npz")
    half = int(g[f"half_{size:g}mm"])
    exact = g[f"kernel_{size:g}mm"]
    n, c = 2 * half + 5, half + 2
    delta = np.zeros((n, n, n), np.float32)
    delta[c, c, c] = 1
    P = oracle_mod.Problem("68Ga", np.ones((n, n, n), np.float32), (size,) * 3, rays=128, precision=precision)
    k = P.forward(delta)[c - half:c + half + 1, c - half:c + half + 1, c - half:c + half + 1].astype(np.float64)
    blur = exact.copy()
    blur[half, half, half] -= 1
    assert np.linalg.norm(k - exact) / np.linalg.norm(blur) < 0.01
    for axis in np.indices(k.shape) - half:
        assert abs((k * axis).sum()) < 1e-6


@pytest.fixture(scope="module")
def fixture_problems(oracle_mod, fixture72):
    rho, x, y, shape, sp = fixture72
    return {(iso, prec): oracle_mod.Problem(iso, rho, sp, rays=32, precision=prec).normalize()
            for iso in ISOTOPES for prec in (64, 32)}


@pytest.mark.parametrize("precision", [64, 32])
@pytest.mark.parametrize("iso", ISOTOPES)
def test_oracle_projector_matches_reference_binary(fixture_problems, fixture72, ref_golden, iso, precision):
    rho, x, y, shape, sp = fixture72
    np.testing.assert_array_equal(ref_golden["fixture_x"], x)
    P = fixture_problems[(iso, precision)]
    assert rel_l2(P.forward(x), ref_golden[f"fixture_fwd_{iso}"]) < 1e-5
    assert rel_l2(P.adjoint(y), ref_golden[f"fixture_adj_{iso}"]) < 1e-5


def test_oracle_exact_range_and_rays(oracle_mod, fixture72, ref_golden):
    rho, x, y, shape, sp = fixture72
    P = oracle_mod.Problem("68Ga", rho, sp, rays=128, precision=64).normalize()
    assert rel_l2(P.forward(x), ref_golden["fixture_fwd_128_68Ga"]) < 1e-5
    P = oracle_mod.Problem("68Ga", rho, sp, rays=32, precision=32, exact_range=True).normalize()
    assert rel_l2(P.forward(x), ref_golden["fixture_fwd_exact_68Ga"]) < 1e-5
    ones = P.adjoint(np.ones(shape))
    assert rel_l2(ones, ref_golden["fixture_adj_one_68Ga"]) < 1e-6


@pytest.mark.parametrize("iso", ["68Ga", "82Rb", "18F"])
def test_oracle_identity_and_conservation(fixture_problems, fixture72, iso):
    rho, x, y, shape, sp = fixture72
    P = fixture_problems[(iso, 64)]
    ax, aty = P.forward(x), P.adjoint(y)
    lhs, rhs = np.sum(ax * y), np.sum(x.astype(np.float64) * aty)
    assert abs(lhs / rhs - 1) < 1e-12
    assert abs(ax.sum() / x.sum(dtype=np.float64) - 1) < 1e-12
    assert np.all(ax[~P.support] == 0)
    one = P.adjoint(np.ones(shape))
    np.testing.assert_allclose(one[P.support], 1, rtol=1e-12)
    assert np.all(one[~P.support] == 0)


EM_CASES = {"em_b0.1_it3": (3, 0.1, 20.0, True), "em_b0_it4_plain": (4, 0.0, 20.0, False),
            "em_b0.2_it2_plain": (2, 0.2, 20.0, False), "em_b0.03_it6": (6, 0.03, 20.0, True),
            "em_b0_it25": (25, 0.0, 20.0, True)}


@pytest.mark.parametrize("precision", [64, 32])
@pytest.mark.parametrize("case", sorted(EM_CASES))
def test_oracle_correction_matches_reference_binary(fixture_problems, fixture72, ref_golden, case, precision):
    rho, x, y, shape, sp = fixture72
    it, beta, gamma, accel = EM_CASES[case]
    out = fixture_problems[("68Ga", precision)].correct(x, it, beta, gamma, accel)
    assert rel_l2(out, ref_golden[f"fixture_{case}"]) < 1e-5


def test_oracle_small_phantom_matches_reference_binary(oracle_mod, ref_golden):
    from prc_mlem_b200 import phantoms
    rho, truth, sp = phantoms.small_phantom(seed=1)
    np.testing.assert_array_equal(ref_golden["small_rho"], rho)
    P = oracle_mod.Problem("18F", rho, sp, rays=32, precision=64).normalize()
    assert rel_l2(P.forward(truth), ref_golden["small_fwd"]) < 1e-5
    assert rel_l2(P.adjoint(truth), ref_golden["small_adj"]) < 1e-5
    out = P.correct(ref_golden["small_g"], 4, 0.0, 20.0, False)
    assert rel_l2(out, ref_golden["small_em_b0_it4_plain"]) < 1e-5


def test_zero_iterations_passthrough(fixture_problems, fixture72):
    rho, x, y, shape, sp = fixture72
    src = x.copy()
    src[5, 4, 5] = 0
    out = fixture_problems[("68Ga", 32)].correct(src, 0)
    np.testing.assert_array_equal(out, src)


# ---- RDP formulas (tests/test_rdp.py of the reference), checked on the oracle's update ----
def surrogate_step(old, em, gradient, curvature, beta):
    a = beta * curvature
    b = 1 + beta * (gradient - curvature * old)
    if a == 0:
        return em / b
    root = math.sqrt(b * b + 4 * a * em)
    if b < 0:
        return (root - b) / (2 * a)
    return 2 * em / (b + root) if em > 0 else 0.0


def pair_terms(fj, fk, gamma, eps, w):
    d = fj - fk
    D = fj + fk + gamma * abs(d) + eps
    grad = w * d * (fj + 3 * fk + gamma * abs(d) + 2 * eps) / D ** 2
    half_quad = (2 * (fj + fk + eps) + gamma * abs(d)) / D ** 2
    hess = 2 * (2 * fk + eps) ** 2 / D ** 3
    return grad, 2 * w * max(half_quad, hess)


def test_rdp_derivatives_against_finite_differences():
    def penalty(x, y, gamma, eps):
        return (x - y) ** 2 / (x + y + gamma * abs(x - y) + eps)

    for gamma in (0.0, 2.0, 10.0, 50.0):
        for eps in (0.0, 0.17):
            for x, y in ((0.2, 1.3), (4.0, 0.7), (2.0, 2.0)):
                h = 1e-5
                g, _ = pair_terms(x, y, gamma, eps, 1.0)
                fd = (penalty(x + h, y, gamma, eps) - penalty(x - h, y, gamma, eps)) / (2 * h)
                assert abs(g - fd) < 2e-7


def test_oracle_update_matches_scalar_minimisation(oracle_mod):
    """A two-voxel volume: the oracle's closed-form root minimises the separable surrogate
    -em log x + x + beta (G dx + C dx^2 / 2) (tests/test_rdp.py:69-83)."""
    rng = np.random.default_rng(42)
    rho = np.ones((1, 1, 2), np.float32)
    P = oracle_mod.Problem("68Ga", rho, (1.0, 1.0, 1.0), precision=64)
    for _ in range(40):
        fj, fk = np.exp(rng.uniform(-2, 2, 2))
        back = np.exp(rng.uniform(-1, 1))
        beta = np.exp(rng.uniform(-2, 1))
        gamma, eps = 2.0, 1e-3
        f = np.array([[[fj, fk]]])
        out = P.update(f, np.full_like(f, back), beta, gamma, eps)[0, 0, 0]
        grad, curv = pair_terms(fj, fk, gamma, eps, 1.0)
        em = fj * back
        expect = surrogate_step(fj, em, grad, curv, beta)
        assert abs(out - expect) <= 1e-12 * max(1.0, expect)

        def objective(x):
            dx = x - fj
            return -em * math.log(x) + x + beta * (grad * dx + curv * dx ** 2 / 2)

        opt = minimize_scalar(objective, bounds=(1e-12, 2 * expect + 1), method="bounded", options={"xatol": 1e-11})
        assert abs(out - opt.x) < max(1e-7, out * 1e-6)


def test_zero_em_can_have_a_positive_prior_update():
    assert surrogate_step(old=0, em=0, gradient=-3, curvature=4, beta=1) == 0.5
    assert surrogate_step(old=0, em=0, gradient=1, curvature=4, beta=1) == 0
