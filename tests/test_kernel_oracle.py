"""The FP64 water-kernel quadrature restated from the reference's tests/reference.py
(oracle/kernel_oracle.py), pinned to the fixtures the reference's own module produced
(tests/golden/make_kernel_golden.py).  No GPU is used."""
import numpy as np
import pytest

from conftest import GOLDEN
from oracle import kernel_oracle as ko

ISOTOPES = ("11C", "13N", "15O", "18F", "64Cu", "68Ga", "82Rb", "124I")


@pytest.mark.parametrize("iso", ISOTOPES)
def test_survival_equals_the_reference_module(iso):
    model = np.load(GOLDEN / "range_model.npz")
    br = ko.table_branches(iso)
    np.testing.assert_array_equal(br[:, 1:], model[f"branches_{iso}"][:, 1:].astype(np.float64))
    s = ko.survival(ko.fix_weights(br), model["radius"])
    np.testing.assert_allclose(s, model[f"survival_{iso}"], rtol=0, atol=1e-15)


@pytest.mark.parametrize("size", [4.0, 2.0])
def test_water_kernel_equals_the_reference_module(size):
    g = np.load(GOLDEN / "water_kernel.npz")
    half = int(g[f"half_{size:g}mm"])
    exact = g[f"kernel_{size:g}mm"]
    k = ko.water_kernel(ko.table_branches("68Ga"), (size,) * 3, half)
    assert k.shape == exact.shape
    np.testing.assert_allclose(k, exact, rtol=0, atol=1e-14 * exact.max())


def test_water_kernel_properties():
    """Nonnegative, mass at most one (the tail beyond the box is dropped), peaked at the
    source voxel, first moments near zero (the Fibonacci set is only nearly balanced)."""
    k = ko.water_kernel(ko.table_branches("18F"), (2.0, 2.0, 2.0), 3, n_dirs=400, n_shells=200)
    assert 0.99 < k.sum() <= 1.0 + 1e-12
    assert (k >= 0).all()
    c = np.indices(k.shape) - 3
    for axis in c:
        assert abs((k * axis).sum()) < 2e-3
    assert k[3, 3, 3] == k.max()


def test_fix_weights_sums_to_one_and_touches_only_the_lightest():
    br = ko.table_branches("82Rb")
    fixed = ko.fix_weights(br)
    assert abs(fixed[:, 0].sum() - 1.0) < 1e-15
    heavy = int(np.argmax(br[:, 0]))
    assert fixed[heavy, 0] == br[heavy, 0]
    np.testing.assert_array_equal(fixed[:, 1:], br[:, 1:])


def test_fibonacci_directions_are_unit_and_balanced():
    d = ko.fibonacci_directions(1000)
    np.testing.assert_allclose(np.linalg.norm(d, axis=1), 1.0, atol=1e-14)
    assert np.abs(d.mean(0)).max() < 2e-3


def test_empty_quadrature():
    k = ko.water_kernel(ko.table_branches("68Ga"), (1.0, 1.0, 1.0), 0, n_dirs=10, n_shells=0)
    assert k.shape == (1, 1, 1) and k[0, 0, 0] == 0.0


@pytest.mark.parametrize("size", [2.0, 4.0])
@pytest.mark.parametrize("iso", ISOTOPES)
def test_projector_oracle_water_kernel_for_every_isotope(iso, size):
    """The FP64 projector oracle (128 rays, ray-traced) against the FP64 quadrature in
    homogeneous water, for all eight isotopes: within 2 % of the blur (measured 0.6-1.6 %; the
    reference checks 68Ga at 1 %, tests/test_solver.py:216-243) with zero first moments."""
    from oracle import oracle
    _, _, cutoff = oracle.isotope(iso)
    half = int(np.ceil(1.2 * cutoff / size)) + 1
    exact = ko.water_kernel(ko.table_branches(iso), (size,) * 3, half)
    n, c = 2 * half + 5, half + 2
    delta = np.zeros((n, n, n), np.float32)
    delta[c, c, c] = 1
    P = oracle.Problem(iso, np.ones((n, n, n), np.float32), (size,) * 3, rays=128, precision=64)
    k = P.forward(delta)[c - half:c + half + 1, c - half:c + half + 1, c - half:c + half + 1].astype(np.float64)
    blur = exact.copy()
    blur[half, half, half] -= 1
    assert np.linalg.norm(k - exact) / np.linalg.norm(blur) < 0.02
    for axis in np.indices(k.shape) - half:
        assert abs((k * axis).sum()) < 1e-6
