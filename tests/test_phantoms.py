"""The seeded phantom generators (no GPU): the stretched small phantom reproduces the small
phantom on its own grid, and keeps its tissue classes on the clinical grid."""
import numpy as np

from prc_mlem_b200 import phantoms


def test_scaled_small_phantom_reproduces_the_small_phantom():
    a = phantoms.small_phantom(seed=1)
    b = phantoms.scaled_small_phantom(seed=1, shape=(24, 32, 32), spacing=(2.0, 2.0, 2.0))
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and a[2] == b[2]


def test_scaled_small_phantom_on_the_clinical_grid():
    rho, truth, sp = phantoms.scaled_small_phantom()
    assert rho.shape == truth.shape == (159, 128, 128) and sp == (0.776, 0.776, 0.795)
    assert set(np.unique(rho)) == {np.float32(phantoms.AIR), np.float32(0.3), np.float32(1.0), np.float32(1.85)}
    body = rho >= 0.05
    assert 0.3 < body.mean() < 0.5 and np.all(truth[~body] == 0) and truth.max() > 2
