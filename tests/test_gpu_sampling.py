"""prc_poisson (device Poisson counts): the same counts as its CPU restatement, the Poisson
moments across the inversion / PTRS switch, determinism, and the data helper."""
import math

import numpy as np
import pytest
import torch

import prc_mlem_b200 as pm
from oracle import sampling_oracle as so
from prc_mlem_b200 import phantoms

pytestmark = pytest.mark.gpu


def draw(mean, scale, seed):
    d = torch.as_tensor(np.ascontiguousarray(mean, np.float32)).cuda()
    out = torch.empty_like(d)
    assert pm.lib().prc_poisson(d.data_ptr(), d.numel(), scale, seed, out.data_ptr(), None) == 0
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_counts_equal_the_cpu_restatement():
    rng = np.random.default_rng(7)
    mean = rng.uniform(0.0, 5.0, 6000).astype(np.float32)
    mean[:10] = [0, -1, np.nan, np.inf, 1e-30, 3.9, 4.0, 1e3, 2e4, 0.5]
    got = draw(mean, 10.0, 12345)
    want = np.array(so.poisson(mean.tolist(), 10.0, 12345), np.float32)
    assert np.mean(got == want) > 0.9995  # libm and CUDA may differ by an ulp in log/exp/lgamma
    assert np.all(np.abs(got - want) <= 1)


@pytest.mark.parametrize("lam", [0.3, 5.0, 9.99, 10.0, 30.0, 1e3, 1e5])
def test_poisson_moments(lam):
    n = 1 << 20
    x = draw(np.full(n, lam, np.float32), 1.0, 99).astype(np.float64)
    assert abs(x.mean() - lam) < 6 * math.sqrt(lam / n)
    assert abs(x.var() / lam - 1) < 6 * math.sqrt(2.0 / n) + 1e-3
    assert np.all(x == np.floor(x)) and x.min() >= 0


def test_determinism_and_seeds():
    mean = np.linspace(0, 40, 100000).astype(np.float32)
    a, b, c = draw(mean, 1.0, 5), draw(mean, 1.0, 5), draw(mean, 1.0, 6)
    assert np.array_equal(a, b) and not np.array_equal(a, c)


def test_device_data_helper_scales_to_the_total():
    rho, truth, sp = phantoms.small_phantom(seed=1)
    d = torch.from_numpy(truth).cuda()
    g = phantoms.poisson_counts_device(d, 1e6, seed=3).cpu().numpy()
    assert abs(g.sum() / 1e6 - 1) < 5 / math.sqrt(1e6)
    assert np.all(g[truth == 0] == 0)
