"""The CPU restatement of the device Poisson sampler, pinned to the published Philox4x32-10
known-answer vectors (no GPU)."""
import math

import numpy as np

from oracle import sampling_oracle as so

KAT = [((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
       ((0xFFFFFFFF,) * 4, (0xFFFFFFFF, 0xFFFFFFFF), (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
       ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
        (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1))]


def test_philox_known_answers():
    for ctr, key, want in KAT:
        assert so.philox4x32_10(ctr, key) == want


def test_oracle_moments_and_edge_cases():
    for lam in (0.7, 4.0, 25.0):
        x = np.array(so.poisson([1.0] * 4000, lam, seed=3))
        assert abs(x.mean() - lam) < 5 * math.sqrt(lam / 4000)
        assert abs(x.var() / lam - 1) < 0.15
        assert np.all(x == np.floor(x)) and np.all(x >= 0)
    assert so.poisson([0.0, -1.0, float("nan"), float("inf")], 5.0, seed=1) == [0.0, 0.0, 0.0, 0.0]
