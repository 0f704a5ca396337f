"""CPU restatement of the device Poisson sampler (prc_poisson) -- TEST INFRASTRUCTURE ONLY.

Philox4x32-10 (Salmon, Moraes, Dror and Shaw, SC 2011) in exact integer arithmetic, pinned by
the published known-answer vectors; the per-voxel uniform stream (counter = index low, index
high, draw block, 0; key = seed low, seed high); inversion below a mean of 10 and PTRS
(Hormann 1993) above, in double precision.  Only tests/ use this module.
"""
from __future__ import annotations

import math

M0, M1, W0, W1 = 0xD2511F53, 0xCD9E8D57, 0x9E3779B9, 0xBB67AE85
MASK = 0xFFFFFFFF


def philox4x32_10(ctr, key):
    c0, c1, c2, c3 = ctr
    k0, k1 = key
    for _ in range(10):
        p0, p1 = M0 * c0, M1 * c2
        c0, c1, c2, c3 = ((p1 >> 32) ^ c1 ^ k0) & MASK, p1 & MASK, ((p0 >> 32) ^ c3 ^ k1) & MASK, p0 & MASK
        k0, k1 = (k0 + W0) & MASK, (k1 + W1) & MASK
    return c0, c1, c2, c3


class Uniforms:
    def __init__(self, index, seed):
        self.key = (seed & MASK, (seed >> 32) & MASK)
        self.lo, self.hi, self.block, self.bits, self.used = index & MASK, (index >> 32) & MASK, 0, (), 4

    def next(self):
        if self.used == 4:
            self.bits = philox4x32_10((self.lo, self.hi, self.block, 0), self.key)
            self.block += 1
            self.used = 0
        v = self.bits[self.used]
        self.used += 1
        return (v + 0.5) * (1.0 / 4294967296.0)


def poisson_sample(lam, u):
    if not lam > 0.0:
        return 0.0
    if lam < 10.0:
        x = u.next()
        p = math.exp(-lam)
        F, k = p, 0
        while x > F and k < 1000:
            k += 1
            p *= lam / k
            F += p
        return float(k)
    slam, loglam = math.sqrt(lam), math.log(lam)
    b = 0.931 + 2.53 * slam
    a = -0.059 + 0.02483 * b
    inv_alpha, v_r = 1.1239 + 1.1328 / (b - 3.4), 0.9277 - 3.6224 / (b - 2.0)
    for _ in range(1000):
        U, V = u.next() - 0.5, u.next()
        us = 0.5 - abs(U)
        k = math.floor((2.0 * a / us + b) * U + lam + 0.43)
        if us >= 0.07 and V <= v_r:
            return float(k)
        if k < 0 or (us < 0.013 and V > us):
            continue
        if math.log(V) + math.log(inv_alpha) - math.log(a / (us * us) + b) <= -lam + k * loglam - math.lgamma(k + 1.0):
            return float(k)
    return float(math.floor(lam + 0.5))


def poisson(mean, scale, seed):
    """Counts of every voxel, as prc_poisson draws them."""
    out = []
    for i, m in enumerate(mean):
        lam = scale * float(m) if math.isfinite(m) and m > 0 else 0.0
        out.append(poisson_sample(lam, Uniforms(i, seed)))
    return out
