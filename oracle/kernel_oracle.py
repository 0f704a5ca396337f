"""FP64 homogeneous range kernel by radial quadrature — TEST INFRASTRUCTURE ONLY.

Restates the reference's own CPU computation, tests/reference.py of jlherraiz/PRC_MLEM:
``survival`` (tests/reference.py:20-26) and the voxel-averaged water kernel ``kernel``
(tests/reference.py:53-82), so that this CPU path can be timed where the reference's sources
are not present and can check the projector's homogeneous kernels.  Only tests/ and the CPU
leg of bench.py use it.

The quadrature: a point emitter at the centre of voxel (0, 0, 0) of a homogeneous medium of the
given density; path lengths up to ``cutoff_mm`` water-equivalent are cut into ``n_shells`` shells
with quadratic spacing; a shell's probability mass (the drop of the survival function across it)
is spread evenly over ``n_dirs`` Fibonacci-sphere directions at the shell's mid radius, and each
point is deposited into the (2h+1)^3 neighbourhood by trilinear weights (equivalent to uniform
emission over the source voxel with centre deposition).  Output is indexed [z, y, x].

Pinned by tests/golden/water_kernel.npz and tests/golden/range_model.npz, which the reference's
own module produced (tests/golden/make_kernel_golden.py).
"""
from __future__ import annotations

import numpy as np


def fix_weights(branches) -> np.ndarray:
    """Branch table [n, 5] = (weight, a, b, c, f) in FP64, with the weights made to sum to one by
    adjusting the lightest branch (the reference's FP64 weight fix, tests/reference.py:61)."""
    br = np.array(branches, dtype=np.float64).reshape(-1, 5)
    light = int(np.argmin(br[:, 0]))
    br[light, 0] += 1.0 - br[:, 0].sum()
    return br


def survival(branches, r) -> np.ndarray:
    """S(r) = sum_b w_b exp(-((a_b r)^(1+f_b) + (b_b r)^2.5 + (c_b r)^3.5)) in FP64, r in mm of
    water (prc.cu:65-72 in float, tests/reference.py:20-26 in FP64).  ``branches`` are used as given."""
    r = np.asarray(r, dtype=np.float64)
    total = np.zeros_like(r)
    for w, a, b, c, f in np.asarray(branches, dtype=np.float64).reshape(-1, 5):
        x = b * r
        y = c * r
        exponent = (a * r) ** (1.0 + f) + x * x * np.sqrt(x) + y * y * y * np.sqrt(y)
        total += w * np.exp(-exponent)
    return total


def fibonacci_directions(n: int) -> np.ndarray:
    """n unit vectors [n, 3] (x, y, z) on the golden-angle spiral, z from 1 - 1/n down to -1 + 1/n."""
    k = np.arange(n, dtype=np.float64)
    z = 1.0 - (2.0 * k + 1.0) / n
    golden = (1.0 + 5.0 ** 0.5) / 2.0
    phi = 2.0 * np.pi * k / golden
    rho = np.sqrt(1.0 - z * z)
    return np.stack([rho * np.cos(phi), rho * np.sin(phi), z], axis=1)


def shell_masses(branches, density: float, cutoff_mm: float, n_shells: int):
    """(mid radius in mm of medium, probability mass) of each quadrature shell."""
    t = np.linspace(0.0, 1.0, n_shells + 1)
    edges = cutoff_mm * t * t / density
    s = survival(branches, density * edges)
    return 0.5 * (edges[:-1] + edges[1:]), s[:-1] - s[1:]


def splat_trilinear(points: np.ndarray, weights: np.ndarray, half_width: int, out: np.ndarray) -> None:
    """Adds ``weights`` at ``points`` [m, 3] (voxel units, origin at the central voxel) to the flat
    (2h+1)^3 array ``out`` ([z, y, x] order) with trilinear weights; corners outside are dropped."""
    n = 2 * half_width + 1
    base = np.floor(points)
    frac = points - base
    cell = base.astype(np.int64) + half_width
    for corner in range(8):
        step = np.array([corner & 1, (corner >> 1) & 1, (corner >> 2) & 1])
        idx = cell + step
        share = weights * np.prod(np.where(step == 1, frac, 1.0 - frac), axis=1)
        keep = np.all((idx >= 0) & (idx < n), axis=1)
        flat = (idx[keep, 2] * n + idx[keep, 1]) * n + idx[keep, 0]
        out += np.bincount(flat, share[keep], n ** 3)


def water_kernel(branches, voxel_mm, half_width: int, density: float = 1.0, cutoff_mm: float = 30.0,
                 n_dirs: int = 1000, n_shells: int = 600, shells_per_chunk: int = 100) -> np.ndarray:
    """Voxel-averaged homogeneous kernel [z, y, x] of shape (2h+1)^3 (tests/reference.py:53-82).
    ``branches`` is the isotope's raw table; the FP64 weight fix is applied here."""
    br = fix_weights(branches)
    radius, mass = shell_masses(br, density, cutoff_mm, n_shells)
    dirs = fibonacci_directions(n_dirs)
    voxel = np.asarray(voxel_mm, dtype=np.float64)
    n = 2 * half_width + 1
    out = np.zeros(n ** 3)
    for s0 in range(0, n_shells, shells_per_chunk):
        r = radius[s0:s0 + shells_per_chunk]
        points = (r[:, None, None] * dirs[None] / voxel).reshape(-1, 3)
        weights = np.repeat(mass[s0:s0 + shells_per_chunk], n_dirs) / n_dirs
        splat_trilinear(points, weights, half_width, out)
    return out.reshape(n, n, n)


def table_branches(name: str) -> np.ndarray:
    """The isotope's coefficient table [n, 5] as the reference's quadrature reads it: the float32
    constants of prc.cu's table (tests/reference.py:7-17), widened to FP64.

    The oracle's C module returns them with prc.cu's float weight fix applied; that fix changes
    only the lightest weight, which the FP64 fix in ``water_kernel`` sets again from the others
    (to within 1e-16)."""
    from . import oracle
    nb, br, _ = oracle.isotope(name)
    return br[:nb].astype(np.float64)
