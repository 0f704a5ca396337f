"""Seeded synthetic phantoms (density in g/cm3 and activity), arrays shaped (nz, ny, nx).

The reference ships no image data; its tests build phantoms from a seed
(tests/test_solver.py:143-157).  These generators produce the workloads the engine is
measured and tested on:

* :func:`solver_fixture`  -- the 16x14x12 anisotropic seed-72 fixture of the reference tests;
* :func:`small_phantom`   -- 32x32x24 at 2 mm, water cylinder, lung, bone (18F workload);
* :func:`scaled_small_phantom` -- the same geometry on another grid (surrogate evaluation);
* :func:`torso_phantom`   -- 128x128x159 clinical torso (68Ga workload);
* :func:`poisson_counts`  -- scales a blurred image to a total count and Poisson-samples it;
* :func:`poisson_counts_device` -- the same on the GPU (``prc_poisson``).

Blurring needs the projector, so callers do it (``Projector.forward_host``).
"""
from __future__ import annotations

import numpy as np

AIR = 0.0012
WATER = 1.0


def solver_fixture(seed: int = 72):
    """(rho, x, y, shape, spacing): the fixture of tests/test_solver.py:143-157.

    An ellipsoidal body of density U(0.2, 1.8) with a central air cavity on a 16x14x12 grid
    of 1.1 x 1.6 x 2.3 mm voxels; x and y are positive images on the support.
    """
    shape = (12, 14, 16)
    z, y, x = np.indices(shape)
    body = ((x - 7.5) / 6) ** 2 + ((y - 6.5) / 5) ** 2 + ((z - 5.5) / 5) ** 2 < 1
    cavity = (x - 7.5) ** 2 + (y - 6.5) ** 2 + (z - 5.5) ** 2 < 3
    rng = np.random.default_rng(seed)
    rho = np.where(body & ~cavity, rng.uniform(0.2, 1.8, shape), 0.001).astype(np.float32)
    support = rho >= 0.05
    xs = (rng.uniform(0.1, 2, shape) * support).astype(np.float32)
    ys = (rng.uniform(0.1, 2, shape) * support).astype(np.float32)
    return rho, xs, ys, shape, (1.1, 1.6, 2.3)


def _ellipsoid(shape, centre, radii):
    z, y, x = np.indices(shape, dtype=np.float64)
    cx, cy, cz = centre
    rx, ry, rz = radii
    return ((x - cx) / rx) ** 2 + ((y - cy) / ry) ** 2 + ((z - cz) / rz) ** 2 <= 1.0


def small_phantom(seed: int = 1):
    """(rho, truth, spacing) on a 32x32x24 grid of 2 mm voxels.

    Air outside; a water elliptic cylinder (semi-axes 13 x 10 voxels) through all z; a lung
    ellipsoid (0.30) at (10, 16, 12) with radii (5, 6, 8); a bone sphere (1.85) at (22, 16, 12)
    of radius 3.  Activity 1.0 in the body plus 6 spheres (radius U[2, 4] voxels, centre
    uniform in the body, amplitude U[2, 10]).
    """
    nx, ny, nz = 32, 32, 24
    shape = (nz, ny, nx)
    z, y, x = np.indices(shape, dtype=np.float64)
    cx, cy = (nx - 1) / 2, (ny - 1) / 2
    body = ((x - cx) / 13) ** 2 + ((y - cy) / 10) ** 2 <= 1.0
    rho = np.full(shape, AIR)
    rho[body] = WATER
    rho[_ellipsoid(shape, (10, 16, 12), (5, 6, 8)) & body] = 0.30
    rho[_ellipsoid(shape, (22, 16, 12), (3, 3, 3)) & body] = 1.85
    rng = np.random.default_rng(seed)
    truth = body.astype(np.float64)
    inside = np.argwhere(body)
    for _ in range(6):
        r = rng.uniform(2, 4)
        zc, yc, xc = inside[rng.integers(len(inside))] + rng.uniform(-0.5, 0.5, 3)
        truth[_ellipsoid(shape, (xc, yc, zc), (r, r, r)) & body] += rng.uniform(2, 10)
    return rho.astype(np.float32), truth.astype(np.float32), (2.0, 2.0, 2.0)


def scaled_small_phantom(seed: int = 1, shape=(159, 128, 128), spacing=(0.776, 0.776, 0.795)):
    """(rho, truth, spacing): the small phantom's geometry stretched onto another grid.

    Every position and radius of :func:`small_phantom` (given in voxels of its 32x32x24 grid) is
    scaled by the grid ratio per axis (lesion radii by the mean ratio), with the same seeded
    draws, so shape (24, 32, 32) with 2 mm voxels reproduces :func:`small_phantom` exactly.  At
    128x128x159 it is the learned surrogate's evaluation phantom: one water cylinder, one lung
    ellipsoid and one bone sphere, simpler than the torso.
    """
    nz, ny, nx = shape
    sx, sy, sz = nx / 32.0, ny / 32.0, nz / 24.0
    sr = (sx + sy + sz) / 3.0
    z, y, x = np.indices(shape, dtype=np.float64)
    cx, cy = (nx - 1) / 2, (ny - 1) / 2
    body = ((x - cx) / (13 * sx)) ** 2 + ((y - cy) / (10 * sy)) ** 2 <= 1.0
    rho = np.full(shape, AIR)
    rho[body] = WATER
    rho[_ellipsoid(shape, (10 * sx, 16 * sy, 12 * sz), (5 * sx, 6 * sy, 8 * sz)) & body] = 0.30
    rho[_ellipsoid(shape, (22 * sx, 16 * sy, 12 * sz), (3 * sx, 3 * sy, 3 * sz)) & body] = 1.85
    rng = np.random.default_rng(seed)
    truth = body.astype(np.float64)
    inside = np.argwhere(body)
    for _ in range(6):
        r = rng.uniform(2, 4) * sr
        zc, yc, xc = inside[rng.integers(len(inside))] + rng.uniform(-0.5, 0.5, 3)
        truth[_ellipsoid(shape, (xc, yc, zc), (r, r, r)) & body] += rng.uniform(2, 10)
    return rho.astype(np.float32), truth.astype(np.float32), tuple(spacing)


def torso_phantom(seed: int = 2, shape=(159, 128, 128)):
    """(rho, truth, spacing): a clinical-size torso on 128x128x159 voxels of 0.776x0.776x0.795 mm.

    Density: air outside; a water ellipse (semi-axes 55 x 40 voxels) through all z; two lung
    ellipsoids (0.26); a spine cylinder (1.4, radius 6 voxels); 8 rib arcs (1.85) along the
    body wall.  Activity: background 1.0 in the body, a liver ellipsoid at 4.0 and 12 lesions
    (radius U[1.5, 6] voxels, contrast U[3, 12] times background), half of them in lung.
    """
    nz, ny, nx = shape
    z, y, x = np.indices(shape, dtype=np.float64)
    cx, cy = (nx - 1) / 2, (ny - 1) / 2
    sx = nx / 128.0
    sy = ny / 128.0
    sz = nz / 159.0
    ax, ay = 55 * sx, 40 * sy
    body = ((x - cx) / ax) ** 2 + ((y - cy) / ay) ** 2 <= 1.0
    rho = np.full(shape, AIR)
    rho[body] = WATER
    lungs = []
    for side in (-1, 1):
        lung = _ellipsoid(shape, (cx + side * 26 * sx, cy - 4 * sy, 0.62 * nz), (17 * sx, 24 * sy, 0.33 * nz))
        lungs.append(lung & body)
        rho[lung & body] = 0.26
    spine = ((x - cx) ** 2 + (y - (cy + 28 * sy)) ** 2 <= (6 * min(sx, sy)) ** 2) & body
    rho[spine] = 1.4
    # rib arcs: thin elliptic shells just inside the body wall, 8 levels in z
    shell = np.abs(np.sqrt(((x - cx) / (ax - 4 * sx)) ** 2 + ((y - cy) / (ay - 4 * sy)) ** 2) - 1.0) <= 0.035
    for k in range(8):
        zc = nz * (0.42 + 0.065 * k)
        arc = shell & (np.abs(z - zc) <= 1.2 * sz) & (y < cy + 20 * sy) & body
        rho[arc] = 1.85
    rng = np.random.default_rng(seed)
    truth = body.astype(np.float64)
    liver = _ellipsoid(shape, (cx - 22 * sx, cy + 4 * sy, 0.3 * nz), (24 * sx, 20 * sy, 0.17 * nz)) & body
    truth[liver] = 4.0
    lung_any = lungs[0] | lungs[1]
    lung_idx = np.argwhere(lung_any)
    soft_idx = np.argwhere(body & ~lung_any)
    for k in range(12):
        pool = lung_idx if k % 2 == 0 and len(lung_idx) else soft_idx
        zc, yc, xc = pool[rng.integers(len(pool))] + rng.uniform(-0.5, 0.5, 3)
        r = rng.uniform(1.5, 6)
        contrast = rng.uniform(3, 12)
        lesion = _ellipsoid(shape, (xc, yc, zc), (r, r, r)) & body
        truth[lesion] = contrast
    return rho.astype(np.float32), truth.astype(np.float32), (0.776, 0.776, 0.795)


def poisson_counts_device(d_blurred, total_counts: float, seed: int = 0):
    """Device form of :func:`poisson_counts`: a float32 CUDA tensor of counts drawn on the GPU
    (``prc_poisson``: Philox4x32-10 keyed by ``seed``, inversion below a mean of 10, PTRS above)
    after scaling ``d_blurred`` (a float32 CUDA tensor, negative values count as 0) to
    ``total_counts``.  Counts differ from the host form's (another random stream) but follow
    the same distribution.  The sampling is enqueued on torch's current stream."""
    import ctypes
    import torch
    from . import PrcError, lib
    d = d_blurred.contiguous()
    if d.dtype != torch.float32 or not d.is_cuda:
        raise ValueError("expected a float32 CUDA tensor")
    total = float(torch.clamp(d, min=0).double().sum().item())
    out = torch.empty_like(d)
    scale = total_counts / total if total > 0 else 0.0
    rc = lib().prc_poisson(d.data_ptr(), d.numel(), scale, int(seed), out.data_ptr(),
                           torch.cuda.current_stream(d.device).cuda_stream)
    if rc != 0:
        raise PrcError(rc, lib().prc_last_error().decode())
    return out


def poisson_counts(blurred: np.ndarray, total_counts: float, seed: int = 0) -> np.ndarray:
    """Scale ``blurred`` to ``total_counts`` and draw Poisson counts (float32)."""
    blurred = np.maximum(np.asarray(blurred, dtype=np.float64), 0.0)
    lam = blurred * (total_counts / blurred.sum())
    return np.random.default_rng(seed).poisson(lam).astype(np.float32)
