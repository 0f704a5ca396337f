"""B200 positron-range correction: Python binding of the C ABI in include/prc_b200.h.

The reference (jlherraiz/PRC_MLEM) has no library API; its operator seam is
``class Projector`` (prc.cu:403-450) with ``forward``/``adjoint`` and the MAP-EM loop of
``main`` (prc.cu:659-711).  :class:`Projector` mirrors that seam over ``libprc_b200.so``
(ctypes, no torch types in the ABI).  Device arrays are passed as torch CUDA tensors or raw
device pointers; torch only provides device memory and streams.

There is no CPU fallback: if the shared library has not been built, loading it raises.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

PKG_DIR = Path(__file__).resolve().parent
# PRC_B200_LIB selects another build of the library (for example one compiled with other
# tuning constants); the default is the in-tree build.
LIB_PATH = Path(os.environ.get("PRC_B200_LIB") or PKG_DIR / "lib" / "libprc_b200.so")
CLI_PATH = PKG_DIR / "bin" / "prc"
HEADER_PATH = PKG_DIR.parent / "include" / "prc_b200.h"

PRC_OK = 0
PRC_ERR_ARGUMENT = 1
PRC_PRECISION_FP32 = 0
PRC_PRECISION_BF16 = 1
PRC_PRECISION_BF16_VOLUMES = 2
PRC_PRECISION_FP24 = 3
PRC_CACHE_NONE = 0
PRC_CACHE_NEAR = 1
PRC_CACHE_FULL = 2
PRC_CACHE_SOURCE_MAJOR = 3
PRC_TILE_AUTO, PRC_TILE_8x2x2, PRC_TILE_16x2x1, PRC_TILE_32x1x1, PRC_TILE_4x4x2, PRC_TILE_16x1x2 = range(6)
TILE_SHAPES = {PRC_TILE_8x2x2: (8, 2, 2), PRC_TILE_16x2x1: (16, 2, 1), PRC_TILE_32x1x1: (32, 1, 1),
               PRC_TILE_4x4x2: (4, 4, 2), PRC_TILE_16x1x2: (16, 1, 2)}
ISOTOPES = ("11C", "13N", "15O", "18F", "64Cu", "68Ga", "82Rb", "124I")


class PrcError(RuntimeError):
    """A C-ABI call returned a non-zero status; ``code`` is the PRC_ERR_* value."""

    def __init__(self, code: int, message: str):
        super().__init__(f"prc error {code}: {message}")
        self.code = code


class Geometry(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("dx", ctypes.c_float), ("dy", ctypes.c_float), ("dz", ctypes.c_float)]


class Options(ctypes.Structure):
    _fields_ = [("rays", ctypes.c_int), ("support_rho", ctypes.c_float), ("air_cap_mm", ctypes.c_float),
                ("exact_range", ctypes.c_int), ("cache", ctypes.c_int), ("precision", ctypes.c_int),
                ("tile", ctypes.c_int)]


_P = ctypes.c_void_p
_F = ctypes.POINTER(ctypes.c_float)
_SIGNATURES = {
    "prc_default_options": (None, [ctypes.POINTER(Options)]),
    "prc_isotope_cutoff": (ctypes.c_int, [ctypes.c_char_p, _F]),
    "prc_isotope_count": (ctypes.c_int, []),
    "prc_isotope_name": (ctypes.c_char_p, [ctypes.c_int]),
    "prc_create": (ctypes.c_int, [ctypes.POINTER(Geometry), ctypes.c_char_p, ctypes.POINTER(Options), _P,
                                  ctypes.POINTER(_P)]),
    "prc_destroy": (None, [_P]),
    "prc_active_count": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int64)]),
    "prc_cutoff": (ctypes.c_int, [_P, _F]),
    "prc_device_bytes": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int64)]),
    "prc_cache_mode": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int64),
                                      ctypes.POINTER(ctypes.c_int64)]),
    "prc_stream": (_P, [_P]),
    "prc_forward": (ctypes.c_int, [_P, _P, _P, _P]),
    "prc_adjoint": (ctypes.c_int, [_P, _P, _P, _P]),
    "prc_em_begin": (ctypes.c_int, [_P, _P, _P]),
    "prc_em_iterate": (ctypes.c_int, [_P, ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_int, _P]),
    "prc_em_estimate": (ctypes.c_int, [_P, _P, _P]),
    "prc_em_run": (ctypes.c_int, [_P, _P, _P, ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_int, _P]),
    "prc_em_run_host": (ctypes.c_int, [_P, _P, _P, ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_int]),
    "prc_forward_frames": (ctypes.c_int, [_P, ctypes.c_int, _P, _P, _P]),
    "prc_adjoint_frames": (ctypes.c_int, [_P, ctypes.c_int, _P, _P, _P]),
    "prc_em_run_frames": (ctypes.c_int, [_P, ctypes.c_int, _P, _P, ctypes.c_int, ctypes.c_float, ctypes.c_float,
                                         ctypes.c_int, _P]),
    "prc_em_begin_host": (ctypes.c_int, [_P, _P]),
    "prc_em_estimate_host": (ctypes.c_int, [_P, _P]),
    "prc_forward_host": (ctypes.c_int, [_P, _P, _P]),
    "prc_adjoint_host": (ctypes.c_int, [_P, _P, _P]),
    "prc_sum": (ctypes.c_int, [_P, _P, ctypes.POINTER(ctypes.c_double), _P]),
    "prc_count_deposits": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int64)]),
    "prc_synchronize": (ctypes.c_int, [_P]),
    "prc_launch_count": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int64)]),
    "prc_tile": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int)]),
    "prc_tune_tile": (ctypes.c_int, [ctypes.POINTER(Geometry), ctypes.c_char_p, ctypes.POINTER(Options), _P,
                                     ctypes.POINTER(ctypes.c_int)]),
    "prc_wait_selftest": (ctypes.c_int, [_P, ctypes.c_int]),
    "prc_sum_static": (ctypes.c_int, [_P, ctypes.c_int64, _P, _P]),
    "prc_create_surrogate": (ctypes.c_int, [ctypes.POINTER(Geometry), ctypes.c_char_p, ctypes.POINTER(Options), _P,
                                            _P, ctypes.c_float, ctypes.c_float, ctypes.POINTER(ctypes.c_int64),
                                            ctypes.POINTER(_P)]),
"prc_batch_create": (ctypes.c_int, [ctypes.c_int, _P, ctypes.POINTER(Options), _P, ctypes.c_float,
                                        ctypes.c_float, ctypes.POINTER(_P)]),
    "prc_batch_destroy": (None, [_P]),
    "prc_batch_em_run": (ctypes.c_int, [_P, _P, _P, ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_int]),
    "prc_batch_synchronize": (ctypes.c_int, [_P]),
    "prc_batch_stream": (_P, [_P]),
    "prc_batch_frame": (ctypes.c_int, [_P, ctypes.c_int, ctypes.POINTER(_P)]),
    "prc_batch_warps": (ctypes.c_int, [_P]),
    "prc_batch_profile": (ctypes.c_int, [_P, _P, _P, ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                         ctypes.POINTER(ctypes.c_int)]),
    "prc_nn_gemm_bf16": (ctypes.c_int, [_P, _P, _P, ctypes.c_int, ctypes.c_int, ctypes.c_int, _P, _P]),
    "prc_nn_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_P)]),
    "prc_nn_destroy": (None, [_P]),
    "prc_nn_param_count": (ctypes.c_int64, []),
    "prc_nn_patch_side": (ctypes.c_int, []),
    "prc_nn_set_params": (ctypes.c_int, [_P, _P]),
    "prc_nn_get": (ctypes.c_int, [_P, ctypes.c_int, _P]),
    "prc_nn_forward": (ctypes.c_int, [_P, _P, ctypes.c_int, _P, _P]),
    "prc_nn_backward": (ctypes.c_int, [_P, _P, ctypes.c_int, ctypes.c_float, ctypes.POINTER(ctypes.c_double), _P]),
    "prc_nn_make_samples": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_float, _P,
                                           ctypes.c_uint64, ctypes.c_int, _P, _P, ctypes.c_float, ctypes.c_float,
                                           _P]),
    "prc_eval_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _P, _P, _P, ctypes.c_int, _P, _P,
                                       _P, ctypes.c_double, ctypes.POINTER(ctypes.c_void_p)]),
    "prc_eval_sums": (ctypes.c_int, [_P, _P, _P, _P]),
    "prc_eval_sums_f64": (ctypes.c_int, [_P, _P, _P, _P]),
    "prc_eval_destroy": (None, [_P]),
    "prc_poisson": (ctypes.c_int, [_P, ctypes.c_int64, ctypes.c_double, ctypes.c_uint64, _P, _P]),
    "prc_timing": (ctypes.c_int, [_P, ctypes.c_int]),
    "prc_timing_read": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int64),
                                       ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int64)]),
    "prc_last_error": (ctypes.c_char_p, []),
    "prc_host_alloc": (ctypes.c_int, [ctypes.c_size_t, ctypes.POINTER(_P)]),
    "prc_host_free": (None, [_P]),
}

class Frame(ctypes.Structure):
    _fields_ = [("geometry", Geometry), ("isotope", ctypes.c_char_p), ("density_host", ctypes.c_void_p)]


_lib_handle = None


def lib() -> ctypes.CDLL:
    """The loaded ``libprc_b200.so``; raises if it was not built (no fallback exists)."""
    global _lib_handle
    if _lib_handle is None:
        if not LIB_PATH.is_file():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C {PKG_DIR / 'csrc'}` "
                               "or __graft_entry__.build(); there is no CPU fallback")
        handle = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib_handle = handle
    return _lib_handle


def _check(rc: int) -> None:
    if rc != PRC_OK:
        raise PrcError(rc, lib().prc_last_error().decode())


def isotope_cutoff(isotope: str) -> float:
    """99.95 % water-equivalent range cutoff [mm] (prc.cu:83-91); host only."""
    c = ctypes.c_float()
    _check(lib().prc_isotope_cutoff(isotope.encode(), ctypes.byref(c)))
    return c.value


def default_options() -> Options:
    o = Options()
    lib().prc_default_options(ctypes.byref(o))
    return o


def _ptr(x) -> int:
    """Device pointer of a torch CUDA tensor (or an int pointer)."""
    if isinstance(x, int):
        return x
    if not x.is_cuda or x.dtype.itemsize != 4 or not x.is_contiguous():
        raise ValueError("expected a contiguous float32 CUDA tensor")
    return x.data_ptr()


def _host(a: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


def tune_tile(isotope: str, density: np.ndarray, spacing, rays: int = 128, support_rho: float = 0.05,
              air_cap_mm: float = 50.0, cache: int = PRC_CACHE_FULL, precision: int = PRC_PRECISION_FP32) -> int:
    """The source tile the autotuner finds fastest for this configuration (prc_tune_tile); later
    Projectors of the same configuration with tile=PRC_TILE_AUTO use it."""
    density = _host(density)
    nz, ny, nx = density.shape
    geo = Geometry(nx, ny, nz, *(float(s) for s in spacing))
    opts = default_options()
    opts.rays, opts.support_rho, opts.air_cap_mm = rays, support_rho, air_cap_mm
    opts.cache, opts.precision = int(cache), int(precision)
    t = ctypes.c_int()
    _check(lib().prc_tune_tile(ctypes.byref(geo), isotope.encode(), ctypes.byref(opts), density.ctypes.data,
                               ctypes.byref(t)))
    return t.value


class Projector:
    """Heterogeneous range-blur operator A for one density map (prc.cu:403-450).

    ``density`` is a float array of shape (nz, ny, nx) in g/cm3; ``spacing`` is (dx, dy, dz)
    in mm.  Construction runs the normalisation pass on the current CUDA device.
    """

    def __init__(self, isotope: str, density: np.ndarray, spacing, rays: int = 128, support_rho: float = 0.05,
                 air_cap_mm: float = 50.0, exact_range: bool = False, cache: int = PRC_CACHE_FULL,
                 precision: int = PRC_PRECISION_FP32, surrogate=None, target_scale: float = 1.0,
                 fallback_nrmse: float = 0.0, tile: int = PRC_TILE_AUTO):
        """surrogate: None for the plain projector; a trained network (prc_mlem_b200.surrogate.Network)
        or the string "traced" for the radial coefficient field (prc_create_surrogate).
        ``fallbacks`` then counts the (source, far ray) pairs the tracer kept on exact weights."""
        density = _host(density)
        if density.ndim != 3:
            raise ValueError("density must be a (nz, ny, nx) array")
        nz, ny, nx = density.shape
        self.shape = density.shape
        self.spacing = tuple(float(s) for s in spacing)
        self.isotope = isotope
        geo = Geometry(nx, ny, nz, *self.spacing)
        opts = default_options()
        opts.rays, opts.support_rho, opts.air_cap_mm = rays, support_rho, air_cap_mm
        opts.exact_range, opts.cache, opts.precision = int(exact_range), int(cache), int(precision)
        opts.tile = int(tile)
        h = _P()
        self.fallbacks = 0
        if surrogate is None:
            _check(lib().prc_create(ctypes.byref(geo), isotope.encode(), ctypes.byref(opts),
                                    density.ctypes.data, ctypes.byref(h)))
        else:
            net = None if isinstance(surrogate, str) else surrogate.handle
            fb = ctypes.c_int64()
            _check(lib().prc_create_surrogate(ctypes.byref(geo), isotope.encode(), ctypes.byref(opts),
                                              density.ctypes.data, net, target_scale, fallback_nrmse,
                                              ctypes.byref(fb), ctypes.byref(h)))
            self.fallbacks = fb.value
        self._h = h
        self.support = np.maximum(density, np.float32(1e-3)) >= np.float32(support_rho)

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().prc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self) -> int:
        return self._h.value

    @property
    def n_active(self) -> int:
        v = ctypes.c_int64()
        _check(lib().prc_active_count(self._h, ctypes.byref(v)))
        return v.value

    @property
    def cutoff(self) -> float:
        v = ctypes.c_float()
        _check(lib().prc_cutoff(self._h, ctypes.byref(v)))
        return v.value

    @property
    def device_bytes(self) -> int:
        v = ctypes.c_int64()
        _check(lib().prc_device_bytes(self._h, ctypes.byref(v)))
        return v.value

    @property
    def cache_mode(self) -> tuple[int, int, int]:
        """(PRC_CACHE_* in effect, source-major field entries, target-major field entries)."""
        m, e, t = ctypes.c_int(), ctypes.c_int64(), ctypes.c_int64()
        _check(lib().prc_cache_mode(self._h, ctypes.byref(m), ctypes.byref(e), ctypes.byref(t)))
        return m.value, e.value, t.value

    @property
    def stream(self) -> int:
        return lib().prc_stream(self._h) or 0

    def timing(self, enable: bool) -> None:
        """Bracket every projection launch with CUDA events (True starts a new measurement)."""
        _check(lib().prc_timing(self._h, int(bool(enable))))

    def timing_read(self) -> dict:
        """Summed device milliseconds and launch counts of the projections since timing(True)."""
        fm, am, fn, an = ctypes.c_double(), ctypes.c_double(), ctypes.c_int64(), ctypes.c_int64()
        _check(lib().prc_timing_read(self._h, ctypes.byref(fm), ctypes.byref(fn), ctypes.byref(am), ctypes.byref(an)))
        return {"forward_ms": fm.value, "forward_launches": fn.value, "adjoint_ms": am.value,
                "adjoint_launches": an.value}

    # device-memory operators -------------------------------------------------------------
    def forward(self, d_in, d_out, stream=None) -> None:
        """d_out = A d_in (overwritten) -- Projector::forward, prc.cu:430-434."""
        _check(lib().prc_forward(self._h, _ptr(d_in), _ptr(d_out), stream))

    def adjoint(self, d_in, d_out, stream=None) -> None:
        """d_out[s] = (A^T d_in)[s] on tissue voxels -- Projector::adjoint, prc.cu:436."""
        _check(lib().prc_adjoint(self._h, _ptr(d_in), _ptr(d_out), stream))

    def em_begin(self, d_g, stream=None) -> None:
        _check(lib().prc_em_begin(self._h, _ptr(d_g), stream))

    def em_iterate(self, n: int, beta: float, gamma: float, accelerate: bool, stream=None) -> None:
        _check(lib().prc_em_iterate(self._h, n, beta, gamma, int(accelerate), stream))

    def em_estimate(self, d_out, stream=None) -> None:
        _check(lib().prc_em_estimate(self._h, _ptr(d_out), stream))

    def correct(self, d_g, d_out, iterations: int, beta: float = 0.2, gamma: float = 20.0,
                accelerate: bool = True, stream=None) -> None:
        """MAP-EM correction of d_g into d_out (prc.cu:659-711), fully on device.

        Enqueued on ``stream`` (default: the engine's own stream) and asynchronous to the host
        and to torch's current stream: call ``synchronize()`` before reading d_out elsewhere."""
        _check(lib().prc_em_run(self._h, _ptr(d_g), _ptr(d_out), iterations, beta, gamma, int(accelerate), stream))

    # frames sharing this projector (one density map, many activity volumes) ---------------
    @staticmethod
    def _pointers(vols):
        return (ctypes.c_void_p * len(vols))(*[_ptr(x) for x in vols])

    def forward_frames(self, d_ins, d_outs, stream=None) -> None:
        """d_outs[i] = A d_ins[i] for every frame; the stored field is read once per pass of up to
        four frames.  Each result equals ``forward(d_ins[i], d_outs[i])`` bit for bit."""
        _check(lib().prc_forward_frames(self._h, len(d_ins), self._pointers(d_ins), self._pointers(d_outs), stream))

    def adjoint_frames(self, d_ins, d_outs, stream=None) -> None:
        """d_outs[i][s] = (A^T d_ins[i])[s] on tissue voxels for every frame."""
        _check(lib().prc_adjoint_frames(self._h, len(d_ins), self._pointers(d_ins), self._pointers(d_outs), stream))

    def correct_frames(self, d_gs, d_outs, iterations: int, beta: float = 0.2, gamma: float = 20.0,
                       accelerate: bool = True, stream=None) -> None:
        """MAP-EM correction of every frame (one ``correct`` per frame, prc.cu:659-711) with the
        projections of all frames done together.  Asynchronous like ``correct``."""
        _check(lib().prc_em_run_frames(self._h, len(d_gs), self._pointers(d_gs), self._pointers(d_outs), iterations,
                                       beta, gamma, int(accelerate), stream))

    def synchronize(self) -> None:
        _check(lib().prc_synchronize(self._h))

    def sum(self, d_x) -> float:
        v = ctypes.c_double()
        _check(lib().prc_sum(self._h, _ptr(d_x), ctypes.byref(v), None))
        return v.value

    @property
    def tile(self) -> int:
        """The source tile (PRC_TILE_*) of the stored field."""
        v = ctypes.c_int()
        _check(lib().prc_tile(self._h, ctypes.byref(v)))
        return v.value

    @property
    def launches(self) -> int:
        """Kernels this handle has enqueued since it was created (prc_launch_count)."""
        v = ctypes.c_int64()
        _check(lib().prc_launch_count(self._h, ctypes.byref(v)))
        return v.value

    def count_deposits(self) -> int:
        v = ctypes.c_int64()
        _check(lib().prc_count_deposits(self._h, ctypes.byref(v)))
        return v.value

    # host-memory forms -------------------------------------------------------------------
    def forward_host(self, x: np.ndarray) -> np.ndarray:
        x = _host(x)
        out = np.empty_like(x)
        _check(lib().prc_forward_host(self._h, x.ctypes.data, out.ctypes.data))
        return out

    def adjoint_host(self, y: np.ndarray) -> np.ndarray:
        y = _host(y)
        out = np.empty_like(y)
        _check(lib().prc_adjoint_host(self._h, y.ctypes.data, out.ctypes.data))
        return out

    def correct_host(self, g: np.ndarray, iterations: int, beta: float = 0.2, gamma: float = 20.0,
                     accelerate: bool = True) -> np.ndarray:
        g = _host(g)
        out = np.empty_like(g)
        _check(lib().prc_em_run_host(self._h, g.ctypes.data, out.ctypes.data, iterations, beta, gamma,
                                     int(accelerate)))
        return out


class Batch:
    """Many frames (density maps of any grid, isotope) corrected together: one launch per MAP-EM
    phase for all frames, the schedule captured into a CUDA graph (prc_batch_*).

    frames: list of (isotope, density (nz, ny, nx), spacing (dx, dy, dz)).  Frames that pass the
    same density array object with the same isotope and spacing (the frames of one study) share
    one projector.
    """

    def __init__(self, frames, rays: int = 128, support_rho: float = 0.05, cache: int = PRC_CACHE_FULL,
                 precision: int = PRC_PRECISION_FP32, surrogate=None, target_scale: float = 1.0,
                 fallback_nrmse: float = 0.0):
        self._keep = []
        arr = (Frame * len(frames))()
        self.shapes = []
        converted = {}  # one host array per distinct density object, so shared maps stay shared
        for i, (iso, rho, spacing) in enumerate(frames):
            rho = converted.setdefault(id(rho), _host(rho))
            nz, ny, nx = rho.shape
            self._keep.append(rho)
            self.shapes.append(rho.shape)
            iso_b = iso.encode()
            self._keep.append(iso_b)
            arr[i] = Frame(Geometry(nx, ny, nz, *[float(s) for s in spacing]), iso_b, rho.ctypes.data)
        opts = default_options()
        opts.rays, opts.support_rho, opts.cache, opts.precision = rays, support_rho, int(cache), int(precision)
        h = _P()
        _check(lib().prc_batch_create(len(frames), ctypes.cast(arr, _P), ctypes.byref(opts),
                                      None if surrogate is None else surrogate.handle, target_scale,
                                      fallback_nrmse, ctypes.byref(h)))
        self._h = h
        self._keep = []

    def close(self):
        if getattr(self, "_h", None):
            lib().prc_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self) -> int:
        return lib().prc_batch_stream(self._h) or 0

    @property
    def warps(self) -> int:
        return lib().prc_batch_warps(self._h)

    def correct(self, d_gs, d_outs, iterations: int, beta: float = 0.2, gamma: float = 20.0,
                accelerate: bool = True) -> None:
        """Enqueues a MAP-EM run of every frame (device tensors, one per frame)."""
        n = len(d_gs)
        g = (ctypes.c_void_p * n)(*[_ptr(x) for x in d_gs])
        o = (ctypes.c_void_p * n)(*[_ptr(x) for x in d_outs])
        _check(lib().prc_batch_em_run(self._h, g, o, iterations, beta, gamma, int(accelerate)))

    def profile(self, d_gs, d_outs, iterations: int, beta: float = 0.2, gamma: float = 20.0,
                accelerate: bool = True) -> dict:
        """Device time of one graph replay of the run and the summed device time of the same
        launches made one by one (prc_batch_profile)."""
        n = len(d_gs)
        g = (ctypes.c_void_p * n)(*[_ptr(x) for x in d_gs])
        o = (ctypes.c_void_p * n)(*[_ptr(x) for x in d_outs])
        gm, lm, nl = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        _check(lib().prc_batch_profile(self._h, g, o, iterations, beta, gamma, int(accelerate), ctypes.byref(gm),
                                       ctypes.byref(lm), ctypes.byref(nl)))
        return {"graph_ms": gm.value, "launches_ms": lm.value, "launches": nl.value}

    def synchronize(self) -> None:
        _check(lib().prc_batch_synchronize(self._h))

    def frame_handle(self, i: int) -> int:
        h = _P()
        _check(lib().prc_batch_frame(self._h, i, ctypes.byref(h)))
        return h.value

    def device_bytes(self, i: int) -> int:
        """Device memory frame i's handle allocated itself (a frame sharing another frame's
        projector counts only its own MAP-EM volumes and scratch)."""
        v = ctypes.c_int64()
        _check(lib().prc_device_bytes(self.frame_handle(i), ctypes.byref(v)))
        return v.value

    def forward(self, i: int, d_in, d_out) -> None:
        """Forward projection of frame i with its own projector (its handle's stream)."""
        h = self.frame_handle(i)
        _check(lib().prc_forward(h, _ptr(d_in), _ptr(d_out), None))
        _check(lib().prc_synchronize(h))

    def cache_mode(self, i: int):
        m, e, t = ctypes.c_int(), ctypes.c_int64(), ctypes.c_int64()
        _check(lib().prc_cache_mode(self.frame_handle(i), ctypes.byref(m), ctypes.byref(e), ctypes.byref(t)))
        return m.value, e.value, t.value


def header_symbols() -> list[str]:
    """Every function the public headers (include/*.h) declare (used to check the exports)."""
    import re
    names = set()
    for header in sorted(HEADER_PATH.parent.glob("*.h")):
        names.update(re.findall(r"^\s*(?:[\w\s\*]+?)\b(prc_\w+)\s*\(", header.read_text(), re.M))
    return sorted(names)
