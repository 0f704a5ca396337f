"""ctypes wrapper of the CPU oracle (oracle/prc_oracle.c) -- TEST INFRASTRUCTURE ONLY.

Imported by tests/, __graft_entry__.smoke() and the CPU-baseline leg of bench.py as the
checker.  It restates prc.cu (jlherraiz/PRC_MLEM) on the CPU in FP64 (analytic survival or an
FP64 table) and in float (the reference's 4097-entry table and float arithmetic).
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "build" / "liboracle.so"
NEAR = 125


class Params(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("sx", ctypes.c_float), ("sy", ctypes.c_float), ("sz", ctypes.c_float),
                ("cutoff", ctypes.c_float), ("support_rho", ctypes.c_float), ("air_cap", ctypes.c_float),
                ("n_rays", ctypes.c_int), ("n_branch", ctypes.c_int), ("br", (ctypes.c_float * 5) * 3),
                ("table_bins", ctypes.c_int), ("exact_range", ctypes.c_int), ("threads", ctypes.c_int)]


_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def lib():
    global _lib
    if _lib is None:
        if not LIB.is_file():
            build()
        _lib = ctypes.CDLL(str(LIB))
        _lib.oracle_count_deposits_f64.restype = ctypes.c_long
        _lib.oracle_count_deposits_f32.restype = ctypes.c_long
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def isotope(name: str):
    """(n_branch, branches[3,5] float32 with the weight fix, cutoff) as prc.cu computes them."""
    n = ctypes.c_int()
    br = np.zeros((3, 5), np.float32)
    cut = ctypes.c_float()
    if lib().oracle_isotope(name.encode(), ctypes.byref(n), _p(br), ctypes.byref(cut)) != 0:
        raise ValueError(f"unknown isotope {name}")
    return n.value, br, cut.value


class Problem:
    """One density map prepared as prc.cu:598-613 does: clamp >= 1e-3, support, active list.

    ``precision`` is 64 (FP64) or 32 (float, mirroring the device code).  For FP64,
    ``table_bins`` 0 means the analytic survival function.
    """

    def __init__(self, isotope_name, density, spacing, rays=128, support_rho=0.05, air_cap=50.0,
                 precision=64, table_bins=0, exact_range=False, threads=0):
        density = np.ascontiguousarray(density, dtype=np.float32)
        self.shape = density.shape
        nz, ny, nx = density.shape
        n_branch, br, cutoff = isotope(isotope_name)
        p = Params()
        p.nx, p.ny, p.nz = nx, ny, nz
        p.sx, p.sy, p.sz = spacing
        p.cutoff, p.support_rho, p.air_cap = cutoff, support_rho, air_cap
        p.n_rays, p.n_branch = rays, n_branch
        for b in range(3):
            for k in range(5):
                p.br[b][k] = float(br[b, k])
        p.table_bins, p.exact_range, p.threads = table_bins, int(exact_range), threads
        self.params = p
        self.cutoff = cutoff
        self.precision = precision
        self.dtype = np.float64 if precision == 64 else np.float32
        self.sfx = "f64" if precision == 64 else "f32"
        self.rho = np.maximum(density, np.float32(1e-3))
        self.support = (self.rho >= np.float32(support_rho))
        self.support_u8 = np.ascontiguousarray(self.support.astype(np.uint8))
        self.active = np.ascontiguousarray(np.flatnonzero(self.support.ravel()).astype(np.int32))
        self.W = None
        self.near = None

    @property
    def n_active(self) -> int:
        return len(self.active)

    def _fn(self, name):
        return getattr(lib(), f"oracle_{name}_{self.sfx}")

    def normalize(self):
        """W_s and the near-block weights (NormOp pass, prc.cu:420)."""
        self.W = np.zeros(self.n_active, self.dtype)
        self.near = np.zeros((self.n_active, NEAR), self.dtype)
        self._fn("normalize")(ctypes.byref(self.params), _p(self.rho), _p(self.active),
                              ctypes.c_int(self.n_active), _p(self.W), _p(self.near))
        return self

    def _ready(self):
        if self.W is None:
            self.normalize()

    def forward(self, f):
        self._ready()
        f = np.ascontiguousarray(f, dtype=self.dtype)
        out = np.zeros(self.shape, self.dtype)
        self._fn("forward")(ctypes.byref(self.params), _p(self.rho), _p(self.active), ctypes.c_int(self.n_active),
                            _p(self.W), _p(self.near), _p(f), _p(out))
        return out

    def adjoint(self, y, out=None):
        """A^T y on tissue voxels; ``out`` (default zeros) keeps its other voxels."""
        self._ready()
        y = np.ascontiguousarray(y, dtype=self.dtype)
        out = np.zeros(self.shape, self.dtype) if out is None else np.ascontiguousarray(out, dtype=self.dtype)
        self._fn("adjoint")(ctypes.byref(self.params), _p(self.rho), _p(self.active), ctypes.c_int(self.n_active),
                            _p(self.W), _p(self.near), _p(y), _p(out))
        return out

    def update(self, f, back, beta, gamma, eps):
        f = np.ascontiguousarray(f, dtype=self.dtype)
        back = np.ascontiguousarray(back, dtype=self.dtype)
        out = np.zeros(self.shape, self.dtype)
        t = ctypes.c_double if self.precision == 64 else ctypes.c_float
        self._fn("update")(ctypes.byref(self.params), _p(f), _p(back), _p(self.support_u8), _p(out),
                           t(beta), t(gamma), t(eps))
        return out

    def clamp_input(self, img):
        """prc.cu:604-612: activity clamped >= 0 and zeroed off the support."""
        img = np.maximum(np.asarray(img, dtype=np.float32), np.float32(0))
        return np.where(self.support, img, np.float32(0)).astype(np.float32)

    def correct(self, img, iterations, beta=0.2, gamma=20.0, accelerate=True):
        """The full MAP-EM loop of prc.cu:659-711 on the clamped, supported input."""
        self._ready()
        g = np.ascontiguousarray(self.clamp_input(img), dtype=self.dtype)
        out = np.zeros(self.shape, self.dtype)
        self._fn("correct")(ctypes.byref(self.params), _p(self.rho), _p(self.active), ctypes.c_int(self.n_active),
                            _p(self.support_u8), _p(self.W), _p(self.near), _p(g), ctypes.c_int(iterations),
                            ctypes.c_float(beta), ctypes.c_float(gamma), ctypes.c_int(int(accelerate)), _p(out))
        return out

    def count_deposits(self) -> int:
        self._ready()
        return int(self._fn("count_deposits")(ctypes.byref(self.params), _p(self.rho), _p(self.active),
                                              ctypes.c_int(self.n_active), _p(self.near)))


def survival(isotope_name, r, f32=False, table_bins=0):
    """S(r) as the projector evaluates it (analytic FP64, FP64 table, or the float table)."""
    prob = Problem(isotope_name, np.ones((1, 1, 1), np.float32), (1, 1, 1), table_bins=table_bins)
    r = np.ascontiguousarray(r, dtype=np.float64)
    s = np.zeros_like(r)
    lib().oracle_survival(ctypes.byref(prob.params), ctypes.c_int(int(f32)), _p(r), _p(s), ctypes.c_long(r.size))
    return s


def survival_table_f32(isotope_name):
    prob = Problem(isotope_name, np.ones((1, 1, 1), np.float32), (1, 1, 1))
    t = np.zeros(4097, np.float32)
    lib().oracle_survival_table_f32(ctypes.byref(prob.params), _p(t))
    return t, prob.cutoff


def ray(k, n, f32=False):
    x = np.zeros(3)
    d = np.zeros(3)
    lib().oracle_ray(ctypes.c_int(int(f32)), ctypes.c_int(k), ctypes.c_int(n), _p(x), _p(d))
    return x, d


def max_threads() -> int:
    return int(lib().oracle_max_threads())
