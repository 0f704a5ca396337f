"""The C-ABI library without a GPU: it loads, exports every function include/prc_b200.h
declares, and its host-only entry points (isotope table, cutoffs, argument validation that
precedes any CUDA call) behave."""
import ctypes
import subprocess

import numpy as np
import pytest

import prc_mlem_b200 as pm


def test_library_exports_every_header_symbol():
    declared = pm.header_symbols()
    assert len(declared) >= 25
    out = subprocess.run(["nm", "-D", "--defined-only", str(pm.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = [s for s in declared if s not in exported]
    assert not missing, missing
    lib = pm.lib()
    for s in declared:
        assert getattr(lib, s)


def test_isotopes_and_cutoffs_match_oracle(oracle_mod):
    lib = pm.lib()
    names = [lib.prc_isotope_name(i).decode() for i in range(lib.prc_isotope_count())]
    assert tuple(names) == pm.ISOTOPES
    assert lib.prc_isotope_name(99) is None
    for iso in names:
        _, _, cutoff = oracle_mod.isotope(iso)
        assert pm.isotope_cutoff(iso) == cutoff  # bit-identical float bisection (prc.cu:83-91)


def test_default_options_are_the_reference_defaults():
    o = pm.default_options()
    assert (o.rays, o.exact_range, o.cache, o.precision) == (128, 0, pm.PRC_CACHE_FULL, pm.PRC_PRECISION_FP32)
    assert abs(o.support_rho - 0.05) < 1e-7 and o.air_cap_mm == 50.0


def test_unknown_isotope_is_an_error():
    with pytest.raises(pm.PrcError) as e:
        pm.isotope_cutoff("99Zz")
    assert e.value.code == 2


def _create(geo, iso, opts, density):
    h = ctypes.c_void_p()
    rc = pm.lib().prc_create(ctypes.byref(geo), iso, ctypes.byref(opts), density.ctypes.data, ctypes.byref(h))
    return rc, h


@pytest.mark.parametrize("field,value", [("nx", 0), ("dy", 0.0), ("dz", float("nan"))])
def test_create_rejects_bad_geometry_before_cuda(field, value):
    geo = pm.Geometry(2, 2, 2, 1.0, 1.0, 1.0)
    setattr(geo, field, value)
    rc, h = _create(geo, b"68Ga", pm.default_options(), np.ones(8, np.float32))
    assert rc == 1 and not h.value
    assert b"Invalid" in pm.lib().prc_last_error()


@pytest.mark.parametrize("field,value", [("rays", 3), ("rays", 0), ("air_cap_mm", 0.0), ("support_rho", -1.0),
                                         ("precision", 7), ("cache", 5), ("cache", -1)])
def test_create_rejects_bad_options_before_cuda(field, value):
    opts = pm.default_options()
    setattr(opts, field, value)
    rc, h = _create(pm.Geometry(2, 2, 2, 1.0, 1.0, 1.0), b"68Ga", opts, np.ones(8, np.float32))
    assert rc == 1 and not h.value


def test_create_rejects_index_overflow_and_isotope_and_nonfinite():
    rc, _ = _create(pm.Geometry(65536, 65536, 1, 1.0, 1.0, 1.0), b"68Ga", pm.default_options(), np.ones(8, np.float32))
    assert rc == 8
    rc, _ = _create(pm.Geometry(2, 2, 2, 1.0, 1.0, 1.0), b"99Zz", pm.default_options(), np.ones(8, np.float32))
    assert rc == 2
    d = np.ones(8, np.float32)
    d[3] = np.nan
    rc, _ = _create(pm.Geometry(2, 2, 2, 1.0, 1.0, 1.0), b"68Ga", pm.default_options(), d)
    assert rc == 3
    assert b"Non-finite" in pm.lib().prc_last_error()


def test_null_arguments_are_rejected():
    lib = pm.lib()
    assert lib.prc_forward(None, None, None, None) == 1
    assert lib.prc_em_iterate(None, 1, 0.0, 0.0, 0, None) == 1
    assert lib.prc_synchronize(None) == 1
    lib.prc_destroy(None)
