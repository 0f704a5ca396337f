"""Parity with the reference executable at the clinical sizes (prc.cu:643-720 run on the same
inputs): the 128x128x159 torso at 0.776x0.776x0.795 mm for 68Ga (the benchmark configuration),
82Rb and 124I (the long-range configuration), and the 200^3 82Rb torso at 0.776 mm isotropic.

For every case the reference executable (oracle/_ref/prc, built from prc.cu for sm_100a) makes
the measured data itself -- its forward blur of the truth with 128 rays, Poisson-sampled at 5e7
counts -- and then projects and corrects that data (--mode forward / adjoint / correct with 6
MAP-EM iterations, beta 0.03, gamma 20, acceleration on, support density 0.05).  The engine runs
the same inputs through the C ABI.  Tolerances: every fp32 form within 1e-5 relative L2 of the
reference (its forward scatters with atomics, so the summation order differs), the 24-bit stored
field (fp32 weights rounded to 16 mantissa bits) too; the bf16 stored field within 2e-3 relative
L2 per projection and 1 % NRMSE for the corrected image.
"""
import numpy as np
import pytest

import prc_mlem_b200 as pm
from conftest import nrmse, rel_l2
from oracle import ref_exe
from prc_mlem_b200 import phantoms

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_exe.available(), reason="oracle/_ref/prc not built (needs prc.cu)")]

RAYS, ITERS, BETA, GAMMA, COUNTS = 128, 6, 0.03, 20.0, 5e7
EM_OPTS = ("--rays", str(RAYS), "--iterations", str(ITERS), "--beta", str(BETA), "--gamma", str(GAMMA),
           "--support-rho", "0.05")
FORMS = {"fp32_field": dict(cache=pm.PRC_CACHE_FULL),
         "traced": dict(cache=pm.PRC_CACHE_NEAR),
         "bf16_field": dict(cache=pm.PRC_CACHE_FULL, precision=pm.PRC_PRECISION_BF16),
         "fp24_field": dict(cache=pm.PRC_CACHE_FULL, precision=pm.PRC_PRECISION_FP24)}
_cases = {}


def case(iso: str, shape=(159, 128, 128)):
    """Inputs and the reference executable's outputs for one isotope and grid (computed once)."""
    key = (iso, shape)
    if key not in _cases:
        rho, truth, sp = phantoms.torso_phantom(seed=2, shape=shape)
        if shape != (159, 128, 128):
            sp = (0.776, 0.776, 0.776)
        blur = ref_exe.run("forward", iso, truth, rho, sp, "--rays", str(RAYS))["out"]
        g = phantoms.poisson_counts(blur, COUNTS, seed=17)
        support = np.maximum(rho, np.float32(1e-3)) >= np.float32(0.05)
        g_in = np.where(support, g, 0.0).astype(np.float32)  # the input as the reference reads it
        ref = {m: ref_exe.run(m, iso, g, rho, sp, *EM_OPTS)["out"] for m in ("forward", "adjoint", "correct")}
        _cases[key] = (rho, sp, g, g_in, ref)
    return _cases[key]


def check(P, rho, g, g_in, ref, form):
    fwd, adj = P.forward_host(g_in), P.adjoint_host(g_in)
    em = P.correct_host(g, ITERS, BETA, GAMMA, True)
    if form == "bf16_field":
        assert rel_l2(fwd, ref["forward"]) < 2e-3
        assert rel_l2(adj, ref["adjoint"]) < 2e-3
        assert nrmse(em, ref["correct"]) < 1e-2
    else:
        assert rel_l2(fwd, ref["forward"]) < 1e-5
        assert rel_l2(adj, ref["adjoint"]) < 1e-5
        assert rel_l2(em, ref["correct"]) < 1e-5


@pytest.mark.parametrize("form", sorted(FORMS))
@pytest.mark.parametrize("iso", ["68Ga", "82Rb", "124I"])
def test_torso_128x128x159_matches_reference_binary(iso, form):
    rho, sp, g, g_in, ref = case(iso)
    with pm.Projector(iso, rho, sp, rays=RAYS, **FORMS[form]) as P:
        if form != "traced":
            assert P.cache_mode[0] == pm.PRC_CACHE_FULL  # the stored field, not a fallback
        check(P, rho, g, g_in, ref, form)


def test_torso_200_cubed_82rb_matches_reference_binary():
    """The largest configuration: whichever fp32 form the memory planner picks."""
    rho, sp, g, g_in, ref = case("82Rb", (200, 200, 200))
    with pm.Projector("82Rb", rho, sp, rays=RAYS) as P:
        assert P.cache_mode[0] in (pm.PRC_CACHE_FULL, pm.PRC_CACHE_SOURCE_MAJOR)
        check(P, rho, g, g_in, ref, "fp32_field")
