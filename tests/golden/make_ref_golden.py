"""Generates tests/golden/ref_outputs.npz by running the REFERENCE executable (prc.cu of
jlherraiz/PRC_MLEM, compiled for sm_100a by oracle/build_ref.sh into oracle/_ref/prc) on a
B200.  These outputs pin both the CPU oracle and the CUDA engine to the reference itself.

    python tests/golden/make_ref_golden.py [out.npz]

Cases (all inputs are regenerated from seeds by prc_mlem_b200.phantoms):
  fixture_*  -- the seed-72 16x14x12 fixture of tests/test_solver.py:143-157, --rays 32:
                forward/adjoint for every isotope, --exact-range, A^T 1, and MAP-EM runs;
  small_*    -- the 32x32x24 2 mm 18F phantom, --rays 32: forward of the truth, its Poisson
                sample at 1e6 counts, adjoint, and 4 plain RL iterations (--beta 0 --no-accel).
"""
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from prc_mlem_b200 import phantoms  # noqa: E402

EXE = ROOT / "oracle" / "_ref" / "prc"


def run(tmp: Path, tag: str, image, rho, shape, spacing, isotope, mode, *options):
    src, den, out = tmp / f"{tag}_in.raw", tmp / f"{tag}_rho.raw", tmp / f"{tag}_out.raw"
    np.asarray(image, np.float32).tofile(src)
    np.asarray(rho, np.float32).tofile(den)
    nz, ny, nx = shape
    cmd = [str(EXE), isotope, str(nx), str(ny), str(nz), *(str(s) for s in spacing), "--input", str(src),
           "--density", str(den), "--output", str(out), "--mode", mode, *options]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    if r.returncode != 0:
        raise RuntimeError(f"{tag}: {r.stdout}\n{r.stderr}")
    return np.fromfile(out, np.float32).reshape(shape)


def main(path: str) -> None:
    if not EXE.is_file():
        raise SystemExit(f"{EXE} missing: run oracle/build_ref.sh where the reference source is")
    res = {}
    with tempfile.TemporaryDirectory() as d:
        tmp = Path(d)
        rho, x, y, shape, sp = phantoms.solver_fixture()
        res["fixture_rho"], res["fixture_x"], res["fixture_y"] = rho, x, y
        for iso in ("11C", "13N", "15O", "18F", "64Cu", "68Ga", "82Rb", "124I"):
            res[f"fixture_fwd_{iso}"] = run(tmp, "f", x, rho, shape, sp, iso, "forward", "--rays", "32")
            res[f"fixture_adj_{iso}"] = run(tmp, "a", y, rho, shape, sp, iso, "adjoint", "--rays", "32")
        res["fixture_fwd_exact_68Ga"] = run(tmp, "fe", x, rho, shape, sp, "68Ga", "forward", "--rays", "32",
                                            "--exact-range")
        res["fixture_adj_one_68Ga"] = run(tmp, "a1", np.ones(shape, np.float32), rho, shape, sp, "68Ga", "adjoint",
                                          "--rays", "32")
        res["fixture_fwd_128_68Ga"] = run(tmp, "f128", x, rho, shape, sp, "68Ga", "forward", "--rays", "128")
        em_cases = {
            "em_b0.1_it3": ("--iterations", "3", "--beta", "0.1"),
            "em_b0_it4_plain": ("--iterations", "4", "--beta", "0", "--no-accel"),
            "em_b0.2_it2_plain": ("--iterations", "2", "--beta", "0.2", "--no-accel"),
            "em_b0.03_it6": ("--iterations", "6", "--beta", "0.03", "--gamma", "20"),
            "em_b0_it25": ("--iterations", "25", "--beta", "0"),
        }
        for name, opts in em_cases.items():
            res[f"fixture_{name}"] = run(tmp, name, x, rho, shape, sp, "68Ga", "correct", "--rays", "32", *opts)

        srho, truth, ssp = phantoms.small_phantom(seed=1)
        sshape = srho.shape
        res["small_rho"], res["small_truth"] = srho, truth
        blurred = run(tmp, "sf", truth, srho, sshape, ssp, "18F", "forward", "--rays", "32")
        res["small_fwd"] = blurred
        g = phantoms.poisson_counts(blurred, 1e6, seed=11)
        res["small_g"] = g
        res["small_adj"] = run(tmp, "sa", truth, srho, sshape, ssp, "18F", "adjoint", "--rays", "32")
        res["small_em_b0_it4_plain"] = run(tmp, "se", g, srho, sshape, ssp, "18F", "correct", "--rays", "32",
                                           "--beta", "0", "--no-accel", "--iterations", "4")
    np.savez_compressed(path, **res)
    print("wrote", path, len(res), "arrays")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else str(Path(__file__).resolve().parent / "ref_outputs.npz"))
