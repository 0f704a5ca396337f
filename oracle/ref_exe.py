"""Runs the reference executable (prc.cu of jlherraiz/PRC_MLEM compiled for sm_100a by
oracle/build_ref.sh into oracle/_ref/prc) on NumPy volumes.

Test infrastructure only: the parity tests and bench.py's parity and reference legs call it as
the checker; nothing in the product imports it.  The executable's command line is the one of
prc.cu:461-484 (positional ISOTOPE NX NY NZ DX DY DZ, --input/--density/--output raw float32
files, X fastest), and it prints `normalisation ...: X s` (prc.cu:644) and
`iterations X s (Y s each)` (prc.cu:719-720).
"""
from __future__ import annotations

import re
import subprocess
import tempfile
import time
from pathlib import Path

import numpy as np

EXE = Path(__file__).resolve().parent / "_ref" / "prc"


def available() -> bool:
    return EXE.is_file()


def run(mode: str, isotope: str, image: np.ndarray, rho: np.ndarray, spacing, *options: str,
        timeout: float = 900.0) -> dict:
    """One invocation of the reference executable.  Returns {"out": output volume (nz, ny, nx),
    "stdout": its standard output, "wall_s": wall time of the process, "setup_s" and
    "iterations_s": the times it prints itself (None where it printed none)}."""
    if not EXE.is_file():
        raise FileNotFoundError(f"{EXE} is missing: run oracle/build_ref.sh where the reference source is")
    shape = rho.shape
    nz, ny, nx = shape
    with tempfile.TemporaryDirectory(prefix="prc_ref_") as d:
        d = Path(d)
        np.ascontiguousarray(image, np.float32).tofile(d / "in.raw")
        np.ascontiguousarray(rho, np.float32).tofile(d / "rho.raw")
        cmd = [str(EXE), isotope, str(nx), str(ny), str(nz), *(repr(float(s)) for s in spacing),
               "--input", str(d / "in.raw"), "--density", str(d / "rho.raw"), "--output", str(d / "out.raw"),
               "--mode", mode, *options]
        t0 = time.perf_counter()
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
        wall = time.perf_counter() - t0
        if r.returncode != 0:
            raise RuntimeError(f"reference executable failed ({r.returncode}): {r.stdout[-500:]}\n{r.stderr[-500:]}")
        out = np.fromfile(d / "out.raw", np.float32).reshape(shape)
    it = re.search(r"iterations ([0-9.]+) s", r.stdout)
    setup = re.search(r"normalisation .*: ([0-9.]+) s", r.stdout)
    total = re.search(r"total ([0-9.]+) s", r.stdout)
    return {"out": out, "stdout": r.stdout, "wall_s": wall,
            "setup_s": float(setup.group(1)) if setup else None,
            "iterations_s": float(it.group(1)) if it else None,
            "total_s": float(total.group(1)) if total else None}
