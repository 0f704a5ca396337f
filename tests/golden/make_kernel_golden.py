"""Generates tests/golden/water_kernel.npz and range_model.npz from the reference's own
FP64 range-model quadrature, tests/reference.py of jlherraiz/PRC_MLEM.

Run where the reference checkout is readable, giving its directory as the argument or in
PRC_REFERENCE_DIR:
    python tests/golden/make_kernel_golden.py path/to/PRC_MLEM
It imports the reference module (read-only), evaluates
  * reference.kernel(68Ga, voxel, half) for 4 mm and 2 mm voxels -- the homogeneous water
    kernel the reference's GPU test compares against (tests/test_solver.py:216-243);
  * reference.survival for all 8 isotopes on a radius grid and range_table_error
    (tests/test_rdp.py:18-24);
and writes the arrays.  The fixtures travel with the repository; the reference does not.
"""
import os
import sys
from pathlib import Path

import numpy as np


def main(ref_root: str) -> None:
    ref = Path(ref_root)
    sys.path.insert(0, str(ref / "tests"))
    import reference  # the reference's own module

    _, isotopes, bins = reference.read_model(ref / "prc.cu")
    out = Path(__file__).resolve().parent
    kernels = {}
    for size in (4.0, 2.0):
        half = int(np.ceil(10 / size)) + 1
        kernels[f"kernel_{size:g}mm"] = reference.kernel(isotopes["68Ga"], (size,) * 3, half)
        kernels[f"half_{size:g}mm"] = np.int64(half)
    np.savez_compressed(out / "water_kernel.npz", **kernels)

    r = np.linspace(0.0, 20.0, 401)
    model = {"radius": r, "bins": np.int64(bins)}
    for name, br in isotopes.items():
        fixed = np.array(br, np.float64)
        fixed[np.argmin(fixed[:, 0]), 0] += 1 - fixed[:, 0].sum()
        model[f"branches_{name}"] = np.array(br, np.float32)
        model[f"survival_{name}"] = reference.survival(fixed, r)
        model[f"table_error_{name}"] = np.float64(reference.range_table_error(br, bins))
    np.savez_compressed(out / "range_model.npz", **model)
    print("wrote", out / "water_kernel.npz", out / "range_model.npz")


if __name__ == "__main__":
    ref_dir = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PRC_REFERENCE_DIR")
    if not ref_dir:
        raise SystemExit("give the reference checkout as the argument or in PRC_REFERENCE_DIR")
    main(ref_dir)
