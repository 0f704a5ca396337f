#!/usr/bin/env bash
# Compiles the reference executable (prc.cu of jlherraiz/PRC_MLEM) from its own source file,
# exactly as its build.sh does but for sm_100a, into oracle/_ref/prc.  It is test
# infrastructure only: the golden-fixture script and the parity tests run it as the
# reference, nothing in the product links or executes it.
#   usage: bash oracle/build_ref.sh [path/to/PRC_MLEM]   (or the checkout in PRC_REFERENCE_DIR)
set -euo pipefail
here="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
ref="${1:-${PRC_REFERENCE_DIR:-}}"
if [[ -z "$ref" || ! -f "$ref/prc.cu" ]]; then
    echo "reference source not given or not found (argument or PRC_REFERENCE_DIR); skipping" >&2
    exit 0
fi
mkdir -p "$here/_ref"
if [[ -x "$here/_ref/prc" && "$here/_ref/prc" -nt "$ref/prc.cu" ]]; then
    exit 0
fi
nvcc -O3 -gencode arch=compute_100a,code=sm_100a "$ref/prc.cu" -o "$here/_ref/prc"
