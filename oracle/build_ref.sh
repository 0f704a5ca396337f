#!/usr/bin/env bash
# Compiles the reference executable (prc.cu of jlherraiz/PRC_MLEM) from its own source file,
# exactly as its build.sh does but for sm_100a, into oracle/_ref/prc.  It is test
# infrastructure only: the golden-fixture script and the parity tests run it as the
# reference, nothing in the product links or executes it.
#   usage: bash oracle/build_ref.sh [path/to/reference]
set -euo pipefail
here="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
ref="${1:-/root/reference}"
if [[ ! -f "$ref/prc.cu" ]]; then
    echo "reference source not found at $ref/prc.cu; skipping" >&2
    exit 0
fi
mkdir -p "$here/_ref"
if [[ -x "$here/_ref/prc" && "$here/_ref/prc" -nt "$ref/prc.cu" ]]; then
    exit 0
fi
nvcc -O3 -gencode arch=compute_100a,code=sm_100a "$ref/prc.cu" -o "$here/_ref/prc"
