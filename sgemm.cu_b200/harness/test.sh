#!/bin/bash
# Correctness sweep through the library's public API, with the reference's
# test.sh parameters: every square size 2..3072, the reference's criterion
# (relative error <= 1e-4 against the naive kernel), one result line per size
# in test_results/.  Usage: sgemm.cu_b200/harness/test.sh [extra test_sgemm flags]
#   e.g. --path=bf16x6 to sweep the split-precision path instead.
set -e
here="$(cd "$(dirname "$0")/.." && pwd)"
matsize_max=3072
matsize_min=2
matsize_step=1
save_dir="test_results"
mkdir -p "${save_dir}"
make -C "${here}" -j bin/test_sgemm > /dev/null
# flags given on the command line come first, so they override these defaults
"${here}/bin/test_sgemm" "$@" --savedir="${save_dir}" --mmax=${matsize_max} \
    --mmin=${matsize_min} --mstep=${matsize_step}
