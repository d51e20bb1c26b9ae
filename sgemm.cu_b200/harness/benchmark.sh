#!/bin/bash
# GFLOP/s sweep with the reference's benchmark.sh parameters (93 sizes from
# 1024 in steps of 128, a 4096^3 warm-up of 500 calls), writing the
# reference's `matsize gflops` files to benchmark_results/ so its
# plot_benchmark_results.py reads them unchanged.  CUBLAS=1 adds the cuBLAS
# lane.  Unlike the reference's script this changes no GPU setting
# (persistence mode, clocks): the library and its tools only read them.
# Usage: [CUBLAS=1] sgemm.cu_b200/harness/benchmark.sh [extra benchmark_sgemm flags]
set -e
here="$(cd "$(dirname "$0")/.." && pwd)"
npts=93
matsize_step=128
matsize_min=1024
warmup_matsize=4096
warmup_iter=500
save_dir="benchmark_results"
mkdir -p "${save_dir}"
make -C "${here}" -j bin/benchmark_sgemm > /dev/null
# flags given on the command line come first, so they override these defaults
"${here}/bin/benchmark_sgemm" "$@" --fname=sgemm_b200 --savedir="${save_dir}" \
    --wniter=${warmup_iter} --wmsize=${warmup_matsize} --mmin=${matsize_min} \
    --mstep=${matsize_step} --npts=${npts}
if [ "${CUBLAS:-0}" -eq 1 ]; then
    "${here}/bin/benchmark_sgemm" "$@" --lib=cublas --fname=cublas --savedir="${save_dir}" \
        --wniter=${warmup_iter} --wmsize=${warmup_matsize} --mmin=${matsize_min} \
        --mstep=${matsize_step} --npts=${npts}
fi
