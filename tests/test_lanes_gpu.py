"""GPU tests of the reference's two executable lanes, rebuilt on this library.

  bin/test_sgemm       the reference's correctness lane (test.cu:18-121) over
                       the range its test.sh runs (test.sh:3-5: every square
                       size 2..3072), which covers every k remainder modulo the
                       k block and every edge mask of the tiles
  bin/benchmark_sgemm  the reference's benchmark lane (benchmark.cu:22-208),
                       this library's kernels and the cuBLAS comparison lane
                       (benchmark.cu:150-164, --lib=cublas), whose output
                       files must load the way the reference's plot script
                       reads them (plot_benchmark_results.py:20-23)
"""
import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "sgemm.cu_b200", "bin")


def test_reference_test_sh_range_every_size(tmp_path):
    """test.sh's sweep: m = n = k from 2 to 3072 in steps of 1, alpha 1.5,
    beta 0.5, U[0,1) inputs, each result within the reference's 1e-4 relative
    criterion of the naive kernel; the harness exits non-zero on any failure."""
    r = subprocess.run([os.path.join(BIN, "test_sgemm"), "--mmin=2", "--mmax=3072", "--mstep=1",
                        f"--savedir={tmp_path}"], capture_output=True, text=True, timeout=1800)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    assert "PASSED: 3071 / 3071" in r.stdout
    assert "FAILED: 0" in r.stdout
    report = (tmp_path / "sgemm.cu.txt").read_text()
    assert report.count("n_false = 0, n_nan = 0, n_inf = 0") == 3071


def _bench(lane_args, fname, savedir):
    cmd = [os.path.join(BIN, "benchmark_sgemm"), "--wniter=3", "--wmsize=1024", "--mmin=1024",
           "--mstep=1024", "--npts=2", f"--fname={fname}", f"--savedir={savedir}"] + lane_args
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return r.stdout


def test_benchmark_lanes_write_the_reference_plot_format(tmp_path):
    """Both lanes (ours and cuBLAS) at 1024^3 and 2048^3 write `matsize gflops`
    lines that the reference's plot script loads unchanged: every *.txt in the
    directory through np.loadtxt(path).T, legend = file stem."""
    _bench([], "sgemm_b200", tmp_path)
    _bench(["--lib=cublas"], "cublas", tmp_path)
    lanes = {}
    for path in Path(tmp_path).glob("*.txt"):  # plot_benchmark_results.py:20-23
        matsize, max_gflops = np.loadtxt(path).T
        lanes[path.stem] = dict(zip(matsize.astype(int).tolist(), max_gflops.tolist()))
    assert set(lanes) == {"sgemm_b200", "cublas"}
    for name, pts in lanes.items():
        assert sorted(pts) == [1024, 2048], name
        assert all(g > 1000 for g in pts.values()), (name, pts)  # GFLOP/s, integers
    # context, not a bound: both lanes are FP32 GEMMs on the same part
    print("lanes (GFLOP/s):", lanes)
