"""CPU tests of the oracle (no GPU): generator, kernel_basic restatement, FP64
GEMM and error statistics, and the pins against the reference's own outputs
(tests/golden/, produced by the reference's kernels built from its sources).

Reference semantics being restated: src/kernels/basic.cuh:14-25 (kernel_basic)
and common/helper_matrix.h:51-86 (compare_mats).
"""
import json
import os
from fractions import Fraction

import numpy as np
import pytest

import oracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

M64 = (1 << 64) - 1


# ------------------------------------------------- pure-Python restatements --

def _mix(z):
    z = (z + 0x9E3779B97F4A7C15) & M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


def _key(seed, tag):
    return _mix(seed ^ _mix((0xA0761D6478BD642F + tag) & M64))


def _value(key, idx, dist):
    b = _mix((key + idx) & M64)
    if dist == 0:
        return np.float32(((b >> 40) - (1 << 23)) / 8388608.0)
    if dist == 1:
        return np.float32((b >> 40) / 16777216.0)
    sign = b & 1
    e = ((b >> 1) % 21) - 10
    mant = (b >> 41) & 0x7FFFFF
    bits = (sign << 31) | ((127 + e) << 23) | mant
    return np.array([bits], dtype=np.uint32).view(np.float32)[0]


def _fma32(a, b, c):
    """fmaf with round-to-nearest-even, computed exactly."""
    exact = Fraction(float(a)) * Fraction(float(b)) + Fraction(float(c))
    f = np.float32(float(exact))
    best = f
    for cand in (np.nextafter(f, np.float32(-np.inf)), np.nextafter(f, np.float32(np.inf))):
        d_best = abs(Fraction(float(best)) - exact)
        d_c = abs(Fraction(float(cand)) - exact)
        if d_c < d_best or (d_c == d_best and
                            (cand.view(np.uint32) & 1) == 0 and (best.view(np.uint32) & 1) == 1):
            best = cand
    return np.float32(best)


def _basic_python(A, B, C, alpha, beta, basic=True):
    """Exact restatement: FMA chain over p, then kernel_basic's epilogue
    fma(acc, alpha, c*beta) or the tiled kernels' fma(c, beta, acc*alpha)."""
    m, k = A.shape
    n = B.shape[1]
    out = C.copy()
    for y in range(m):
        for x in range(n):
            acc = np.float32(0)
            for p in range(k):
                acc = _fma32(A[y, p], B[p, x], acc)
            if basic:
                cb = np.float32(C[y, x] * np.float32(beta))
                out[y, x] = _fma32(acc, np.float32(alpha), cb)
            else:
                v = np.float32(acc * np.float32(alpha))
                out[y, x] = _fma32(C[y, x], np.float32(beta), v) if beta != 0 else v
    return out


# ----------------------------------------------------------------- generator --

@pytest.mark.parametrize("dist", [0, 1, 2])
def test_generator_matches_python_restatement(dist):
    X = oracle.fill(7, 9, seed=123, tag=5, dist=dist)
    key = _key(123, 5)
    for r in range(7):
        for c in range(9):
            assert X[r, c].view(np.uint32) == _value(key, r * 9 + c, dist).view(np.uint32)


def test_generator_ranges_and_rows():
    u = oracle.fill(64, 257, 0, 1, 0)
    assert u.min() >= -1.0 and u.max() < 1.0
    v = oracle.fill(64, 257, 0, 1, 1)
    assert v.min() >= 0.0 and v.max() < 1.0
    w = oracle.fill(64, 257, 0, 1, 2)
    e = np.floor(np.log2(np.abs(w.astype(np.float64))))
    assert e.min() >= -10 and e.max() <= 10
    assert (w > 0).any() and (w < 0).any()
    rows = [3, 0, 63, 17]
    np.testing.assert_array_equal(oracle.fill_rows(rows, 257, 0, 1, 2), w[rows])
    # different seeds / tags give different matrices
    assert not np.array_equal(oracle.fill(8, 8, 0, 1, 0), oracle.fill(8, 8, 1, 1, 0))
    assert not np.array_equal(oracle.fill(8, 8, 0, 1, 0), oracle.fill(8, 8, 0, 2, 0))


# ---------------------------------------------------- kernel_basic restatement --

@pytest.mark.parametrize("shape", [(1, 1, 1), (3, 5, 7), (6, 4, 9)])
@pytest.mark.parametrize("ab", [(1.5, 0.5), (1.0, 0.0), (-2.0, 3.0)])
def test_basic_matches_exact_python(shape, ab):
    m, n, k = shape
    alpha, beta = ab
    A = oracle.fill(m, k, 9, 1, 0)
    B = oracle.fill(k, n, 9, 2, 0)
    C = oracle.fill(m, n, 9, 3, 0)
    for basic in (True, False):
        got = oracle.sgemm_basic(A, B, C, alpha, beta, basic=basic)
        want = _basic_python(A, B, C, alpha, beta, basic=basic)
        np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))


def test_basic_rows_matches_full():
    A = oracle.fill(40, 33, 2, 1, 0)
    B = oracle.fill(33, 300, 2, 2, 0)
    C = oracle.fill(40, 300, 2, 3, 0)
    full = oracle.sgemm_basic(A, B, C, 1.5, 0.5)
    rows = [0, 7, 39, 12]
    part = oracle.sgemm_basic_rows(rows, A, B, C[rows], 1.5, 0.5)
    np.testing.assert_array_equal(part, full[rows])


def test_beta_zero_semantics():
    A = oracle.fill(5, 6, 1, 1, 0)
    B = oracle.fill(6, 7, 1, 2, 0)
    C = np.full((5, 7), np.nan, dtype=np.float32)
    # tiled-kernel semantics: C not read when beta == 0
    tiled = oracle.sgemm_basic(A, B, C, 1.0, 0.0, basic=False)
    assert np.isfinite(tiled).all()
    # kernel_basic semantics: C always read, NaN * 0 = NaN propagates
    basic = oracle.sgemm_basic(A, B, C, 1.0, 0.0, basic=True)
    assert np.isnan(basic).all()


def test_thread_count_does_not_change_bits():
    A = oracle.fill(70, 129, 4, 1, 2)
    B = oracle.fill(129, 300, 4, 2, 2)
    C = oracle.fill(70, 300, 4, 3, 2)
    one = oracle.sgemm_basic(A, B, C, 1.5, 0.5, threads=1)
    many = oracle.sgemm_basic(A, B, C, 1.5, 0.5, threads=4)
    np.testing.assert_array_equal(one.view(np.uint32), many.view(np.uint32))


# --------------------------------------------------------------- FP64 / error --

def test_dgemm_matches_numpy():
    A = oracle.fill(50, 70, 3, 1, 0)
    B = oracle.fill(70, 90, 3, 2, 0)
    C = oracle.fill(50, 90, 3, 3, 0)
    ref, mag = oracle.dgemm(A, B, C, 1.5, 0.5)
    want = 1.5 * (A.astype(np.float64) @ B.astype(np.float64)) + 0.5 * C.astype(np.float64)
    np.testing.assert_allclose(ref, want, rtol=1e-13, atol=1e-13)
    wmag = 1.5 * (np.abs(A.astype(np.float64)) @ np.abs(B.astype(np.float64))) + 0.5 * np.abs(C)
    np.testing.assert_allclose(mag, wmag, rtol=1e-13)
    rows = [1, 49, 20]
    r2, m2 = oracle.dgemm(A, B, C[rows], 1.5, 0.5, row_ids=rows)
    np.testing.assert_allclose(r2, ref[rows], rtol=1e-15, atol=0)


def test_error_stats_catch_planted_error():
    A = oracle.fill(30, 40, 5, 1, 0)
    B = oracle.fill(40, 50, 5, 2, 0)
    C0 = oracle.fill(30, 50, 5, 3, 0)
    ref, mag = oracle.dgemm(A, B, C0, 1.5, 0.5)
    good = oracle.sgemm_basic(A, B, C0, 1.5, 0.5)
    s = oracle.error_stats(good, ref, mag)
    assert s["max_componentwise"] < 40 * 2 ** -24 * 2  # FP32 chain of 40 FMAs
    bad = good.copy()
    bad[7, 11] *= 1.01  # plant a mistake in the oracle's own output
    sb = oracle.error_stats(bad, ref, mag)
    assert sb["max_componentwise"] > 100 * s["max_componentwise"]
    bad[0, 0] = np.nan
    assert oracle.error_stats(bad, ref, mag)["non_finite"] == 1


# ------------------------------------------------- pins against the reference --

def _golden_cases():
    idx = os.path.join(GOLDEN, "index.json")
    if not os.path.exists(idx):
        return []
    with open(idx) as f:
        return json.load(f)["cases"]


def test_golden_fixtures_present():
    cases = _golden_cases()
    assert cases, "tests/golden/index.json missing: run tests/golden/make_golden.py on a B200"
    kernels = {c["ref_kernel"] for c in cases}
    assert {"sgemm_128x128x8", "sgemm_128x256x8", "kernel_basic"} <= kernels


def _golden(case):
    m, n, k = case["m"], case["n"], case["k"]
    A = oracle.fill(m, k, case["seed"], 1, case["dist"])
    B = oracle.fill(k, n, case["seed"], 2, case["dist"])
    C = oracle.fill(m, n, case["seed"], 3, case["dist"])
    got = np.fromfile(os.path.join(GOLDEN, case["file"]), dtype=np.float32).reshape(m, n)
    return A, B, C, got


def _reference_correct(case):
    """sgemm_128x128x8 built for sm_100a is only correct with a single k block
    (k <= 8); see test_reference_128x128x8_defect_on_sm100."""
    return case["ref_kernel"] != "sgemm_128x128x8" or case["k"] <= 8


@pytest.mark.parametrize("case", [c for c in _golden_cases() if _reference_correct(c)],
                         ids=lambda c: c["name"])
def test_oracle_reproduces_reference_outputs(case):
    """Fixtures hold the reference's own kernels' outputs on the oracle's
    seeded inputs.  The oracle must reproduce them bit for bit:
    kernel_basic with the basic epilogue, the tiled kernels with theirs."""
    A, B, C, got = _golden(case)
    want = oracle.sgemm_basic(A, B, C, case["alpha"], case["beta"],
                              basic=case["ref_kernel"] == "kernel_basic")
    assert np.array_equal(got, want), (
        f"{int((got != want).sum())} of {got.size} elements differ")


@pytest.mark.parametrize("case", [c for c in _golden_cases() if not _reference_correct(c)],
                         ids=lambda c: c["name"])
def test_reference_128x128x8_defect_on_sm100(case):
    """Recorded finding: the reference's sgemm_128x128x8, compiled from its
    sources for sm_100a, returns wrong values whenever its main loop runs
    (k > 8).  Its output is far from FP64 while the oracle's is within FP32
    rounding, so these fixtures cannot pin the oracle; they pin the defect."""
    A, B, C, got = _golden(case)
    ref, mag = oracle.dgemm(A, B, C, case["alpha"], case["beta"])
    bad = oracle.error_stats(got, ref, mag)["max_componentwise"]
    want = oracle.sgemm_basic(A, B, C, case["alpha"], case["beta"], basic=False)
    good = oracle.error_stats(want, ref, mag)["max_componentwise"]
    assert good < 1e-6
    assert bad > 1e-3
