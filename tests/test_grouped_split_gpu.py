"""GPU tests of the grouped split-precision launch (no reference counterpart;
each problem keeps sgemm()'s contract, src/sgemm.cuh:19-30).

One grouped pre-pass and one persistent tcgen05 kernel run every problem of a
table.  Each problem's result must equal sgemm_b200_split's on its own, bit
for bit: the tiles run the same planes through the same MMA order and the same
K chunks, whatever else shares the launch and whichever CTA takes the tile.
"""
import numpy as np
import pytest

import oracle
import sgemm_b200 as sg

pytestmark = pytest.mark.gpu

PATHS = ["bf16x6", "tf32x3"]


def _torch():
    import torch
    return torch


def _make(shapes, seed0, pad=0):
    """Problems with seeded operands; C0 copies for the reference runs."""
    torch = _torch()
    specs, keep = [], []
    for i, (m, n, k) in enumerate(shapes):
        A = torch.empty((m, k + pad), device="cuda")[:, :k] if pad else torch.empty((m, k),
                                                                                    device="cuda")
        B = torch.empty((k, n + pad), device="cuda")[:, :n] if pad else torch.empty((k, n),
                                                                                    device="cuda")
        C = torch.empty((m, n), device="cuda")
        if k:
            sg.fill_random(A, seed0 + i, 1, sg.DIST_UNIFORM_PM1)
            sg.fill_random(B, seed0 + i, 2, sg.DIST_UNIFORM_PM1)
        sg.fill_random(C, seed0 + i, 3, sg.DIST_UNIFORM_PM1)
        alpha, beta = (1.5, 0.5) if i % 3 else (1.0, 0.0)
        specs.append((A, B, C, alpha, beta))
        keep.append(C.clone())
    torch.cuda.synchronize()
    return specs, keep


@pytest.mark.parametrize("path", PATHS)
def test_grouped_split_equals_single_calls(path):
    torch = _torch()
    # tile edges (m < 128, n < 256, ragged both), k remainders, a deep k, a
    # problem of many tiles, k == 0 (C := beta*C on the plain path)
    shapes = [(128, 256, 64), (100, 200, 33), (300, 520, 1001), (16, 4096, 1024),
              (129, 257, 255), (1024, 768, 2048), (64, 64, 8), (257, 300, 0), (1, 1, 1),
              (777, 513, 777)]
    specs, c0 = _make(shapes, 900)
    probs = sg.make_problems(specs)
    sg.grouped_split(path, probs)
    torch.cuda.synchronize()
    assert sg.device_status() == sg.OK
    for (A, B, C, alpha, beta), C0 in zip(specs, c0):
        want = C0.clone()
        if A.shape[1]:
            sg.sgemm_split(path, A, B, want, alpha, beta)
        else:
            sg.sgemm(A, B, want, alpha, beta)
        torch.cuda.synchronize()
        assert torch.equal(C, want), (path, A.shape, B.shape)


@pytest.mark.parametrize("path", PATHS)
def test_grouped_split_strides_and_accuracy(path):
    """Operands with row strides that are not multiples of 4 (the pre-pass
    reads any stride), and FP64 accuracy within the split tests' bound."""
    torch = _torch()
    shapes = [(200, 136, 100), (333, 444, 555)]
    specs, c0 = _make(shapes, 950, pad=3)
    sg.grouped_split(path, sg.make_problems(specs))
    torch.cuda.synchronize()
    for (A, B, C, alpha, beta), C0 in zip(specs, c0):
        hA, hB, hC0 = A.cpu().numpy(), B.cpu().numpy(), C0.cpu().numpy()
        ref, mag = oracle.dgemm(hA, hB, hC0, alpha, beta)
        e = oracle.error_stats(C.cpu().numpy(), ref, mag)
        ep = oracle.error_stats(oracle.sgemm_basic(hA, hB, hC0, alpha, beta, basic=False), ref,
                                mag)
        assert e["non_finite"] == 0
        assert e["max_componentwise"] <= 1.5 * ep["max_componentwise"] + 2.0 ** -23


@pytest.mark.parametrize("path", PATHS)
def test_grouped_split_many_uneven_problems(path):
    """96 problems of the grouped workload's distribution (M, N, K log-uniform
    on [64, 1024], multiples of 8) in one launch: more tiles than SMs, so CTAs
    run several tiles each; every result equals the sequential calls'."""
    torch = _torch()
    rng = np.random.default_rng(3)
    vals = np.exp(rng.uniform(np.log(64), np.log(1024), size=(96, 3)))
    shapes = [tuple(int(max(8, round(v / 8) * 8)) for v in row) for row in vals]
    specs, c0 = _make(shapes, 1000)
    seq = [(A, B, C0.clone(), alpha, beta) for (A, B, C, alpha, beta), C0 in zip(specs, c0)]
    sg.grouped_split(path, sg.make_problems(specs))
    sg.grouped_split_sequential(path, sg.make_problems(seq))
    torch.cuda.synchronize()
    assert sg.device_status() == sg.OK
    for (A, B, C, alpha, beta), (_, _, Cs, _, _) in zip(specs, seq):
        assert torch.equal(C, Cs), (A.shape, B.shape)
