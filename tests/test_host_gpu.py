"""GPU tests of sgemm_b200_host (operands in host memory, staged through HBM
in row bands with the copies overlapping the kernels).

The reference's callers do cudaMemcpy(A, B, C) -> sgemm() -> cudaMemcpy(C)
(test.cu:70-80, benchmark.cu:69-73); the host entry point replaces that
sequence, so its result must equal the device entry point's on the same
inputs bit for bit (each band is the same GEMM on a block of rows, and each C
element keeps its k-ordered accumulation).
"""
import numpy as np
import pytest

import oracle
import sgemm_b200 as sg

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    return torch


def _host(x, ld=None, pinned=True):
    """Host tensor holding x, optionally inside a wider row stride ld whose
    extra columns are NaN canaries."""
    torch = _torch()
    rows, cols = x.shape
    ld = ld or cols
    big = torch.full((rows, ld), float("nan"), dtype=torch.float32, pin_memory=pinned)
    big[:, :cols] = torch.from_numpy(x)
    return big, big[:, :cols]


def _device_result(path, A, B, C, alpha, beta):
    torch = _torch()
    dA = torch.from_numpy(A).cuda()
    dB = torch.from_numpy(B).cuda()
    dC = torch.from_numpy(C).cuda()
    sg.gemm(path, dA, dB, dC, alpha, beta)
    torch.cuda.synchronize()
    return dC.cpu().numpy()


def _host_result(path, A, B, C, alpha, beta, lds=(None, None, None), pinned=True, stream=None):
    torch = _torch()
    _, hA = _host(A, lds[0], pinned)
    _, hB = _host(B, lds[1], pinned)
    bigC, hC = _host(C, lds[2], pinned)
    sg.sgemm_host(hA, hB, hC, alpha, beta, path=path, stream=stream)
    if stream is not None:
        stream.synchronize()
    else:
        torch.cuda.synchronize()
    return bigC, hC.numpy().copy()


@pytest.mark.parametrize("m,n,k", [(8192, 8192, 1024), (8192, 1024, 2048), (3001, 2999, 1003),
                                   (4100, 640, 2500), (200, 300, 50), (1, 4096, 4096),
                                   (5003, 5003, 700)])
def test_plain_host_equals_device(m, n, k):
    A, B, C = (oracle.fill(m, k, 21, 1, 0), oracle.fill(k, n, 21, 2, 0),
               oracle.fill(m, n, 21, 3, 0))
    want = _device_result("plain", A, B, C, 1.5, 0.5)
    bigC, got = _host_result("plain", A, B, C, 1.5, 0.5)
    assert np.array_equal(got, want)
    if m >= 3001:  # the blocked pipeline actually ran
        assert sg.host_plan(m, n, k)[0] < m


@pytest.mark.parametrize("plan", [(640, [1000, 1500, 500]), (3001, [3000]), (200, [128, 2872]),
                                  (1024, [512, 512, 512, 1464])])
def test_host_planned_equals_device(plan):
    # every valid block plan gives the device entry point's bits
    m, n, k = 3001, 3000, 700
    A, B, C = (oracle.fill(m, k, 12, 1, 0), oracle.fill(k, n, 12, 2, 0),
               oracle.fill(m, n, 12, 3, 0))
    want = _device_result("plain", A, B, C, 1.5, 0.5)
    torch = _torch()
    _, hA = _host(A)
    _, hB = _host(B)
    _, hC = _host(C)
    sg.sgemm_host(hA, hB, hC, 1.5, 0.5, plan=plan)
    torch.cuda.synchronize()
    assert np.array_equal(hC.numpy(), want)


def test_plain_host_strided_and_canaries():
    m, n, k = 2500, 1100, 900
    A, B, C = (oracle.fill(m, k, 5, 1, 0), oracle.fill(k, n, 5, 2, 0), oracle.fill(m, n, 5, 3, 0))
    want = _device_result("plain", A, B, C, -0.75, 2.0)
    bigC, got = _host_result("plain", A, B, C, -0.75, 2.0, lds=(k + 3, n + 5, n + 7))
    assert np.array_equal(got, want)
    # the padding columns of C are untouched
    assert np.isnan(bigC[:, n:].numpy()).all()


def test_beta_zero_never_reads_c():
    torch = _torch()
    m, n, k = 3000, 1024, 1024
    A, B = oracle.fill(m, k, 9, 1, 0), oracle.fill(k, n, 9, 2, 0)
    want = _device_result("plain", A, B, np.zeros((m, n), np.float32), 1.0, 0.0)
    _, hA = _host(A)
    _, hB = _host(B)
    hC = torch.full((m, n), float("nan"), dtype=torch.float32, pin_memory=True)
    sg.sgemm_host(hA, hB, hC, 1.0, 0.0)
    torch.cuda.synchronize()
    assert np.array_equal(hC.numpy(), want)


def test_k_zero_scales_c():
    # k == 0: C := beta*C (alpha*0 + beta*C in one rounding), on every block
    torch = _torch()
    m, n = 5000, 3000
    C = oracle.fill(m, n, 3, 3, 0)
    hA = torch.empty((m, 0), dtype=torch.float32, pin_memory=True)
    hB = torch.empty((0, n), dtype=torch.float32, pin_memory=True)
    _, hC = _host(C)
    l = sg.lib()
    assert l.sgemm_b200_host(0, m, n, 0, sg._f(1.5), 16, 1, 16, n, sg._f(0.5), hC.data_ptr(), n,
                             None) == sg.OK
    torch.cuda.synchronize()
    assert np.array_equal(hC.numpy(), C * np.float32(0.5))


def test_pageable_memory_same_result():
    m, n, k = 2048, 1536, 1024
    A, B, C = (oracle.fill(m, k, 4, 1, 0), oracle.fill(k, n, 4, 2, 0), oracle.fill(m, n, 4, 3, 0))
    want = _device_result("plain", A, B, C, 1.5, 0.5)
    _, got = _host_result("plain", A, B, C, 1.5, 0.5, pinned=False)
    assert np.array_equal(got, want)


def test_user_stream_ordering():
    torch = _torch()
    m, n, k = 4096, 2048, 1024
    A, B, C = (oracle.fill(m, k, 6, 1, 0), oracle.fill(k, n, 6, 2, 0), oracle.fill(m, n, 6, 3, 0))
    want = _device_result("plain", A, B, C, 1.5, 0.5)
    s = torch.cuda.Stream()
    _, got = _host_result("plain", A, B, C, 1.5, 0.5, stream=s)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("path", ["bf16x6", "tf32x3"])
def test_split_host_equals_device(path):
    m, n, k = 4096, 1024, 2048
    A, B, C = (oracle.fill(m, k, 8, 1, 0), oracle.fill(k, n, 8, 2, 0), oracle.fill(m, n, 8, 3, 0))
    want = _device_result(path, A, B, C, 1.5, 0.5)
    _, got = _host_result(path, A, B, C, 1.5, 0.5)
    assert np.array_equal(got, want)


def test_host_rejects_bad_arguments():
    torch = _torch()
    A = torch.zeros((64, 32), dtype=torch.float32)
    B = torch.zeros((32, 16), dtype=torch.float32)
    C = torch.zeros((64, 16), dtype=torch.float32)
    l = sg.lib()
    alpha = sg._f(1.0)
    beta = sg._f(0.0)
    # lda < k
    assert l.sgemm_b200_host(0, 64, 16, 32, alpha, A.data_ptr(), 16, B.data_ptr(), 16, beta,
                             C.data_ptr(), 16, None) == sg.ERR_INVALID_ARG
    # unknown path
    assert l.sgemm_b200_host(7, 64, 16, 32, alpha, A.data_ptr(), 32, B.data_ptr(), 16, beta,
                             C.data_ptr(), 16, None) == sg.ERR_INVALID_ARG
    # nothing to do
    assert l.sgemm_b200_host(0, 0, 16, 32, alpha, A.data_ptr(), 32, B.data_ptr(), 16, beta,
                             C.data_ptr(), 16, None) == sg.OK


@pytest.mark.parametrize("m,n,k,beta", [(4096, 4096, 4096, 0.5), (4096, 3000, 6000, 0.0),
                                        (3000, 4099, 4100, 0.5), (4097, 4101, 8192, 0.0),
                                        (3001, 5003, 5000, 0.5),
                                        (2500, 4224, 4100, 0.5)])
def test_kouter_plan_equals_device(m, n, k, beta):
    """Shapes where sgemm_host takes the k-outer plan (k slices streamed in,
    sums carried between launches in device memory, then row bands with the
    epilogue): the same bits as the device entry point, and NaN canaries
    beyond C's columns untouched."""
    k1, slices, rows = sg.host_plan_kouter(m, n, k, beta != 0)
    assert 0 < k1 < k and k1 % 128 == 0 and slices >= 1 and rows % 128 == 0
    A = oracle.fill(m, k, 61, 1, 0)
    B = oracle.fill(k, n, 61, 2, 0)
    C = oracle.fill(m, n, 61, 3, 0)
    want = _device_result("plain", A, B, C, 1.5, beta)
    bigC, got = _host_result("plain", A, B, C, 1.5, beta, lds=(k + 3, n + 5, n + 7))
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    assert np.isnan(bigC.numpy()[:, n:]).all()
