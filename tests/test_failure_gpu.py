"""GPU test of the failure path of the kernels' bounded waits.

Every mbarrier wait in the GEMM kernels gives up after a wall-clock limit,
records SGEMM_B200_ERR_TIMEOUT in the library's device status word and lets
the kernel return.  sgemm_b200_selftest_wait_timeout runs that path on
purpose: one thread waits, with a short limit, on a barrier phase that nothing
completes.  Nothing faults or hangs; the test checks that the host sees the
timeout, that reading the status clears it, and that the device still
computes correct GEMMs afterwards.
"""
import time

import numpy as np
import pytest

import oracle
import sgemm_b200 as sg

pytestmark = pytest.mark.gpu


def test_bounded_wait_reports_timeout_and_device_stays_usable():
    import torch

    assert sg.device_status() == sg.OK  # start clean (also clears any earlier record)
    t0 = time.perf_counter()
    sg.selftest_wait_timeout(50_000)  # 50 ms
    status = sg.device_status()  # synchronises, then reads and clears
    waited = time.perf_counter() - t0
    assert status == sg.ERR_TIMEOUT
    assert waited >= 0.045, waited
    assert sg.device_status() == sg.OK

    # the context is intact: a GEMM right after is bit-exact with the oracle
    m, n, k = 300, 200, 100
    A, B, C = (oracle.fill(m, k, 2, 1, 0), oracle.fill(k, n, 2, 2, 0), oracle.fill(m, n, 2, 3, 0))
    dA, dB, dC = (torch.from_numpy(x).cuda() for x in (A, B, C))
    sg.sgemm(dA, dB, dC, 1.5, 0.5)
    torch.cuda.synchronize()
    want = oracle.sgemm_basic(A, B, C, 1.5, 0.5, basic=False)
    assert np.array_equal(dC.cpu().numpy(), want)
    assert sg.device_status() == sg.OK


def test_selftest_on_a_user_stream():
    import torch

    s = torch.cuda.Stream()
    sg.selftest_wait_timeout(20_000, stream=s)
    s.synchronize()
    assert sg.device_status() == sg.ERR_TIMEOUT
    assert sg.device_status() == sg.OK
