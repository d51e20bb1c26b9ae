"""GPU tests of serving requests that carry the caller's own matrices.

The reference's callers own their matrices and copy them to the device
themselves before calling sgemm() (test.cu:69-81, benchmark.cu:68-73).  The
server accepts the same two forms: device matrices used in place
(sgemm_b200_server_submit_device) and host matrices it copies in and back
(sgemm_b200_server_submit_host).  Each result must be the library's own result
for that GEMM: bit for bit the oracle's restatement of the reference's
arithmetic on the plain path, bit for bit sgemm_b200_split on a split path --
whatever batch the request lands in.
"""
import numpy as np
import pytest

import oracle
import sgemm_b200 as sg

pytestmark = pytest.mark.gpu

SHAPES = [(300, 520, 1001), (16, 4096, 4096), (777, 777, 777), (64, 1000, 33), (129, 257, 513)]


def _torch():
    import torch
    return torch


def _padded(x, pad):
    """A CUDA tensor view of x with row stride cols + pad (pad 0: contiguous)."""
    torch = _torch()
    rows, cols = x.shape
    big = torch.full((rows, cols + pad), float("nan"), device="cuda")
    big[:, :cols] = torch.from_numpy(x).cuda()
    return big[:, :cols]


def _want(path, A, B, C, alpha, beta):
    if path == "plain":
        return oracle.sgemm_basic(A, B, C, alpha, beta, basic=False)
    torch = _torch()
    dC = torch.from_numpy(C).cuda()
    sg.sgemm_split(path, torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda(), dC, alpha, beta)
    torch.cuda.synchronize()
    return dC.cpu().numpy()


@pytest.mark.parametrize("path", ["plain", "bf16x6"])
def test_caller_device_operands_in_a_mix(path):
    torch = _torch()
    srv = sg.Server(1 << 33, slots=2, max_batch=16, path=path, keep_results=True)
    cases = []
    for i, (m, n, k) in enumerate(SHAPES):
        A = oracle.fill(m, k, 700 + i, 1, 0)
        B = oracle.fill(k, n, 700 + i, 2, 0)
        C = oracle.fill(m, n, 700 + i, 3, 0)
        pad = (0, 3, 8, 1, 0)[i]  # general strides, some not multiples of 4
        dA, dB, dC = _padded(A, pad), _padded(B, pad), _padded(C, pad)
        alpha, beta = (1.5, 0.5) if i % 2 == 0 else (1.0, 0.0)
        if beta == 0.0:
            dC.fill_(float("nan"))  # beta == 0: C must never be read
        cases.append((A, B, C, alpha, beta, dA, dB, dC))
    torch.cuda.synchronize()
    ids = []
    for i, (A, B, C, alpha, beta, dA, dB, dC) in enumerate(cases):
        # generated requests in between, so the caller's requests share batches
        srv.submit(512, 512, 512, seed=i)
        ids.append(srv.submit_device(dA, dB, dC, alpha, beta))
    srv.drain()
    st = srv.stats()
    for rid, (A, B, C, alpha, beta, dA, dB, dC) in zip(ids, cases):
        res = srv.result(rid)
        assert res["C"] == dC.data_ptr() and res["ldc"] == dC.stride(0)
        got = dC.cpu().numpy()
        assert np.array_equal(got, _want(path, A, B, C, alpha, beta)), (path, A.shape, B.shape)
        assert np.array_equal(srv.read_result(rid, *C.shape), got)
    srv.close()
    print(path, st)
    assert st["completed"] == 2 * len(SHAPES) and st["failed"] == 0
    assert sg.device_status() == sg.OK


@pytest.mark.parametrize("path", ["plain", "bf16x6"])
def test_caller_host_operands_copied_in_and_back(path):
    torch = _torch()
    srv = sg.Server(1 << 33, slots=2, max_batch=16, path=path, keep_results=False)
    cases = []
    for i, (m, n, k) in enumerate(SHAPES):
        A = oracle.fill(m, k, 800 + i, 1, 0)
        B = oracle.fill(k, n, 800 + i, 2, 0)
        C = oracle.fill(m, n, 800 + i, 3, 0)
        alpha, beta = (1.5, 0.5) if i % 2 == 0 else (1.0, 0.0)
        hA = torch.from_numpy(A).pin_memory()
        hB = torch.from_numpy(B).pin_memory()
        hC = torch.from_numpy(C if beta else np.full_like(C, np.nan)).pin_memory()
        cases.append((A, B, C, alpha, beta, hA, hB, hC))
    ids = [srv.submit_host(hA, hB, hC, alpha, beta)
           for (A, B, C, alpha, beta, hA, hB, hC) in cases]
    lat = [srv.wait(rid) for rid in ids]  # the copy back is part of completion
    for rid, (A, B, C, alpha, beta, hA, hB, hC) in zip(ids, cases):
        got = hC.numpy()
        assert np.array_equal(got, _want(path, A, B, C, alpha, beta)), (path, A.shape)
        assert np.array_equal(srv.read_result(rid, *C.shape), got)
    srv.close()
    assert all(x > 0 for x in lat)


def test_isolated_time_and_wait():
    srv = sg.Server(1 << 32, slots=2, max_batch=8, path="plain")
    t_small = srv.isolated_ms(64, 4096, 4096)
    t_big = srv.isolated_ms(2048, 2048, 2048)
    assert 0 < t_small < t_big
    rid = srv.submit(256, 256, 256, seed=1)
    assert srv.wait(rid) > 0
    srv.close()
