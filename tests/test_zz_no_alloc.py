"""GPU test of sgemm_b200_split_noalloc, the allocation-free split GEMM.

That entry point is for callers that may not allocate device memory inside a
call (a framework that owns the GPU's allocator, latency-critical loops where
cudaMalloc/cudaFree would synchronise the device, fixed-footprint
deployments).  Its scratch is one static 64 MiB device array inside the
library, shared by every call.  This test calls it through the C ABI and
checks it against the allocating entry point, sgemm_b200_split, on two calls
in a row: the second call runs on whatever the first left in the shared array.
The file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

import oracle
import sgemm_b200 as sg

pytestmark = pytest.mark.gpu

_F = ctypes.POINTER(ctypes.c_float)


def _noalloc_fn():
    f = sg.lib().sgemm_b200_split_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int] * 4 + [_F, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                       ctypes.c_int, _F, ctypes.c_void_p, ctypes.c_int,
                                       ctypes.c_void_p]
    return f


def _call_noalloc(path, A, B, C, alpha, beta):
    m, k = A.shape
    n = B.shape[1]
    a, b = ctypes.c_float(alpha), ctypes.c_float(beta)
    return _noalloc_fn()(sg.PATHS[path], m, n, k, ctypes.byref(a), A.data_ptr(), A.stride(0),
                         B.data_ptr(), B.stride(0), ctypes.byref(b), C.data_ptr(), C.stride(0),
                         None)


@pytest.mark.parametrize("path", ["bf16x6", "tf32x3"])
def test_noalloc_matches_allocating_entry_point_twice(path):
    import torch

    # Two different problems back to back: the second reuses the shared array.
    for seed, (m, n, k) in ((31, (700, 900, 1024)), (32, (257, 130, 333))):
        A = oracle.fill(m, k, seed, 1, 0)
        B = oracle.fill(k, n, seed, 2, 0)
        C = oracle.fill(m, n, seed, 3, 0)
        dA, dB = torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda()
        c_new, c_old = torch.from_numpy(C).cuda(), torch.from_numpy(C).cuda()
        assert _call_noalloc(path, dA, dB, c_new, 1.5, 0.5) == sg.OK
        ws = torch.empty(sg.split_workspace_size(sg.PATHS[path], m, n, k), dtype=torch.uint8,
                         device="cuda")
        sg.sgemm_split(path, dA, dB, c_old, 1.5, 0.5, workspace=ws)
        torch.cuda.synchronize()
        assert sg.device_status() == sg.OK
        got, want = c_new.cpu().numpy(), c_old.cpu().numpy()
        # Same kernels and arithmetic: equal bits, and within the split path's
        # accuracy bound against FP64 (the tolerance the split tests use).
        assert np.array_equal(got, want)
        ref, mag = oracle.dgemm(A, B, C, 1.5, 0.5)
        e = oracle.error_stats(got, ref, mag)
        ep = oracle.error_stats(oracle.sgemm_basic(A, B, C, 1.5, 0.5, basic=False), ref, mag)
        assert e["max_componentwise"] <= 1.5 * ep["max_componentwise"] + 2.0 ** -23


def test_noalloc_refuses_problems_beyond_its_scratch():
    import torch

    n = 4096  # BF16x6 planes for 4096^3 need 192 MiB > 64 MiB
    A = torch.zeros((n, n), device="cuda")
    C = torch.full((n, n), 7.0, device="cuda")
    assert _call_noalloc("bf16x6", A, A, C, 1.0, 0.0) == sg.ERR_NO_MEMORY
    torch.cuda.synchronize()
    assert bool((C == 7.0).all())  # nothing ran
