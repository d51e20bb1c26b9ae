"""GPU test of sgemm_b200_split_noalloc, the allocation-free split GEMM.

That entry point is for callers that may not allocate device memory inside a
call (a framework that owns the GPU's allocator, latency-critical loops where
cudaMalloc/cudaFree would synchronise the device, fixed-footprint
deployments).  Its scratch is one static device array inside the library
(64 MiB of operand planes plus 1 KiB of alignment), shared by every call.
These tests call it through the C ABI and check it against the allocating
entry point, sgemm_b200_split, on two calls in a row (the second call runs on
whatever the first left in the shared array), check that a call allocates
nothing, and check the size limit on both sides.
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


def _memory_state():
    import torch

    torch.cuda.synchronize()
    return sg.pool_usage(), torch.cuda.mem_get_info()[0], torch.cuda.memory_allocated()


@pytest.mark.parametrize("path", ["bf16x6", "tf32x3"])
def test_noalloc_allocates_nothing(path):
    """The property that defines the entry point: a call leaves the library's
    own pool, torch's allocator and the device's free memory as they were.
    Each route (beta != 0, beta == 0, and k == 0, which runs a plain-path
    kernel) is called once before measuring, so that one-time costs that are
    not allocations by the call do not show: CUDA loads a kernel's code onto
    the device the first time it is launched (2 MiB of device memory in a
    fresh process), and the first call looks up the scratch array's address."""
    import torch

    m, n, k = 640, 384, 1000
    A = oracle.fill(m, k, 41, 1, 0)
    B = oracle.fill(k, n, 41, 2, 0)
    C = oracle.fill(m, n, 41, 3, 0)
    dA, dB = torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda()
    outs = [torch.from_numpy(C).cuda() for _ in range(4)]
    # warm-up of every route measured below
    assert _call_noalloc(path, dA, dB, outs[0], 1.5, 0.5) == sg.OK
    warm = torch.from_numpy(C).cuda()
    assert _call_noalloc(path, dA, dB, warm, 1.0, 0.0) == sg.OK
    assert _call_noalloc(path, dA[:, :0], dB[:0, :], warm, 1.5, 0.5) == sg.OK
    del warm
    before = _memory_state()
    assert _call_noalloc(path, dA, dB, outs[1], 1.5, 0.5) == sg.OK
    assert _call_noalloc(path, dA, dB, outs[2], 1.0, 0.0) == sg.OK  # beta == 0: C not read
    # k == 0: C := beta * C, no planes
    assert _call_noalloc(path, dA[:, :0], dB[:0, :], outs[3], 1.5, 0.5) == sg.OK
    after = _memory_state()
    assert sg.device_status() == sg.OK
    assert after == before, f"memory changed across the calls: {before} -> {after}"
    # the results of those calls: beta == 0 against the allocating entry point
    # (C filled with NaN, which must never be read), k == 0 against the oracle
    nan_c = torch.full((m, n), float("nan"), device="cuda")
    assert _call_noalloc(path, dA, dB, nan_c, 1.0, 0.0) == sg.OK
    want = torch.from_numpy(C).cuda()
    sg.sgemm_split(path, dA, dB, want, 1.0, 0.0)
    torch.cuda.synchronize()
    assert torch.equal(outs[2], want) and torch.equal(nan_c, want)
    want_k0 = oracle.sgemm_basic(np.zeros((m, 0), np.float32), np.zeros((0, n), np.float32), C,
                                 1.5, 0.5, basic=False)
    assert np.array_equal(outs[3].cpu().numpy(), want_k0)
    assert torch.equal(outs[0], outs[1])


@pytest.mark.parametrize("path,largest", [("bf16x6", 2361), ("tf32x3", 2048)])
def test_noalloc_size_boundary(path, largest):
    """The largest accepted cube runs and equals the allocating entry point;
    a larger problem is refused before any work."""
    import torch

    p = sg.PATHS[path]
    limit = (64 << 20) + 1024
    assert sg.split_workspace_size(p, largest, largest, largest) <= limit
    n = largest
    A = torch.empty((n, n), device="cuda")
    B = torch.empty((n, n), device="cuda")
    C0 = torch.empty((n, n), device="cuda")
    for t, X in ((1, A), (2, B), (3, C0)):
        sg.fill_random(X, 43, t, sg.DIST_UNIFORM_PM1)
    c_new, c_old = C0.clone(), C0.clone()
    assert _call_noalloc(path, A, B, c_new, 1.5, 0.5) == sg.OK
    sg.sgemm_split(path, A, B, c_old, 1.5, 0.5)
    torch.cuda.synchronize()
    assert sg.device_status() == sg.OK
    assert torch.equal(c_new, c_old)
    # the next cube is refused; TF32X3 at 2048^3 fills the scratch exactly, so
    # there one more row, column or k step (k is padded to a multiple of 8) is
    # refused too -- BF16X6's largest cube leaves slack from that padding
    beyond = [(n + 1, n + 1, n + 1)]
    if path == "tf32x3":
        beyond += [(n + 1, n, n), (n, n + 1, n), (n, n, n + 8)]
    for m2, n2, k2 in beyond:
        assert sg.split_workspace_size(p, m2, n2, k2) > limit
        A2 = torch.zeros((m2, k2), device="cuda")
        B2 = torch.zeros((k2, n2), device="cuda")
        C2 = torch.full((m2, n2), 7.0, device="cuda")
        assert _call_noalloc(path, A2, B2, C2, 1.0, 0.0) == sg.ERR_NO_MEMORY
        torch.cuda.synchronize()
        assert bool((C2 == 7.0).all())  # nothing ran


def test_noalloc_refuses_problems_beyond_its_scratch():
    import torch

    n = 4096  # BF16x6 planes for 4096^3 need 192 MiB > 64 MiB
    A = torch.zeros((n, n), device="cuda")
    C = torch.full((n, n), 7.0, device="cuda")
    assert _call_noalloc("bf16x6", A, A, C, 1.0, 0.0) == sg.ERR_NO_MEMORY
    torch.cuda.synchronize()
    assert bool((C == 7.0).all())  # nothing ran
