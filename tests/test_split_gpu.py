"""GPU tests of the split-precision tensor-core paths (BF16x6, TF32x3).

No reference counterpart exists (the reference has no tensor-core path); the
contract is sgemm()'s (src/sgemm.cuh:19-30).  Accuracy is measured against the
FP64 oracle with the componentwise metric
    max |c - c64| / (|alpha| (|A||B|)_ij + |beta| |C0|_ij)
next to the plain FFMA path's error on the same inputs.
"""
import numpy as np
import pytest

import oracle
import sgemm_b200 as sg

pytestmark = pytest.mark.gpu

PATHS = ["bf16x6", "tf32x3"]

# Small shapes: the split path's componentwise error must stay within
# 1.5x the plain FFMA path's on the same inputs, plus one FP32 ulp (2^-23)
# of slack for the rounding of the final alpha/beta step.  BF16x6 keeps ~24
# significant bits per operand (the three dropped products are below
# 3 * 2^-24 |a||b|); TF32x3 keeps ~22.
ULP = 2.0 ** -23


def _bound(plain_err):
    return 1.5 * plain_err + ULP


def _torch():
    import torch
    return torch


def _run(path, A, B, C, alpha, beta, ws=True, lds=(None, None, None)):
    torch = _torch()
    m, k = A.shape
    n = B.shape[1]

    def dev(x, ld):
        rows, cols = x.shape
        big = torch.full((rows, ld or cols), float("nan"), device="cuda")
        big[:, :cols] = torch.from_numpy(x).cuda()
        return big, big[:, :cols]

    bA, dA = dev(A, lds[0])
    bB, dB = dev(B, lds[1])
    bC, dC = dev(C, lds[2])
    work = None
    if ws:
        work = torch.empty(sg.split_workspace_size(sg.PATHS[path], m, n, k), dtype=torch.uint8,
                           device="cuda")
    sg.sgemm_split(path, dA, dB, dC, alpha, beta, workspace=work)
    torch.cuda.synchronize()
    assert sg.device_status() == sg.OK
    full = bC.cpu().numpy()
    if lds[2]:
        assert np.isnan(full[:, n:]).all(), "wrote outside the C tile"
    return full[:, :n]


def _errors(got, A, B, C, alpha, beta):
    ref, mag = oracle.dgemm(A, B, C, alpha, beta)
    return oracle.error_stats(got, ref, mag)


SHAPES = [(1, 1, 1), (7, 13, 9), (128, 256, 32), (129, 257, 33), (200, 136, 1001),
          (255, 300, 17), (300, 520, 64), (513, 260, 130)]


@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: "x".join(map(str, s)))
def test_split_accuracy_small(path, shape):
    m, n, k = shape
    A = oracle.fill(m, k, 11, 1, 0)
    B = oracle.fill(k, n, 11, 2, 0)
    C = oracle.fill(m, n, 11, 3, 0)
    got = _run(path, A, B, C, 1.5, 0.5)
    e = _errors(got, A, B, C, 1.5, 0.5)
    plain = oracle.sgemm_basic(A, B, C, 1.5, 0.5, basic=False)
    ep = _errors(plain, A, B, C, 1.5, 0.5)
    print(f"{path} {shape}: split {e['max_componentwise']:.3e} plain "
          f"{ep['max_componentwise']:.3e}")
    assert e["non_finite"] == 0
    assert e["max_componentwise"] <= _bound(ep["max_componentwise"])


@pytest.mark.parametrize("path", PATHS)
def test_split_pow2_inputs(path):
    """sign * 2^e * U[1,2), e in [-10, 10]: wide dynamic range."""
    m, n, k = 260, 300, 512
    A = oracle.fill(m, k, 12, 1, 2)
    B = oracle.fill(k, n, 12, 2, 2)
    C = oracle.fill(m, n, 12, 3, 2)
    got = _run(path, A, B, C, 1.5, 0.5)
    e = _errors(got, A, B, C, 1.5, 0.5)
    ep = _errors(oracle.sgemm_basic(A, B, C, 1.5, 0.5, basic=False), A, B, C, 1.5, 0.5)
    print(path, e, ep)
    assert e["max_componentwise"] <= _bound(ep["max_componentwise"])


@pytest.mark.parametrize("path", PATHS)
def test_split_beta_zero_and_strides(path):
    m, n, k = 140, 270, 45
    A = oracle.fill(m, k, 13, 1, 0)
    B = oracle.fill(k, n, 13, 2, 0)
    C = np.full((m, n), np.nan, dtype=np.float32)
    got = _run(path, A, B, C, 1.0, 0.0, lds=(47, 275, 273))
    assert np.isfinite(got).all()
    Z = np.zeros_like(C)
    e = _errors(got, A, B, Z, 1.0, 0.0)
    ep = _errors(oracle.sgemm_basic(A, B, Z, 1.0, 0.0, basic=False), A, B, Z, 1.0, 0.0)
    assert e["max_componentwise"] <= _bound(ep["max_componentwise"])


@pytest.mark.parametrize("path", PATHS)
def test_split_internal_workspace(path):
    """workspace=None: the call allocates and frees it stream-ordered."""
    m, n, k = 300, 200, 100
    A = oracle.fill(m, k, 14, 1, 0)
    B = oracle.fill(k, n, 14, 2, 0)
    C = oracle.fill(m, n, 14, 3, 0)
    a = _run(path, A, B, C, 1.5, 0.5, ws=True)
    b = _run(path, A, B, C, 1.5, 0.5, ws=False)
    assert np.array_equal(a, b)  # deterministic


def test_split_workspace_too_small():
    torch = _torch()
    A = torch.zeros((64, 64), device="cuda")
    ws = torch.empty(16, dtype=torch.uint8, device="cuda")
    with pytest.raises(sg.SgemmError) as e:
        sg.sgemm_split("bf16x6", A, A, A.clone(), 1.0, 0.0, workspace=ws)
    assert e.value.status == sg.ERR_NO_MEMORY


@pytest.mark.parametrize("size", [8192, 16384])
@pytest.mark.parametrize("dist", [0, 2], ids=["upm1", "pow2"])
def test_split_error_not_worse_than_plain(dist, size):
    """Whole matrices at 8192^3 and 16384^3 on the GPU FP64 oracle, for
    uniform[-1, 1) and for sign * 2^e * U[1, 2) entries: each split path's
    error must not exceed the plain FFMA path's on every statistic the
    target names -- max relative (over elements with |c64| >= 1e-3 max|c64|),
    mean relative, and max componentwise."""
    torch = _torch()
    n = size
    A = torch.empty((n, n), device="cuda")
    B = torch.empty((n, n), device="cuda")
    C0 = torch.empty((n, n), device="cuda")
    for t, X in ((1, A), (2, B), (3, C0)):
        sg.fill_random(X, 21, t, dist)
    ref, mag = oracle.gpu_reference(A, B, C0, 1.5, 0.5)
    results = {}
    C = C0.clone()
    sg.sgemm(A, B, C, 1.5, 0.5)
    results["plain"] = oracle.gpu_error_stats_vs(C, ref, mag)
    for path in PATHS:
        C.copy_(C0)
        sg.sgemm_split(path, A, B, C, 1.5, 0.5)
        torch.cuda.synchronize()
        results[path] = oracle.gpu_error_stats_vs(C, ref, mag)
    del ref, mag, C
    torch.cuda.empty_cache()
    for k, v in results.items():
        print(size, dist, k, v)
    assert sg.device_status() == sg.OK
    for path in PATHS:
        assert results[path]["non_finite"] == 0
        for stat in ("max_rel", "mean_rel", "max_componentwise"):
            assert results[path][stat] <= results["plain"][stat], (path, stat, results)


def _bf16_rn(x):
    """float32 -> nearest bfloat16 (ties to even), as float32 (finite inputs)."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def _tf32_rna(x):
    """float32 -> nearest TF32 (10-bit mantissa), ties away from zero, as the
    conversion cvt.rna.tf32.f32 rounds (finite inputs)."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = (u + 0x1000) & ~np.uint64(0x1FFF)
    return r.astype(np.uint32).view(np.float32)


def _planes(path, X):
    """The split of every element of X into the path's planes (float32)."""
    X = X.astype(np.float32)
    if path == "bf16x6":
        h = _bf16_rn(X)
        r1 = (X - h).astype(np.float32)
        m = _bf16_rn(r1)
        r2 = (r1 - m).astype(np.float32)
        return [h, m, _bf16_rn(r2)]
    h = _tf32_rna(X)
    return [h, _tf32_rna((X - h).astype(np.float32))]


@pytest.mark.parametrize("path", ["bf16x6", "tf32x3"])
@pytest.mark.parametrize("m,n,k", [(70, 90, 45), (130, 200, 136), (3, 257, 1)],
                         ids=["ragged", "multi_tile", "thin"])
def test_prepass_planes_bit_exact(path, m, n, k):
    """The pre-pass planes, read back from the caller's workspace, equal a
    numpy restatement of the split bit for bit: A as [split][m][kp] row-major,
    B transposed as [split][n][kp], kp = k rounded up to 8, zeros in the
    padding; BF16x6 stores h, m, l as bfloat16 (each the nearest bfloat16 of
    the remainder), TF32x3 stores h, l as float32 rounded to TF32."""
    torch = _torch()
    A, B, C = (oracle.fill(r, c, 31, t, 2) for r, c, t in ((m, k, 1), (k, n, 2), (m, n, 3)))
    p = sg.PATHS[path]
    ws = torch.zeros(sg.split_workspace_size(p, m, n, k) // 4 + 1, dtype=torch.float32,
                     device="cuda")
    dA, dB, dC = (torch.from_numpy(x).cuda() for x in (A, B, C))
    sg.sgemm_split(path, dA, dB, dC, 1.5, 0.5, workspace=ws)
    torch.cuda.synchronize()
    raw = ws.cpu().numpy().view(np.uint8)
    base = (-ws.data_ptr()) % 1024
    kp = (k + 7) // 8 * 8
    ns, esz = (3, 2) if path == "bf16x6" else (2, 4)
    a_bytes = (ns * m * kp * esz + 1023) // 1024 * 1024

    def read(off, rows):
        blob = raw[base + off: base + off + ns * rows * kp * esz]
        if esz == 2:
            v = (blob.view(np.uint16).astype(np.uint32) << 16).view(np.float32)
        else:
            v = blob.view(np.float32)
        return v.reshape(ns, rows, kp)

    got_a, got_b = read(0, m), read(a_bytes, n)
    Ap = np.zeros((m, kp), np.float32)
    Ap[:, :k] = A
    Bt = np.zeros((n, kp), np.float32)
    Bt[:, :k] = B.T
    for s, (pa, pb) in enumerate(zip(_planes(path, Ap), _planes(path, Bt))):
        assert np.array_equal(got_a[s].view(np.uint32), pa.view(np.uint32)), f"A plane {s}"
        assert np.array_equal(got_b[s].view(np.uint32), pb.view(np.uint32)), f"B plane {s}"
