"""GPU parity of the plain FFMA path against the oracle and the reference's
own kernels.  All comparisons are exact (float equality): the plain path
accumulates every C element over k in increasing order with one FMA per term,
then applies alpha and beta the way the reference does
(src/kernels/128x256x8.cuh:224-239, :331-337, :365-380;
src/kernels/basic.cuh:18-24), so its outputs are bit-identical.
"""
import os
import subprocess

import numpy as np
import pytest

import oracle
import sgemm_b200 as sg

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _torch():
    import torch
    return torch


def _inputs(m, n, k, seed, dist):
    return (oracle.fill(m, k, seed, 1, dist), oracle.fill(k, n, seed, 2, dist),
            oracle.fill(m, n, seed, 3, dist))


def _dev(x, ld=None):
    """Copy a host matrix to the device, optionally inside a wider allocation
    (row stride ld) whose extra columns hold NaN canaries."""
    torch = _torch()
    rows, cols = x.shape
    ld = ld or cols
    big = torch.full((rows, ld), float("nan"), dtype=torch.float32, device="cuda")
    big[:, :cols] = torch.from_numpy(x).cuda()
    return big, big[:, :cols]


def _run_ours(A, B, C, alpha, beta, lds=(None, None, None), config=-1):
    torch = _torch()
    bA, dA = _dev(A, lds[0])
    bB, dB = _dev(B, lds[1])
    bC, dC = _dev(C, lds[2])
    sg.sgemm(dA, dB, dC, alpha, beta, config=config)
    torch.cuda.synchronize()
    assert sg.device_status() == sg.OK
    full = bC.cpu().numpy()
    if lds[2]:
        assert np.isnan(full[:, C.shape[1]:]).all(), "wrote outside the C tile"
    return full[:, :C.shape[1]]


def _assert_equal(got, want):
    diff = got != want
    both_nan = np.isnan(got) & np.isnan(want)
    n = int((diff & ~both_nan).sum())
    assert n == 0, f"{n} of {got.size} elements differ (max |d| "\
        f"{np.nanmax(np.abs(got.astype(np.float64) - want)):.3e})"


SHAPES = [(1, 1, 1), (2, 3, 4), (7, 13, 9), (31, 33, 35), (64, 64, 64), (127, 129, 128),
          (128, 256, 32), (129, 257, 33), (200, 136, 1001), (255, 300, 17), (1000, 1000, 1000),
          (97, 1031, 61), (1031, 97, 263)]


@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: "x".join(map(str, s)))
@pytest.mark.parametrize("ab", [(1.5, 0.5), (1.0, 0.0)], ids=["a1.5b0.5", "a1b0"])
def test_plain_bit_exact_vs_oracle(shape, ab):
    m, n, k = shape
    alpha, beta = ab
    A, B, C = _inputs(m, n, k, 1, 0)
    got = _run_ours(A, B, C, alpha, beta)
    want = oracle.sgemm_basic(A, B, C, alpha, beta, basic=False)
    _assert_equal(got, want)


@pytest.mark.parametrize("cfg", range(len(sg.config_names())))
@pytest.mark.parametrize("shape", [(130, 270, 77), (64, 128, 32), (300, 64, 100)],
                         ids=lambda s: "x".join(map(str, s)))
def test_every_config_bit_exact(cfg, shape):
    names = sg.config_names()
    if cfg >= len(names):
        pytest.skip("config not built")
    m, n, k = shape
    A, B, C = _inputs(m, n, k, 2, 2)
    if names[cfg].startswith("tma_") and (k % 4 or n % 4):
        # TMA needs 16-byte row strides; a forced TMA config must refuse.
        with pytest.raises(sg.SgemmError) as e:
            _run_ours(A, B, C, 1.5, 0.5, config=cfg)
        assert e.value.status == sg.ERR_INVALID_ARG
        return
    got = _run_ours(A, B, C, 1.5, 0.5, config=cfg)
    _assert_equal(got, oracle.sgemm_basic(A, B, C, 1.5, 0.5, basic=False))


@pytest.mark.parametrize("name", ["tma_28x256_w4p_t7x8_s4", "tma_28x256_w4p_t7x8_s3"])
@pytest.mark.parametrize("m,n,k,ldc,ab", [
    (1024, 1024, 1024, None, (1.0, 0.0)),   # 37 x 4 tiles, the last row tile 16 rows
    (1000, 1000, 1000, None, (1.5, 0.5)),   # 36 x 4 tiles, ragged columns
    (57, 300, 72, 301, (1.5, 0.5)),         # C rows not 16-byte aligned: staged epilogue
    (28, 256, 8, None, (1.0, 0.0)),         # exactly one tile, one k block
], ids=["1024", "1000", "ldc_odd", "one_tile"])
def test_seven_row_thread_tile_bit_exact(name, m, n, k, ldc, ab):
    # the 28 x 256 tile: 7 rows per thread, so each warp's rows start at a
    # multiple of 28 and the A swizzle phase follows the row, not the lane
    cfg = sg.config_names().index(name)
    A, B, C = _inputs(m, n, k, 9, 0)
    if ab[1] == 0.0:
        C = np.full((m, n), np.nan, dtype=np.float32)  # beta == 0: C is never read
    got = _run_ours(A, B, C, *ab, lds=(None, None, ldc), config=cfg)
    if ab[1] == 0.0:
        assert np.isfinite(got).all()
    _assert_equal(got, oracle.sgemm_basic(A, B, C, *ab, basic=False))


@pytest.mark.parametrize("size,beta,want", [
    (1024, 0.0, "tma_28x256_w4p_t7x8_s4"),
    (1024, 0.5, "tma_28x256_w4p_t7x8_s4"),
    (1000, 0.5, "tma_28x256_w4p_t7x8_s4"),
    (2048, 0.5, "tma_28x256_w4p_t7x8_s3"),
    (8192, 0.5, "tma_128x64_w4_t8x8_s3"),
])
def test_dispatch_picks_the_measured_fastest_tile(size, beta, want):
    # the cost model's choice at sizes where every configuration was timed
    # against the others on a B200: a change to the model (or to a tile's
    # shared memory or registers, which set its CTAs per SM) that moves one of
    # these sizes off its fastest tile fails here
    assert sg.config_names()[sg.select_config(size, size, size, beta=beta)] == want


@pytest.mark.parametrize("lds", [(None, None, None), (36, 52, 60), (33, 49, 51), (37, 48, 50)],
                         ids=["packed", "ld_aligned", "ld_odd", "lda_odd"])
def test_general_strides_and_canaries(lds):
    m, n, k = 45, 47, 33
    A, B, C = _inputs(m, n, k, 3, 0)
    got = _run_ours(A, B, C, 1.5, 0.5, lds=lds)
    _assert_equal(got, oracle.sgemm_basic(A, B, C, 1.5, 0.5, basic=False))


@pytest.mark.parametrize("m,n,k,pads", [(1001, 3001, 777, (1, 1, 1)), (1003, 1500, 1201, (2, 0, 3)),
                                        (997, 1501, 1000, (0, 1, 0))],
                         ids=["pack_a_and_b", "pack_a", "pack_b"])
def test_pack_path_matches_the_oracle(m, n, k, pads):
    # row strides that are not multiples of 4 floats on problems above 512^3:
    # the offending operands are packed to aligned rows, then the TMA kernel
    # runs; the result is the oracle's, bit for bit
    A, B, C = _inputs(m, n, k, 23, 0)
    lds = (k + pads[0], n + pads[1], n + pads[2])
    got = _run_ours(A, B, C, 1.5, 0.5, lds=lds)
    _assert_equal(got, oracle.sgemm_basic(A, B, C, 1.5, 0.5, basic=False))


@pytest.mark.parametrize("m,n,k,pads,tile", [
    (1001, 1001, 1001, (1, 1, 1), "tma_28x256_w4p_t7x8_s4"),
    (2049, 2047, 1999, (3, 1, 1), "tma_28x256_w4p_t7x8_s3"),
], ids=["1001_both_packed", "2049_a_packed"])
def test_pack_path_on_the_28_row_tiles(m, n, k, pads, tile):
    # unaligned strides at the sizes where the dispatcher picks a 28 x 256
    # tile: the operands are packed to aligned rows, that tile runs, and the
    # result is the oracle's bit for bit
    lds = (k + pads[0], n + pads[1], n + pads[2])
    assert sg.config_names()[sg.select_config(m, n, k, None, lds[0], None, lds[1],
                                              beta=0.5)] == tile
    A, B, C = _inputs(m, n, k, 29, 0)
    got = _run_ours(A, B, C, 1.5, 0.5, lds=lds)
    _assert_equal(got, oracle.sgemm_basic(A, B, C, 1.5, 0.5, basic=False))


def test_beta_zero_never_reads_c():
    m, n, k = 140, 260, 40
    A, B, _ = _inputs(m, n, k, 4, 0)
    C = np.full((m, n), np.nan, dtype=np.float32)
    got = _run_ours(A, B, C, 1.0, 0.0)
    assert np.isfinite(got).all()
    _assert_equal(got, oracle.sgemm_basic(A, B, C, 1.0, 0.0, basic=False))


def test_k_zero_scales_c():
    m, n = 50, 70
    C = oracle.fill(m, n, 5, 3, 0)
    A = np.zeros((m, 0), dtype=np.float32)
    B = np.zeros((0, n), dtype=np.float32)
    torch = _torch()
    dC = torch.from_numpy(C).cuda()
    dA = torch.zeros((m, 1), device="cuda")[:, :0]
    dB = torch.zeros((1, n), device="cuda")[:0, :]
    sg.sgemm(dA, dB, dC, 1.5, 0.5)
    torch.cuda.synchronize()
    _assert_equal(dC.cpu().numpy(), oracle.sgemm_basic(A, B, C, 1.5, 0.5))


def _device_inputs(m, n, k, seed):
    torch = _torch()
    A = torch.empty((m, k), device="cuda")
    B = torch.empty((k, n), device="cuda")
    C = torch.empty((m, n), device="cuda")
    sg.fill_random(A, seed, 1, sg.DIST_UNIFORM_PM1)
    sg.fill_random(B, seed, 2, sg.DIST_UNIFORM_PM1)
    sg.fill_random(C, seed, 3, sg.DIST_UNIFORM_PM1)
    torch.cuda.synchronize()
    return A, B, C


@pytest.mark.parametrize("shape", [(2600, 2600, 2600), (3001, 3001, 3001), (4096, 4096, 4096),
                                   (2501, 640, 1000)], ids=lambda s: "x".join(map(str, s)))
def test_bit_exact_vs_reference_128x256x8(shape):
    """Same seeded inputs through the reference's own sgemm() (built from its
    sources for sm_100a) and through ours; ldb == ldc == n as the reference
    requires.  With m > 2500 or n > 2500 the reference runs sgemm_128x256x8
    (src/sgemm.cuh:42-44), whose results ours must equal bit for bit."""
    torch = _torch()
    m, n, k = shape
    assert oracle.ref().ref_sgemm_kernel_choice(m, n) == 1
    A, B, C = _device_inputs(m, n, k, 6)
    C_ref = C.clone()
    torch.cuda.synchronize()
    sg.sgemm(A, B, C, 1.5, 0.5)
    oracle.ref_sgemm(A, B, C_ref, 1.5, 0.5)
    torch.cuda.synchronize()
    assert torch.equal(C, C_ref)


def test_reference_128x128x8_defect_vs_ours():
    """Recorded finding: at m, n <= 2500 the reference dispatches
    sgemm_128x128x8, which built for sm_100a returns wrong values once k > 8
    (see tests/test_oracle.py::test_reference_128x128x8_defect_on_sm100).
    Ours must equal the oracle exactly on the same inputs."""
    torch = _torch()
    m = n = k = 1000
    A, B, C = _inputs(m, n, k, 6, 0)
    dA, dB = torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda()
    c_ours, c_ref = torch.from_numpy(C).cuda(), torch.from_numpy(C).cuda()
    sg.sgemm(dA, dB, c_ours, 1.5, 0.5)
    oracle.ref_sgemm(dA, dB, c_ref, 1.5, 0.5)
    torch.cuda.synchronize()
    want = oracle.sgemm_basic(A, B, C, 1.5, 0.5, basic=False)
    _assert_equal(c_ours.cpu().numpy(), want)
    ref, mag = oracle.dgemm(A, B, C, 1.5, 0.5)
    assert oracle.error_stats(c_ref.cpu().numpy(), ref, mag)["max_componentwise"] > 1e-3


def test_reference_naive_kernel_matches_ours():
    """sgemm_b200_basic equals the reference's sgemm_basic()/kernel_basic bit
    for bit (epilogue fma(acc, alpha, c*beta), C always read)."""
    torch = _torch()
    m, n, k = 77, 91, 129
    A, B, C = _inputs(m, n, k, 7, 0)
    dA, dB = torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda()
    c1, c2 = torch.from_numpy(C).cuda(), torch.from_numpy(C).cuda()
    sg.sgemm_basic(dA, dB, c1, 1.5, 0.5)
    oracle.ref_sgemm(dA, dB, c2, 1.5, 0.5, basic=True)
    torch.cuda.synchronize()
    _assert_equal(c1.cpu().numpy(), oracle.sgemm_basic(A, B, C, 1.5, 0.5, basic=True))
    assert torch.equal(c1, c2)


@pytest.mark.parametrize("rows,cols,ld", [(33, 129, 129), (40, 256, 256), (33, 129, 132),
                                          (3, 5000, 5003), (70000, 3, 4)],
                         ids=["odd_rows", "aligned", "aligned_pitch_ragged", "wide", "tall"])
def test_device_fill_matches_host_generator(rows, cols, ld):
    # every element's value depends only on (seed, tag, row * cols + col):
    # scalar and float4 stores, any pitch, more rows than one grid dimension
    torch = _torch()
    for dist in (0, 1, 2):
        big = torch.full((rows, ld), float("nan"), device="cuda")
        X = big[:, :cols]
        sg.fill_random(X, 99, 4, dist)
        torch.cuda.synchronize()
        want = oracle.fill(rows, cols, 99, 4, dist)
        got = big.cpu().numpy()
        assert np.array_equal(got[:, :cols].view(np.uint32), want.view(np.uint32))
        assert np.isnan(got[:, cols:]).all()


@pytest.mark.parametrize("size", [4096, 8192])
def test_large_sizes_sampled_rows(size):
    """Full-size check by property: 48 sampled rows recomputed by the oracle
    from the generator must match exactly."""
    torch = _torch()
    m = n = k = size
    A = torch.empty((m, k), device="cuda")
    B = torch.empty((k, n), device="cuda")
    C = torch.empty((m, n), device="cuda")
    for t, X in ((1, A), (2, B), (3, C)):
        sg.fill_random(X, 8, t, sg.DIST_UNIFORM_PM1)
    rows = np.linspace(0, m - 1, 48).astype(np.int32)
    C0_rows = C[torch.from_numpy(rows).long().cuda()].cpu().numpy()
    sg.sgemm(A, B, C, 1.5, 0.5)
    torch.cuda.synchronize()
    got = C[torch.from_numpy(rows).long().cuda()].cpu().numpy()
    hA = oracle.fill(m, k, 8, 1, 0)
    hB = oracle.fill(k, n, 8, 2, 0)
    want = oracle.sgemm_basic_rows(rows, hA, hB, C0_rows, 1.5, 0.5, basic=False)
    _assert_equal(got, want)


def test_compat_entry_on_default_stream():
    torch = _torch()
    import ctypes
    m, n, k = 65, 66, 67
    A, B, C = _inputs(m, n, k, 9, 1)
    dA, dB, dC = (torch.from_numpy(x).cuda() for x in (A, B, C))
    a, b = ctypes.c_float(1.5), ctypes.c_float(0.5)
    sg.lib().sgemm(m, n, k, ctypes.byref(a), dA.data_ptr(), k, dB.data_ptr(), n, ctypes.byref(b),
                   dC.data_ptr(), n)
    torch.cuda.synchronize()
    assert sg.lib().sgemm_b200_last_status() == sg.OK
    _assert_equal(dC.cpu().numpy(), oracle.sgemm_basic(A, B, C, 1.5, 0.5, basic=False))


def test_cpp_harness_sweep(tmp_path):
    exe = os.path.join(ROOT, "sgemm.cu_b200", "bin", "test_sgemm")
    r = subprocess.run([exe, "--mmin=2", "--mmax=300", "--mstep=23",
                        f"--savedir={tmp_path}"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "FAILED: 0" in r.stdout


@pytest.mark.parametrize("m,n,k,ld_pad", [(2048, 1536, 1024, 0), (1001, 3001, 777, 1)])
def test_plain_path_captures_into_a_cuda_graph(m, n, k, ld_pad):
    # one launch with by-value tensor maps (aligned case) or the pack path's
    # stream-ordered scratch plus the launch (unaligned case): both capture,
    # and every replay gives the direct call's bits
    torch = _torch()
    A, B, C = _inputs(m, n, k, 17, 0)
    lds = (k + ld_pad, n + ld_pad, n + ld_pad) if ld_pad else (None, None, None)
    want = _run_ours(A, B, C, 1.5, 0.5, lds=lds)
    _, dA = _dev(A, lds[0])
    _, dB = _dev(B, lds[1])
    bigC, dC = _dev(C, lds[2])
    C0 = dC.clone()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        sg.sgemm(dA, dB, dC, 1.5, 0.5, stream=s)  # first call outside capture: lazy set-up
        s.synchronize()
        dC.copy_(C0)
        s.synchronize()
        with torch.cuda.graph(g, stream=s):
            sg.sgemm(dA, dB, dC, 1.5, 0.5, stream=s)
    for _ in range(2):
        dC.copy_(C0)
        g.replay()
        torch.cuda.synchronize()
        assert np.array_equal(dC.cpu().numpy(), want)
    del g


def _special(shape, seed):
    """U[-1,1) entries with subnormals, exact zeros, signed zeros, magnitudes
    whose products overflow to +-Inf, and a few NaNs mixed in."""
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1, 1, size=shape).astype(np.float32)
    pick = rng.random(shape)
    x[pick < 0.05] = (rng.uniform(-1, 1, size=shape) * 1e-39).astype(np.float32)[pick < 0.05]
    x[(pick >= 0.05) & (pick < 0.08)] = 0.0
    x[(pick >= 0.08) & (pick < 0.09)] = -0.0
    x[(pick >= 0.09) & (pick < 0.092)] = np.float32(3e38)
    x[(pick >= 0.092) & (pick < 0.0925)] = np.nan
    return x


@pytest.mark.parametrize("config", ["default", "cpa"])
def test_special_values_bit_exact(config):
    # subnormals are kept (no flush to zero), Inf and NaN propagate: the packed
    # FMA core rounds exactly like the reference's fmaf chain
    A = _special((300, 257), 1)
    B = _special((257, 200), 2)
    C = _special((300, 200), 3)
    cfg = -1 if config == "default" else sg.config_names().index("cpa_64x128_w4_t8x8_s4")
    got = _run_ours(A, B, C, 1.5, 0.5, config=cfg)
    want = oracle.sgemm_basic(A, B, C, 1.5, 0.5, basic=False)
    _assert_equal(got, want)
    # the products of subnormals with ordinary values are subnormal, not zero
    tiny = np.full((64, 64), 1e-39, np.float32)
    one = np.eye(64, dtype=np.float32)
    got = _run_ours(tiny, one, np.zeros((64, 64), np.float32), 1.0, 0.0, config=cfg)
    assert np.array_equal(got, tiny)


@pytest.mark.parametrize("m,n,k,pad", [(300, 200, 150, 0), (257, 129, 1000, 3), (64, 1000, 33, 8)])
def test_column_major_callers_swap_operands(m, n, k, pad):
    # the reference's convention for column-major data (src/sgemm.cuh:31-33):
    # swap (A, lda) with (B, ldb) and m with n, since C^T = B^T * A^T.  A
    # column-major m x k array with leading dimension lda is, byte for byte,
    # a row-major k x m array with row stride lda, so nothing is copied.
    import ctypes

    torch = _torch()
    A, B, C = _inputs(m, n, k, 23, 0)
    want = oracle.sgemm_basic(A, B, C, 1.5, 0.5, basic=False)
    lda, ldb, ldc = m + pad, k + pad, m + pad
    _, dAc = _dev(np.ascontiguousarray(A.T), lda)  # A column-major: k rows of lda
    _, dBc = _dev(np.ascontiguousarray(B.T), ldb)  # B column-major: n rows of ldb
    bigC, dCc = _dev(np.ascontiguousarray(C.T), ldc)  # C column-major: n rows of ldc
    a, b = ctypes.c_float(1.5), ctypes.c_float(0.5)
    st = sg.lib().sgemm_b200(n, m, k, ctypes.byref(a), dBc.data_ptr(), ldb, dAc.data_ptr(), lda,
                             ctypes.byref(b), dCc.data_ptr(), ldc, None)
    assert st == sg.OK
    torch.cuda.synchronize()
    _assert_equal(np.ascontiguousarray(dCc.cpu().numpy().T), want)
