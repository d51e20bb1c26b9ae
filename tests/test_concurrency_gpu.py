"""GPU tests of concurrent use and of randomized shapes.

The library keeps per-device state (device properties, kernel attributes,
the memory pool, the host-path engine) behind locks, and every entry point
takes a stream.  These tests run several host threads at once, each on its
own stream and its own mix of entry points, and check every result against
the same call made alone; and they compare the plain path bit for bit with
the oracle on seeded random shapes, strides and scalars.
"""
import threading

import numpy as np
import pytest

import oracle
import sgemm_b200 as sg

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    return torch


def _job(i):
    """(kind, m, n, k, alpha, beta) of thread i's call."""
    kinds = ["plain", "bf16x6", "tf32x3", "host"]
    m, n, k = 300 + 97 * i, 200 + 61 * i, 150 + 83 * i
    return kinds[i % 4], m, n, k, 1.0 + 0.25 * i, 0.5 if i % 2 else 0.0


def _run(kind, m, n, k, alpha, beta, seed, stream=None):
    torch = _torch()
    A, B, C = (oracle.fill(m, k, seed, 1, 0), oracle.fill(k, n, seed, 2, 0),
               oracle.fill(m, n, seed, 3, 0))
    if kind == "host":
        hA, hB = torch.from_numpy(A).pin_memory(), torch.from_numpy(B).pin_memory()
        hC = torch.from_numpy(C).pin_memory()
        sg.sgemm_host(hA, hB, hC, alpha, beta, stream=stream)
        (stream or torch.cuda.current_stream()).synchronize()
        return hC.numpy().copy()
    dA, dB, dC = (torch.from_numpy(x).cuda() for x in (A, B, C))
    if kind == "plain":
        sg.sgemm(dA, dB, dC, alpha, beta, stream=stream)
    else:
        sg.gemm(kind, dA, dB, dC, alpha, beta, stream=stream)
    (stream or torch.cuda.current_stream()).synchronize()
    return dC.cpu().numpy()


def test_threads_on_their_own_streams_match_single_calls():
    torch = _torch()
    n_threads = 8
    want = [_run(*_job(i), seed=40 + i) for i in range(n_threads)]
    got = [None] * n_threads
    errors = []
    barrier = threading.Barrier(n_threads)

    def worker(i):
        try:
            torch.cuda.set_device(0)
            s = torch.cuda.Stream()
            barrier.wait()
            for _ in range(3):
                got[i] = _run(*_job(i), seed=40 + i, stream=s)
        except Exception as e:  # report from the main thread
            errors.append((i, repr(e)))

    threads = [threading.Thread(target=worker, args=(i,)) for i in range(n_threads)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    for i in range(n_threads):
        assert np.array_equal(got[i], want[i]), f"thread {i} ({_job(i)[0]})"
    assert sg.device_status() == sg.OK


def test_randomized_shapes_strides_and_scalars_bit_exact():
    # seeded: shapes up to 600, row strides padded by 0..9 floats (aligned and
    # unaligned, so both loaders and the pack path run), alpha/beta including
    # zero, negative and non-representable-in-bf16 values
    torch = _torch()
    rng = np.random.default_rng(2026)
    for trial in range(40):
        m, n, k = (int(x) for x in rng.integers(1, 601, size=3))
        if trial % 10 == 0:
            k = int(rng.integers(0, 3))  # k of 0..2
        pads = [int(x) for x in rng.integers(0, 10, size=3)]
        alpha = float(rng.choice([1.0, -0.75, 1.5, 3.1415927]))
        beta = float(rng.choice([0.0, 0.5, -2.0, 1.0]))
        A, B, C = (oracle.fill(m, k, 900 + trial, 1, 0), oracle.fill(k, n, 900 + trial, 2, 0),
                   oracle.fill(m, n, 900 + trial, 3, 0))
        want = oracle.sgemm_basic(A, B, C, alpha, beta, basic=False)

        def dev(x, pad):
            r, c = x.shape
            big = torch.full((r, c + pad), float("nan"), device="cuda")
            if c:
                big[:, :c] = torch.from_numpy(x).cuda()
            return big, big[:, :c]

        _, dA = dev(A, pads[0])
        _, dB = dev(B, pads[1])
        bigC, dC = dev(C, pads[2])
        if k == 0:
            lda, ldb = 1, n + pads[1]
            st = sg.lib().sgemm_b200(m, n, 0, sg._f(alpha), 16, lda, 16, ldb, sg._f(beta),
                                     dC.data_ptr(), n + pads[2], None)
            assert st == sg.OK
        else:
            sg.sgemm(dA, dB, dC, alpha, beta)
        torch.cuda.synchronize()
        got = dC.cpu().numpy()
        both_nan = np.isnan(got) & np.isnan(want)
        assert np.array_equal(got[~both_nan], want[~both_nan]), \
            f"trial {trial}: {m}x{n}x{k} pads {pads} alpha {alpha} beta {beta}"
        if pads[2]:
            assert np.isnan(bigC[:, n:].cpu().numpy()).all(), f"trial {trial} wrote padding"
    assert sg.device_status() == sg.OK


@pytest.mark.parametrize("name", ["tma_28x256_w4p_t7x8_s3", "tma_28x256_w4p_t7x8_s4",
                                  "tma_128x64_w4p_t8x8_s4", "tma_128x64_w4_t8x8_s3"])
def test_concurrent_band_gemms_bit_exact(name):
    """Row bands of one problem as separate GEMMs, 16 in flight on four
    streams, sixteen times over: each band's bits equal one whole launch's.
    Compute warps read a shared-memory stage through the generic proxy and
    the next TMA refill writes it through the async proxy; only a proxy fence
    orders the two.  Without it, band GEMMs of the 28 x 256 producer tile
    run concurrently like this occasionally returned one warp's 28 x 32
    patch with one k block's products taken from the refill."""
    torch = _torch()
    m, n, k, rows = 8192, 4096, 3072, 512
    cfg = sg.config_names().index(name)
    A = torch.empty((m, k), device="cuda")
    B = torch.empty((k, n), device="cuda")
    C0 = torch.empty((m, n), device="cuda")
    for t, X in ((1, A), (2, B), (3, C0)):
        sg.fill_random(X, 71, t, sg.DIST_UNIFORM_PM1)
    want = C0.clone()
    sg.sgemm(A, B, want, 1.5, 0.5)
    streams = [torch.cuda.Stream() for _ in range(4)]
    torch.cuda.synchronize()
    for _ in range(16):
        C = C0.clone()
        torch.cuda.synchronize()
        for b in range(m // rows):
            s = streams[b % 4]
            with torch.cuda.stream(s):
                sg.sgemm(A[b * rows:(b + 1) * rows], B, C[b * rows:(b + 1) * rows], 1.5, 0.5,
                         stream=s, config=cfg)
        torch.cuda.synchronize()
        assert sg.device_status() == sg.OK
        bad = (C.view(torch.int32) != want.view(torch.int32)).nonzero()
        assert bad.numel() == 0, f"{name}: {bad.shape[0]} elements differ, first {bad[:3].tolist()}"
