"""CPU tests of the serving loop's host-side pieces: the HBM pool allocator
and the request-mix generator (no reference counterpart)."""
import ctypes
import math

import pytest

import sgemm_b200 as sg


def _pool(cap):
    return sg.lib().sgemm_b200_pool_create(cap)


def test_pool_first_fit_and_coalescing():
    l = sg.lib()
    p = _pool(4096)
    a = l.sgemm_b200_pool_alloc(p, 1000)  # rounds to 1024
    b = l.sgemm_b200_pool_alloc(p, 1024)
    c = l.sgemm_b200_pool_alloc(p, 2048)
    assert (a, b, c) == (0, 1024, 2048)
    assert l.sgemm_b200_pool_alloc(p, 1) == -1  # full
    assert l.sgemm_b200_pool_used(p) == 4096
    assert l.sgemm_b200_pool_free(p, b) == sg.OK
    assert l.sgemm_b200_pool_largest_free(p) == 1024
    assert l.sgemm_b200_pool_alloc(p, 2048) == -1  # fragmented: no 2 KB hole
    assert l.sgemm_b200_pool_free(p, a) == sg.OK  # coalesces with b's hole
    assert l.sgemm_b200_pool_largest_free(p) == 2048
    assert l.sgemm_b200_pool_alloc(p, 2048) == 0
    assert l.sgemm_b200_pool_free(p, 12345) == sg.ERR_INVALID_ARG  # not an allocation
    assert l.sgemm_b200_pool_free(p, c) == sg.OK
    assert l.sgemm_b200_pool_free(p, 0) == sg.OK
    assert l.sgemm_b200_pool_used(p) == 0
    assert l.sgemm_b200_pool_largest_free(p) == 4096
    l.sgemm_b200_pool_destroy(p)


def test_pool_alignment():
    l = sg.lib()
    p = _pool(1 << 20)
    offs = [l.sgemm_b200_pool_alloc(p, s) for s in (1, 17, 255, 257, 4000)]
    assert all(o % 256 == 0 for o in offs)
    assert len(set(offs)) == len(offs)
    l.sgemm_b200_pool_destroy(p)


def test_workload_mix_and_rate():
    shapes, gaps = sg.serving_workload(20000, 500.0, 3)
    tall = [s for s in shapes if s[1] == 4096 and s[2] == 4096 and s[0] <= 256]
    square = [s for s in shapes if s[0] == s[1] == s[2] and s[0] >= 512]
    assert len(tall) + len(square) == len(shapes)
    assert abs(len(tall) / len(shapes) - 0.6) < 0.02
    assert min(s[0] for s in tall) >= 16 and max(s[0] for s in tall) <= 256
    assert all(s[0] % 8 == 0 and 512 <= s[0] <= 4096 for s in square)
    # log-uniform: the median of the square sizes sits near sqrt(512*4096)
    med = sorted(s[0] for s in square)[len(square) // 2]
    assert abs(math.log(med) - 0.5 * (math.log(512) + math.log(4096))) < 0.1
    mean_gap = sum(gaps) / len(gaps)
    assert abs(mean_gap * 500.0 - 1.0) < 0.05
    # deterministic by seed
    assert sg.serving_workload(50, 500.0, 3) == sg.serving_workload(50, 500.0, 3)
    assert sg.serving_workload(50, 500.0, 3) != sg.serving_workload(50, 500.0, 4)


def test_server_config_validation():
    h = ctypes.c_void_p()
    cfg = sg.ServerConfig(0, 1, 1, 0, 0, 0, 0)  # zero budget
    assert sg.lib().sgemm_b200_server_create(ctypes.byref(h), ctypes.byref(cfg)) == \
        sg.ERR_INVALID_ARG
    cfg = sg.ServerConfig(1 << 30, 0, 1, 0, 0, 0, 0)  # no slots
    assert sg.lib().sgemm_b200_server_create(ctypes.byref(h), ctypes.byref(cfg)) == \
        sg.ERR_INVALID_ARG
