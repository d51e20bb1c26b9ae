"""CPU tests of the C ABI boundary (no GPU compute): the library loads, exports
every function include/*.h declares, and validates arguments before touching
the device.  Reference boundary: src/sgemm.cuh:19-30 (sgemm), :92-103
(sgemm_basic)."""
import ctypes
import os
import re

import pytest

import sgemm_b200 as sg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_functions():
    names = set()
    inc = os.path.join(ROOT, "include")
    for fn in os.listdir(inc):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(inc, fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        text = re.sub(r"typedef[^;]*;", "", text, flags=re.S)
        for m in re.finditer(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", text):
            name = m.group(1)
            if name in ("if", "sizeof", "defined", "while", "for", "return"):
                continue
            names.add(name)
    return sorted(names)


def test_library_loads():
    assert sg.lib() is not None
    assert "sm_100a" in sg.lib().sgemm_b200_version().decode()


@pytest.mark.parametrize("name", _declared_functions())
def test_every_declared_symbol_is_exported(name):
    assert hasattr(sg.lib(), name), f"{name} declared in include/ but not exported"


def test_compat_signature_present():
    # The reference's exact launch surface (C linkage here).
    assert hasattr(sg.lib(), "sgemm") and hasattr(sg.lib(), "sgemm_basic")


def _call(m, n, k, alpha=1.0, beta=0.0, A=16, lda=None, B=16, ldb=None, C=16, ldc=None):
    a = ctypes.c_float(alpha)
    b = ctypes.c_float(beta)
    return sg.lib().sgemm_b200(m, n, k, ctypes.byref(a), A, lda if lda is not None else k,
                               B, ldb if ldb is not None else n, ctypes.byref(b), C,
                               ldc if ldc is not None else n, None)


def test_argument_validation():
    assert _call(-1, 4, 4) == sg.ERR_INVALID_ARG
    assert _call(4, -1, 4) == sg.ERR_INVALID_ARG
    assert _call(4, 4, -1) == sg.ERR_INVALID_ARG
    assert _call(4, 4, 4, lda=3) == sg.ERR_INVALID_ARG
    assert _call(4, 4, 4, ldb=3) == sg.ERR_INVALID_ARG
    assert _call(4, 4, 4, ldc=3) == sg.ERR_INVALID_ARG
    assert _call(4, 4, 4, A=None) == sg.ERR_INVALID_ARG
    assert _call(4, 4, 4, C=None) == sg.ERR_INVALID_ARG
    assert sg.lib().sgemm_b200(4, 4, 4, None, 16, 4, 16, 4, None, 16, 4, None) == \
        sg.ERR_INVALID_ARG
    assert sg.lib().sgemm_b200_last_status() == sg.ERR_INVALID_ARG


def test_empty_problems_are_noops():
    # m == 0 or n == 0: nothing to do, no device needed.
    assert _call(0, 5, 5, A=None, B=None, C=None) == sg.OK
    assert _call(5, 0, 5, A=None, B=None, C=None) == sg.OK


def test_status_strings():
    for s in range(7):
        assert sg.status_string(s)
    assert sg.status_string(99) == "unknown status"


def test_config_table():
    names = sg.config_names()
    assert len(names) >= 4
    assert all(n.startswith(("tma_", "cpa_")) for n in names)
    l = sg.lib()
    # unaligned strides: small problems run a cp.async configuration in place;
    # from 512^3 the offending operands are packed and a TMA configuration runs
    c = l.sgemm_b200_select_config_beta(300, 301, 299, 16, 299, 16, 301, None)
    assert names[c].startswith("cpa_") and l.sgemm_b200_packs(300, 301, 299, 16, 299, 16, 301) == 0
    c = l.sgemm_b200_select_config_beta(3001, 3001, 3001, 16, 3001, 16, 3001, None)
    assert names[c].startswith("tma_") and l.sgemm_b200_packs(3001, 3001, 3001, 16, 3001, 16,
                                                              3001) == 3
    assert l.sgemm_b200_packs(3001, 3000, 3001, 16, 3001, 16, 3000) == 1  # A only
    assert l.sgemm_b200_packs(3000, 3001, 3000, 16, 3000, 16, 3001) == 2  # B only
    assert l.sgemm_b200_packs(3001, 3001, 3001, 16, 3004, 16, 3004) == 0  # padded pitches
    assert l.sgemm_b200_packs(3000, 3000, 3000, 20, 3000, 16, 3000) == 1  # A base not 16-aligned
    c = l.sgemm_b200_select_config_beta(8192, 8192, 8192, 16, 8192, 16, 8192, None)
    assert names[c].startswith("tma_") and l.sgemm_b200_packs(8192, 8192, 8192, 16, 8192, 16,
                                                              8192) == 0


def test_select_config_keeps_its_first_signature():
    # sgemm_b200_select_config(m, n, k, A, lda, B, ldb, C, ldc) is the form the
    # first release exported; the beta-aware query is a separate entry point,
    # and the ABI version tells callers which header the library matches.
    l = sg.lib()
    assert l.sgemm_b200_abi_version() == sg.ABI_VERSION == 2
    for shape in ((300, 301, 299), (1024, 1024, 1024), (8192, 8192, 8192)):
        m, n, k = shape
        old = l.sgemm_b200_select_config(m, n, k, 16, k, 16, n, 16, n)
        assert old == l.sgemm_b200_select_config_beta(m, n, k, 16, k, 16, n, None)
        assert old == l.sgemm_b200_select_config_beta(m, n, k, 16, k, 16, n,
                                                      ctypes.byref(ctypes.c_float(0.5)))


def test_host_entry_validation_and_bands():
    l = sg.lib()
    a = ctypes.c_float(1.0)
    b = ctypes.c_float(0.5)
    # argument checks run before any device work
    assert l.sgemm_b200_host(0, 4, 4, 4, ctypes.byref(a), 16, 3, 16, 4, ctypes.byref(b), 16, 4,
                             None) == sg.ERR_INVALID_ARG
    assert l.sgemm_b200_host(9, 4, 4, 4, ctypes.byref(a), 16, 4, 16, 4, ctypes.byref(b), 16, 4,
                             None) == sg.ERR_INVALID_ARG
    assert l.sgemm_b200_host(0, 0, 4, 4, ctypes.byref(a), None, 4, None, 4, ctypes.byref(b),
                             None, 4, None) == sg.OK
    # blocking: <= 16 row bands of a multiple of 128 rows, <= 4 column chunks
    # (widths multiples of 128 but the last, each >= 512 columns); small
    # problems in one block; the split is the timing model's pick
    rows, chunks = sg.host_plan(8192, 8192, 8192)
    assert sum(chunks) == 8192 and len(chunks) >= 2 and rows % 128 == 0
    assert sg.host_plan(200, 8192, 8192)[0] == 200  # one band; B may still be chunked
    assert sg.host_plan(1000, 1000, 1000) == (1000, [1000])  # < 16 MB moved
    for m, n in ((3001, 4096), (5003, 5003), (8191, 777), (100000, 4096), (16384, 16384)):
        for path in ("plain", "bf16x6", "tf32x3"):
            r, chunks = sg.host_plan(m, n, 4096, True, path)
            assert (r % 128 == 0 and 128 <= r <= m) or r == m
            assert -(-m // r) <= 16 and 1 <= len(chunks) <= 4 and sum(chunks) == n
            assert all(c % 128 == 0 and c >= 512 for c in chunks[:-1])
            assert len(chunks) == 1 or chunks[-1] >= 512
    # the k-outer plan: plain path only, large problems with k >= 2048; its
    # sliced phase ends on a multiple of 128 (whole 32-deep k blocks), leaves
    # a k remainder for the banded phase, and its bands are whole 128-row tiles
    k1, sl, r = sg.host_plan_kouter(8192, 8192, 8192)
    assert 0 < k1 < 8192 and k1 % 128 == 0 and 1 <= sl <= 16 and r % 128 == 0
    assert -(-8192 // r) <= 16
    assert sg.host_plan_kouter(8192, 8192, 1024) == (0, 0, 0)  # short k: block plan
    assert sg.host_plan_kouter(1000, 1000, 1000) == (0, 0, 0)
    for path in ("bf16x6", "tf32x3"):
        assert sg.host_plan_kouter(8192, 8192, 8192, True, path) == (0, 0, 0)
    assert l.sgemm_b200_host_plan_kouter(0, 0, 4, 4, 1, None, None, None) == sg.ERR_INVALID_ARG

def test_host_planned_rejects_invalid_plans():
    # plan checks run before any device work (pointers are never touched)
    l = sg.lib()
    a = ctypes.c_float(1.0)
    b = ctypes.c_float(0.5)

    def call(rows, widths, m=1000, n=600):
        cols = (ctypes.c_int * max(1, len(widths)))(*widths)
        return l.sgemm_b200_host_planned(0, m, n, 64, ctypes.byref(a), 16, 64, 16, n,
                                         ctypes.byref(b), 16, n, rows, cols, len(widths), None)

    assert call(100, [300, 200]) == sg.ERR_INVALID_ARG      # widths sum to 500, not 600
    assert call(100, [300, 300, 0]) == sg.ERR_INVALID_ARG   # empty chunk
    assert call(0, [600]) == sg.ERR_INVALID_ARG             # no rows per band
    assert call(62, [600]) == sg.ERR_INVALID_ARG            # 17 bands > 16
    assert call(100, [100] * 6) == sg.ERR_INVALID_ARG       # 6 chunks > 4
    assert call(100, [], n=600) == sg.ERR_INVALID_ARG       # no chunks
    assert call(100, [600], m=0) == sg.OK                    # nothing to do


def test_selftest_wait_validation():
    # limits outside 1..10^7 microseconds are refused before any device work
    assert sg.lib().sgemm_b200_selftest_wait_timeout(0, None) == sg.ERR_INVALID_ARG
    assert sg.lib().sgemm_b200_selftest_wait_timeout(-5, None) == sg.ERR_INVALID_ARG
    assert sg.lib().sgemm_b200_selftest_wait_timeout(10000001, None) == sg.ERR_INVALID_ARG


@pytest.mark.parametrize("mirror,c_name,header", [
    (sg.Problem, "sgemm_b200_problem", "sgemm_b200.h"),
    (sg.ServerConfig, "sgemm_b200_server_config", "sgemm_b200_serving.h"),
    (sg.ServerStats, "sgemm_b200_server_stats", "sgemm_b200_serving.h"),
    (sg.TraceRecord, "sgemm_b200_server_trace_record", "sgemm_b200_serving.h"),
])
def test_ctypes_mirrors_match_the_c_layout(mirror, c_name, header, tmp_path):
    # compile a probe against the public header and compare size and every
    # field offset with the ctypes mirror
    import shutil
    import subprocess
    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    fields = [name for name, _ in mirror._fields_]
    src = tmp_path / "layout.c"
    src.write_text(
        "#include <stdio.h>\n#include <stddef.h>\n"
        f'#include "{header}"\n'
        "int main(void) {\n"
        f'  printf("%zu\\n", sizeof({c_name}));\n'
        + "".join(f'  printf("%zu\\n", offsetof({c_name}, {f}));\n' for f in fields)
        + "  return 0;\n}\n")
    exe = tmp_path / "layout"
    cuda_inc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), "-I", cuda_inc, str(src), "-o",
                    str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True,
                                          text=True).stdout.split()]
    assert got[0] == ctypes.sizeof(mirror)
    for f, off in zip(fields, got[1:]):
        assert off == getattr(mirror, f).offset, f
