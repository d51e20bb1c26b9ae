"""Python binding of libsgemm_b200.so (ctypes over the C ABI in include/sgemm_b200.h).

The binding is the host-side mirror the Python tests and the benchmark use: it
passes torch CUDA tensors' device pointers straight to the C ABI.  PyTorch is
only the device-memory and stream plumbing; every GEMM runs in the library's
own sm_100a kernels.  There is no fallback: if the shared library is missing
or the device is not sm_100, calls raise.

Reference mapping (szrlee/sgemm.cu):
  sgemm()        -> src/sgemm.cuh:19-90   (plain FFMA path, bit-exact)
  sgemm_basic()  -> src/sgemm.cuh:92-113  (naive one-thread-per-element kernel)
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Sequence

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libsgemm_b200.so")

OK = 0
ERR_INVALID_ARG = 1
ERR_UNSUPPORTED = 2
ERR_CUDA = 3
ERR_TIMEOUT = 4
ERR_NO_MEMORY = 5
ERR_REJECTED = 6

PATH_PLAIN = 0
PATH_BF16X6 = 1
PATH_TF32X3 = 2
PATHS = {"plain": PATH_PLAIN, "bf16x6": PATH_BF16X6, "tf32x3": PATH_TF32X3}

DIST_UNIFORM_PM1 = 0
DIST_UNIFORM_01 = 1
DIST_SIGNED_POW2 = 2


class SgemmError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        msg = status_string(status) if _lib is not None else str(status)
        if _lib is not None and status == ERR_CUDA:
            detail = _lib.sgemm_b200_last_error_detail().decode()
            if detail:
                msg += f" [{detail}]"
        super().__init__(f"{what}: {msg} (status {status})" if what else msg)


class Problem(ctypes.Structure):
    """Mirror of sgemm_b200_problem."""

    _fields_ = [
        ("m", ctypes.c_int), ("n", ctypes.c_int), ("k", ctypes.c_int),
        ("lda", ctypes.c_int), ("ldb", ctypes.c_int), ("ldc", ctypes.c_int),
        ("alpha", ctypes.c_float), ("beta", ctypes.c_float),
        ("A", ctypes.c_void_p), ("B", ctypes.c_void_p), ("C", ctypes.c_void_p),
    ]


class ServerConfig(ctypes.Structure):
    """Mirror of sgemm_b200_server_config."""

    _fields_ = [
        ("hbm_budget_bytes", ctypes.c_size_t), ("slots", ctypes.c_int),
        ("max_batch", ctypes.c_int), ("path", ctypes.c_int), ("keep_results", ctypes.c_int),
        ("inject_alloc_failure_every", ctypes.c_int), ("inject_batch_delay_ms", ctypes.c_int),
    ]


class ServerStats(ctypes.Structure):
    """Mirror of sgemm_b200_server_stats."""

    _fields_ = [
        ("submitted", ctypes.c_int64), ("completed", ctypes.c_int64),
        ("rejected", ctypes.c_int64), ("failed", ctypes.c_int64), ("batches", ctypes.c_int64),
        ("max_batches_in_flight", ctypes.c_int), ("max_batch_size", ctypes.c_int),
        ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double), ("mean_ms", ctypes.c_double),
        ("max_ms", ctypes.c_double), ("gflops", ctypes.c_double), ("wall_s", ctypes.c_double),
        ("peak_pool_bytes", ctypes.c_size_t), ("peak_waiting", ctypes.c_int64),
        ("queue_p50_ms", ctypes.c_double), ("queue_p99_ms", ctypes.c_double),
        ("service_p50_ms", ctypes.c_double), ("service_p99_ms", ctypes.c_double),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class TraceRecord(ctypes.Structure):
    """Mirror of sgemm_b200_server_trace_record."""

    _fields_ = [
        ("request_id", ctypes.c_int64), ("m", ctypes.c_int), ("n", ctypes.c_int),
        ("k", ctypes.c_int), ("batch_size", ctypes.c_int), ("batch", ctypes.c_int64),
        ("submit_ms", ctypes.c_double), ("admit_ms", ctypes.c_double),
        ("launch_ms", ctypes.c_double), ("done_ms", ctypes.c_double),
        ("device_start_ms", ctypes.c_double), ("device_end_ms", ctypes.c_double),
    ]


_lib: Optional[ctypes.CDLL] = None

# The C ABI version this binding was written against (SGEMM_B200_ABI_VERSION).
ABI_VERSION = 2

_I = ctypes.c_int
_P = ctypes.c_void_p
_FP = ctypes.POINTER(ctypes.c_float)
_GEMM_ARGS = [_I, _I, _I, _FP, _P, _I, _P, _I, _FP, _P, _I]


def _declare(lib: ctypes.CDLL) -> None:
    def d(name, res, args):
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args

    d("sgemm_b200", _I, _GEMM_ARGS + [_P])
    d("sgemm_b200_with_config", _I, [_I] + _GEMM_ARGS + [_P])
    d("sgemm_b200_config_count", _I, [])
    d("sgemm_b200_config_name", ctypes.c_char_p, [_I])
    d("sgemm_b200_select_config", _I, [_I, _I, _I, _P, _I, _P, _I, _P, _I])
    d("sgemm_b200_select_config_beta", _I, [_I, _I, _I, _P, _I, _P, _I, _FP])
    d("sgemm_b200_abi_version", _I, [])
    d("sgemm_b200_packs", _I, [_I, _I, _I, _P, _I, _P, _I])
    d("sgemm_b200_basic", _I, _GEMM_ARGS + [_P])
    d("sgemm_b200_texld", _I, _GEMM_ARGS + [_P])
    d("sgemm_b200_split_workspace_size", ctypes.c_size_t, [_I, _I, _I, _I])
    d("sgemm_b200_split", _I, [_I] + _GEMM_ARGS + [_P, ctypes.c_size_t, _P])
    d("sgemm_b200_gemm", _I, [_I] + _GEMM_ARGS + [_P])
    d("sgemm_b200_host", _I, [_I] + _GEMM_ARGS + [_P])
    d("sgemm_b200_host_plan", _I, [_I, _I, _I, _I, _I, ctypes.POINTER(_I), ctypes.POINTER(_I),
                                   _I])
    d("sgemm_b200_host_planned", _I, [_I] + _GEMM_ARGS + [_I, ctypes.POINTER(_I), _I, _P])
    d("sgemm_b200_host_plan_kouter", _I, [_I, _I, _I, _I, _I, ctypes.POINTER(_I),
                                          ctypes.POINTER(_I), ctypes.POINTER(_I)])
    d("sgemm_b200_grouped_plan_create", _I,
      [ctypes.POINTER(_P), ctypes.POINTER(Problem), _I, ctypes.c_char_p])
    d("sgemm_b200_grouped_plan_launch", _I, [_P, _P, _I])
    d("sgemm_b200_grouped_plan_info", _I,
      [_P, ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(_I)])
    d("sgemm_b200_grouped_plan_destroy", None, [_P])
    d("sgemm_b200_grouped", _I, [ctypes.POINTER(Problem), _I, _P])
    d("sgemm_b200_grouped_sequential", _I, [ctypes.POINTER(Problem), _I, _P])
    d("sgemm_b200_grouped_schedule", _I,
      [ctypes.POINTER(Problem), _I, ctypes.c_char_p, ctypes.POINTER(_I), ctypes.POINTER(_I),
       ctypes.POINTER(ctypes.c_size_t)])
    d("sgemm_b200_grouped_bucket", _I, [_I, _I, _I])
    d("sgemm_b200_grouped_split", _I, [_I, ctypes.POINTER(Problem), _I, _P])
    d("sgemm_b200_grouped_split_sequential", _I, [_I, ctypes.POINTER(Problem), _I, _P])
    d("sgemm_b200_autotune_grouped", _I, [ctypes.POINTER(Problem), _I, ctypes.c_char_p])
    d("sgemm_b200_fill_random", _I, [_P, _I, _I, _I, ctypes.c_uint64, ctypes.c_uint32, _I, _P])
    d("sgemm_b200_device_status", _I, [])
    d("sgemm_b200_pool_usage", _I, [ctypes.POINTER(ctypes.c_size_t),
                                     ctypes.POINTER(ctypes.c_size_t)])
    d("sgemm_b200_selftest_wait_timeout", _I, [_I, _P])
    d("sgemm_b200_last_status", _I, [])
    d("sgemm_b200_status_string", ctypes.c_char_p, [_I])
    d("sgemm_b200_last_error_detail", ctypes.c_char_p, [])
    d("sgemm_b200_version", ctypes.c_char_p, [])
    d("sgemm", None, _GEMM_ARGS)
    d("sgemm_basic", None, _GEMM_ARGS)
    S = ctypes.POINTER(ctypes.c_void_p)
    d("sgemm_b200_server_create", _I, [S, ctypes.POINTER(ServerConfig)])
    d("sgemm_b200_server_destroy", None, [_P])
    d("sgemm_b200_server_submit", _I, [_P, _I, _I, _I, ctypes.c_float, ctypes.c_float,
                                      ctypes.c_uint64, ctypes.POINTER(ctypes.c_int64)])
    d("sgemm_b200_server_submit_device", _I, [_P, _I, _I, _I, ctypes.c_float, _P, _I, _P, _I,
                                             ctypes.c_float, _P, _I,
                                             ctypes.POINTER(ctypes.c_int64)])
    d("sgemm_b200_server_submit_host", _I, [_P, _I, _I, _I, ctypes.c_float, _P, _I, _P, _I,
                                           ctypes.c_float, _P, _I, ctypes.POINTER(ctypes.c_int64)])
    d("sgemm_b200_server_wait", _I, [_P, ctypes.c_int64, ctypes.POINTER(ctypes.c_double)])
    d("sgemm_b200_server_isolated_ms", _I, [_P, _I, _I, _I, _I, ctypes.POINTER(ctypes.c_double)])
    d("sgemm_b200_server_drain", _I, [_P])
    d("sgemm_b200_server_result", _I, [_P, ctypes.c_int64, ctypes.POINTER(ctypes.c_double),
                                      ctypes.POINTER(_P), ctypes.POINTER(_I), ctypes.POINTER(_I)])
    d("sgemm_b200_server_read_result", _I, [_P, ctypes.c_int64, ctypes.c_void_p])
    d("sgemm_b200_server_release", _I, [_P, ctypes.c_int64])
    d("sgemm_b200_server_get_stats", _I, [_P, ctypes.POINTER(ServerStats)])
    d("sgemm_b200_server_get_trace", _I, [_P, ctypes.POINTER(TraceRecord), _I,
                                          ctypes.POINTER(ctypes.c_int)])
    d("sgemm_b200_server_run_poisson", _I, [_P, ctypes.c_double, _I, ctypes.c_uint64,
                                           ctypes.POINTER(ServerStats)])
    d("sgemm_b200_serving_workload", _I, [_I, ctypes.c_double, ctypes.c_uint64,
                                         ctypes.POINTER(_I), ctypes.POINTER(ctypes.c_double)])
    d("sgemm_b200_pool_create", _P, [ctypes.c_size_t])
    d("sgemm_b200_pool_destroy", None, [_P])
    d("sgemm_b200_pool_alloc", ctypes.c_int64, [_P, ctypes.c_size_t])
    d("sgemm_b200_pool_free", _I, [_P, ctypes.c_int64])
    d("sgemm_b200_pool_used", ctypes.c_size_t, [_P])
    d("sgemm_b200_pool_largest_free", ctypes.c_size_t, [_P])


def lib() -> ctypes.CDLL:
    """Load the shared library once; raise if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `make -C sgemm.cu_b200` "
                "(or __graft_entry__.build()); there is no fallback path")
        l = ctypes.CDLL(LIB_PATH)
        _declare(l)
        if l.sgemm_b200_abi_version() != ABI_VERSION:
            raise ImportError(f"{LIB_PATH} has C ABI version {l.sgemm_b200_abi_version()}, this "
                              f"binding needs {ABI_VERSION}: rebuild the library")
        _lib = l
    return _lib


def status_string(status: int) -> str:
    return lib().sgemm_b200_status_string(status).decode()


def _check(status: int, what: str) -> None:
    if status != OK:
        raise SgemmError(status, what)


def _f(x: float):
    return ctypes.byref(ctypes.c_float(x))


def _stream_ptr(stream) -> Optional[int]:
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream  # torch.cuda.Stream


def _mat(t, name: str, device: str = "cuda"):
    """(pointer, row stride) of a 2-D row-major float32 tensor on `device`."""
    import torch

    if t.dtype != torch.float32 or t.dim() != 2 or t.device.type != device:
        raise ValueError(f"{name} must be a 2-D float32 {device.upper()} tensor")
    if t.stride(1) != 1:
        raise ValueError(f"{name} must be row-major with unit column stride")
    ld = t.stride(0) if t.size(0) > 1 else max(t.size(1), 1)
    return t.data_ptr(), ld


def sgemm(A, B, C, alpha: float = 1.0, beta: float = 0.0, stream=None, config: int = -1) -> None:
    """C := alpha*A@B + beta*C on the plain FFMA path (in place on C)."""
    m, k = A.shape
    k2, n = B.shape
    if k2 != k or tuple(C.shape) != (m, n):
        raise ValueError("shape mismatch")
    pa, lda = _mat(A, "A")
    pb, ldb = _mat(B, "B")
    pc, ldc = _mat(C, "C")
    _check(lib().sgemm_b200_with_config(config, m, n, k, _f(alpha), pa, lda, pb, ldb, _f(beta),
                                        pc, ldc, _stream_ptr(stream)), "sgemm_b200")


def sgemm_texld(A, B, C, alpha: float = 1.0, beta: float = 0.0, stream=None) -> None:
    """The texture-fetch loader (the reference's pre-Ampere path): same result
    as sgemm(), A and B read through texture objects when aligned."""
    m, k = A.shape
    n = B.shape[1]
    pa, lda = _mat(A, "A")
    pb, ldb = _mat(B, "B")
    pc, ldc = _mat(C, "C")
    _check(lib().sgemm_b200_texld(m, n, k, _f(alpha), pa, lda, pb, ldb, _f(beta), pc, ldc,
                                  _stream_ptr(stream)), "sgemm_b200_texld")


def sgemm_basic(A, B, C, alpha: float = 1.0, beta: float = 0.0, stream=None) -> None:
    """The naive kernel (reference sgemm_basic semantics: always reads C)."""
    m, k = A.shape
    n = B.shape[1]
    pa, lda = _mat(A, "A")
    pb, ldb = _mat(B, "B")
    pc, ldc = _mat(C, "C")
    _check(lib().sgemm_b200_basic(m, n, k, _f(alpha), pa, lda, pb, ldb, _f(beta), pc, ldc,
                                  _stream_ptr(stream)), "sgemm_b200_basic")


def split_workspace_size(path: int, m: int, n: int, k: int) -> int:
    return int(lib().sgemm_b200_split_workspace_size(path, m, n, k))


def sgemm_split(path, A, B, C, alpha: float = 1.0, beta: float = 0.0, workspace=None,
                stream=None) -> None:
    """Split-precision tensor-core GEMM; path is 'bf16x6', 'tf32x3' or the enum."""
    p = PATHS[path] if isinstance(path, str) else int(path)
    m, k = A.shape
    n = B.shape[1]
    pa, lda = _mat(A, "A")
    pb, ldb = _mat(B, "B")
    pc, ldc = _mat(C, "C")
    ws, wsb = (None, 0)
    if workspace is not None:
        ws, wsb = workspace.data_ptr(), workspace.numel() * workspace.element_size()
    _check(lib().sgemm_b200_split(p, m, n, k, _f(alpha), pa, lda, pb, ldb, _f(beta), pc, ldc,
                                  ws, wsb, _stream_ptr(stream)), "sgemm_b200_split")


def gemm(path, A, B, C, alpha: float = 1.0, beta: float = 0.0, stream=None) -> None:
    p = PATHS[path] if isinstance(path, str) else int(path)
    m, k = A.shape
    n = B.shape[1]
    pa, lda = _mat(A, "A")
    pb, ldb = _mat(B, "B")
    pc, ldc = _mat(C, "C")
    _check(lib().sgemm_b200_gemm(p, m, n, k, _f(alpha), pa, lda, pb, ldb, _f(beta), pc, ldc,
                                 _stream_ptr(stream)), "sgemm_b200_gemm")


def sgemm_host(A, B, C, alpha: float = 1.0, beta: float = 0.0, path="plain",
               stream=None, plan=None) -> None:
    """C := alpha*A@B + beta*C with A, B, C in HOST memory (CPU tensors, ideally
    pinned): the library stages blocks of C through HBM with the copies
    overlapping the kernels, and writes C back in place.  `plan` = (rows per
    band, [column chunk widths]) replaces the built-in block plan."""
    p = PATHS[path] if isinstance(path, str) else int(path)
    m, k = A.shape
    k2, n = B.shape
    if k2 != k or tuple(C.shape) != (m, n):
        raise ValueError("shape mismatch")
    pa, lda = _mat(A, "A", "cpu")
    pb, ldb = _mat(B, "B", "cpu")
    pc, ldc = _mat(C, "C", "cpu")
    if plan is None:
        _check(lib().sgemm_b200_host(p, m, n, k, _f(alpha), pa, lda, pb, ldb, _f(beta), pc, ldc,
                                     _stream_ptr(stream)), "sgemm_b200_host")
        return
    rows, widths = plan
    cols = (ctypes.c_int * max(1, len(widths)))(*widths)
    _check(lib().sgemm_b200_host_planned(p, m, n, k, _f(alpha), pa, lda, pb, ldb, _f(beta), pc,
                                         ldc, int(rows), cols, len(widths),
                                         _stream_ptr(stream)), "sgemm_b200_host_planned")


def host_plan(m: int, n: int, k: int, reads_c: bool = True, path="plain") -> tuple:
    """(rows per band, [column chunk widths]) sgemm_host uses for this problem."""
    p = PATHS[path] if isinstance(path, str) else int(path)
    r = ctypes.c_int(0)
    cols = (ctypes.c_int * 16)()
    cnt = lib().sgemm_b200_host_plan(p, m, n, k, int(reads_c), ctypes.byref(r), cols, 16)
    if cnt < 0:
        raise SgemmError(-cnt, "sgemm_b200_host_plan")
    return r.value, [cols[i] for i in range(cnt)]


def host_plan_kouter(m: int, n: int, k: int, reads_c: bool = True, path="plain") -> tuple:
    """(k of the sliced phase, slices, band rows) of sgemm_host's k-outer plan
    for this problem; (0, 0, 0) when it runs the block plan instead."""
    p = PATHS[path] if isinstance(path, str) else int(path)
    k1, sl, r = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0)
    _check(lib().sgemm_b200_host_plan_kouter(p, m, n, k, int(reads_c), ctypes.byref(k1),
                                             ctypes.byref(sl), ctypes.byref(r)),
           "sgemm_b200_host_plan_kouter")
    return k1.value, sl.value, r.value


def fill_random(X, seed: int, tag: int, dist: int = DIST_UNIFORM_PM1, stream=None) -> None:
    """Fill a 2-D float32 CUDA tensor from the seeded counter-based generator."""
    px, ld = _mat(X, "X")
    _check(lib().sgemm_b200_fill_random(px, X.shape[0], X.shape[1], ld, seed, tag, dist,
                                        _stream_ptr(stream)), "sgemm_b200_fill_random")


def config_names() -> list:
    l = lib()
    return [l.sgemm_b200_config_name(i).decode() for i in range(l.sgemm_b200_config_count())]


def select_config(m: int, n: int, k: int, A=None, lda: int = 0, B=None, ldb: int = 0,
                  beta: Optional[float] = None) -> int:
    """Config id of the kernel sgemm() runs (after a pack step, if any) for
    this beta (None: C is read)."""
    pa = A.data_ptr() if A is not None else 16
    pb = B.data_ptr() if B is not None else 16
    return lib().sgemm_b200_select_config_beta(m, n, k, pa, lda or k, pb, ldb or n,
                                               None if beta is None else _f(beta))


def packs(m: int, n: int, k: int, A=None, lda: int = 0, B=None, ldb: int = 0) -> int:
    """Operands sgemm() copies to aligned rows first: bit 0 A, bit 1 B."""
    pa = A.data_ptr() if A is not None else 16
    pb = B.data_ptr() if B is not None else 16
    return lib().sgemm_b200_packs(m, n, k, pa, lda or k, pb, ldb or n)


def selftest_wait_timeout(limit_us: int, stream=None) -> None:
    """Run the bounded-wait failure path once (see include/sgemm_b200.h)."""
    _check(lib().sgemm_b200_selftest_wait_timeout(limit_us, _stream_ptr(stream)),
           "sgemm_b200_selftest_wait_timeout")


def device_status() -> int:
    return lib().sgemm_b200_device_status()


def pool_usage() -> tuple:
    """(used, reserved) bytes of the library's own memory pool on the current
    device; (0, 0) before any call has created it."""
    u, r = ctypes.c_size_t(), ctypes.c_size_t()
    _check(lib().sgemm_b200_pool_usage(ctypes.byref(u), ctypes.byref(r)), "pool_usage")
    return u.value, r.value


def make_problems(specs: Sequence) -> "ctypes.Array":
    """specs: sequence of (A, B, C, alpha, beta) torch tensors/floats."""
    arr = (Problem * len(specs))()
    for i, (A, B, C, alpha, beta) in enumerate(specs):
        pa, lda = _mat(A, "A")
        pb, ldb = _mat(B, "B")
        pc, ldc = _mat(C, "C")
        arr[i] = Problem(A.shape[0], B.shape[1], A.shape[1], lda, ldb, ldc, alpha, beta, pa, pb,
                         pc)
    return arr


def grouped_sequential(problems, stream=None) -> None:
    """The baseline: one plain sgemm_b200 launch per problem, in order."""
    _check(lib().sgemm_b200_grouped_sequential(problems, len(problems), _stream_ptr(stream)),
           "grouped_sequential")


def grouped_split(path, problems, stream=None) -> None:
    """All problems through one grouped split pre-pass and one persistent
    tcgen05 launch (path 'bf16x6' or 'tf32x3')."""
    p = PATHS[path] if isinstance(path, str) else int(path)
    _check(lib().sgemm_b200_grouped_split(p, problems, len(problems), _stream_ptr(stream)),
           "grouped_split")


def grouped_split_sequential(path, problems, stream=None) -> None:
    """The baseline: one sgemm_b200_split call per problem, in order."""
    p = PATHS[path] if isinstance(path, str) else int(path)
    _check(lib().sgemm_b200_grouped_split_sequential(p, problems, len(problems),
                                                     _stream_ptr(stream)),
           "grouped_split_sequential")


def grouped_schedule(problems, tuning_json: Optional[str] = None) -> dict:
    """Host-only schedule summary (tiles, work items, split-K workspace bytes)."""
    t, w, b = ctypes.c_int(), ctypes.c_int(), ctypes.c_size_t()
    _check(lib().sgemm_b200_grouped_schedule(problems, len(problems),
                                             tuning_json.encode() if tuning_json else None,
                                             ctypes.byref(t), ctypes.byref(w), ctypes.byref(b)),
           "grouped_schedule")
    return {"tiles": t.value, "work_items": w.value, "workspace_bytes": b.value}


def grouped_bucket(m: int, n: int, k: int) -> int:
    return lib().sgemm_b200_grouped_bucket(m, n, k)


def autotune_grouped(problems, json_path: str) -> None:
    """Time tile/split-K/stage candidates per size bucket on these problems
    (their C matrices are overwritten) and write the winners to json_path."""
    _check(lib().sgemm_b200_autotune_grouped(problems, len(problems), json_path.encode()),
           "autotune_grouped")


def host_problems(shapes) -> "ctypes.Array":
    """Problem table with placeholder pointers (for host-only schedule queries)."""
    arr = (Problem * len(shapes))()
    for i, (m, n, k) in enumerate(shapes):
        arr[i] = Problem(m, n, k, max(k, 1), max(n, 1), max(n, 1), 1.0, 0.0, 256, 256, 256)
    return arr


class GroupedPlan:
    """Persistent grouped GEMM over a fixed list of problems."""

    def __init__(self, specs: Sequence, tuning_json: Optional[str] = None):
        self._problems = make_problems(specs)
        self._keep = list(specs)  # keep tensors alive
        h = ctypes.c_void_p()
        _check(lib().sgemm_b200_grouped_plan_create(
            ctypes.byref(h), self._problems, len(specs),
            tuning_json.encode() if tuning_json else None), "grouped_plan_create")
        self._h = h

    def launch(self, stream=None, use_graph: bool = True) -> None:
        _check(lib().sgemm_b200_grouped_plan_launch(self._h, _stream_ptr(stream),
                                                    1 if use_graph else 0), "grouped_plan_launch")

    def info(self):
        t, w, g = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _check(lib().sgemm_b200_grouped_plan_info(self._h, ctypes.byref(t), ctypes.byref(w),
                                                  ctypes.byref(g)), "grouped_plan_info")
        return {"tiles": t.value, "work_items": w.value, "grid_ctas": g.value}

    def close(self) -> None:
        if self._h:
            lib().sgemm_b200_grouped_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------ serving --

class Server:
    """Continuous-batching GEMM server (include/sgemm_b200_serving.h)."""

    def __init__(self, hbm_budget_bytes: int = 64 << 30, slots: int = 2, max_batch: int = 32,
                 path="plain", keep_results: bool = False, inject_alloc_failure_every: int = 0,
                 inject_batch_delay_ms: int = 0):
        p = PATHS[path] if isinstance(path, str) else int(path)
        self.cfg = ServerConfig(hbm_budget_bytes, slots, max_batch, p, 1 if keep_results else 0,
                                inject_alloc_failure_every, inject_batch_delay_ms)
        h = ctypes.c_void_p()
        _check(lib().sgemm_b200_server_create(ctypes.byref(h), ctypes.byref(self.cfg)),
               "server_create")
        self._h = h

    def submit(self, m: int, n: int, k: int, alpha: float = 1.0, beta: float = 0.0,
               seed: int = 0) -> int:
        rid = ctypes.c_int64()
        _check(lib().sgemm_b200_server_submit(self._h, m, n, k, alpha, beta, seed,
                                              ctypes.byref(rid)), "server_submit")
        return rid.value

    def submit_device(self, A, B, C, alpha: float = 1.0, beta: float = 0.0) -> int:
        """C := alpha*A@B + beta*C on the caller's CUDA tensors, in place on C.
        The tensors must be ready on the device (synchronise their stream
        first) and left untouched until the request completes."""
        m, k = A.shape
        n = B.shape[1]
        if B.shape[0] != k or tuple(C.shape) != (m, n):
            raise ValueError("shape mismatch")
        pa, lda = _mat(A, "A")
        pb, ldb = _mat(B, "B")
        pc, ldc = _mat(C, "C")
        rid = ctypes.c_int64()
        _check(lib().sgemm_b200_server_submit_device(self._h, m, n, k, alpha, pa, lda, pb, ldb,
                                                     beta, pc, ldc, ctypes.byref(rid)),
               "server_submit_device")
        return rid.value

    def submit_host(self, A, B, C, alpha: float = 1.0, beta: float = 0.0) -> int:
        """The same with host (CPU, ideally pinned) tensors: the server copies
        them in at admission and C back after the batch."""
        m, k = A.shape
        n = B.shape[1]
        if B.shape[0] != k or tuple(C.shape) != (m, n):
            raise ValueError("shape mismatch")
        pa, lda = _mat(A, "A", "cpu")
        pb, ldb = _mat(B, "B", "cpu")
        pc, ldc = _mat(C, "C", "cpu")
        rid = ctypes.c_int64()
        _check(lib().sgemm_b200_server_submit_host(self._h, m, n, k, alpha, pa, lda, pb, ldb,
                                                   beta, pc, ldc, ctypes.byref(rid)),
               "server_submit_host")
        return rid.value

    def wait(self, rid: int) -> float:
        """Block until the request completes; returns its latency in ms."""
        lat = ctypes.c_double()
        _check(lib().sgemm_b200_server_wait(self._h, rid, ctypes.byref(lat)), "server_wait")
        return lat.value

    def isolated_ms(self, m: int, n: int, k: int, reps: int = 5) -> float:
        """Device time of one m x n x k request served alone (server idle)."""
        ms = ctypes.c_double()
        _check(lib().sgemm_b200_server_isolated_ms(self._h, m, n, k, reps, ctypes.byref(ms)),
               "server_isolated_ms")
        return ms.value

    def drain(self) -> None:
        _check(lib().sgemm_b200_server_drain(self._h), "server_drain")

    def result(self, rid: int) -> dict:
        lat, ptr, ld, bs = ctypes.c_double(), ctypes.c_void_p(), ctypes.c_int(), ctypes.c_int()
        _check(lib().sgemm_b200_server_result(self._h, rid, ctypes.byref(lat), ctypes.byref(ptr),
                                              ctypes.byref(ld), ctypes.byref(bs)), "result")
        return {"latency_ms": lat.value, "C": ptr.value, "ldc": ld.value, "batch_size": bs.value}

    def read_result(self, rid: int, m: int, n: int):
        import numpy as np
        out = np.empty((m, n), dtype=np.float32)
        _check(lib().sgemm_b200_server_read_result(self._h, rid, out.ctypes.data), "read_result")
        return out

    def release(self, rid: int) -> None:
        _check(lib().sgemm_b200_server_release(self._h, rid), "release")

    def stats(self) -> dict:
        st = ServerStats()
        _check(lib().sgemm_b200_server_get_stats(self._h, ctypes.byref(st)), "stats")
        return st.as_dict()

    def trace(self) -> list:
        """Completed requests of the statistics window, in completion order:
        one dict per request with times in ms from its first submission."""
        cap = int(self.stats()["completed"])
        buf = (TraceRecord * max(cap, 1))()
        count = ctypes.c_int(0)
        _check(lib().sgemm_b200_server_get_trace(self._h, buf, cap, ctypes.byref(count)),
               "trace")
        return [{name: getattr(buf[i], name) for name, _ in TraceRecord._fields_}
                for i in range(count.value)]

    def run_poisson(self, rate_per_s: float, n_requests: int, seed: int = 0) -> dict:
        st = ServerStats()
        _check(lib().sgemm_b200_server_run_poisson(self._h, rate_per_s, n_requests, seed,
                                                   ctypes.byref(st)), "run_poisson")
        return st.as_dict()

    def close(self) -> None:
        if self._h:
            lib().sgemm_b200_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def serving_workload(n: int, rate: float, seed: int):
    """The serving mix (host-only): list of (m, n, k) and inter-arrival gaps."""
    mnk = (ctypes.c_int * (3 * n))()
    gaps = (ctypes.c_double * n)()
    _check(lib().sgemm_b200_serving_workload(n, rate, seed, mnk, gaps), "serving_workload")
    return [tuple(mnk[3 * i:3 * i + 3]) for i in range(n)], list(gaps)
