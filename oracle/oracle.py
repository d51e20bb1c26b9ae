"""TEST INFRASTRUCTURE ONLY: ctypes binding of the oracle libraries.

  liboracle.so       CPU restatement of kernel_basic (reference
                     src/kernels/basic.cuh:14-25), FP64 GEMM, error stats, and
                     the seeded generator (oracle.c)
  liboracle_gpu.so   FP64 GEMM on the GPU for 8192^3 / 16384^3 accuracy checks
  _ref/libref_sgemm.so
                     the reference's own sgemm()/sgemm_basic() compiled for
                     sm_100a from its sources (ref_sgemm.cu)
  _ref/libref_sgemm_v{1,2,3}.so
                     the same sources with their PTX macros given a "memory"
                     clobber (ref_sgemm_variant.cu): loads only, stores only,
                     all -- used to locate the sgemm_128x128x8 defect

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg (and its
reference arm, which times the reference itself) may use this module, and only
as the checker or as the thing being compared against.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
CPU_LIB = os.path.join(HERE, "liboracle.so")
GPU_LIB = os.path.join(HERE, "liboracle_gpu.so")
REF_LIB = os.path.join(HERE, "_ref", "libref_sgemm.so")

_cpu = None
_gpu = None
_ref = None
_ref_variants = {}

_F32P = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_F64P = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_I32P = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_I = ctypes.c_int


def cpu() -> ctypes.CDLL:
    global _cpu
    if _cpu is None:
        l = ctypes.CDLL(CPU_LIB)
        l.oracle_fill.argtypes = [_F32P, _I, _I, _I, ctypes.c_uint64, ctypes.c_uint32, _I]
        l.oracle_fill_rows.argtypes = [_F32P, _I32P, _I, _I, ctypes.c_uint64, ctypes.c_uint32, _I]
        l.oracle_sgemm_basic.argtypes = [_I, _I, _I, ctypes.c_float, _F32P, _I, _F32P, _I,
                                         ctypes.c_float, _F32P, _I, _I, _I]
        l.oracle_sgemm_basic_rows.argtypes = [_I, _I32P, _I, _I, ctypes.c_float, _F32P, _I, _F32P,
                                              _I, ctypes.c_float, _F32P, _I, _I, _I]
        l.oracle_dgemm_rows.argtypes = [_I, ctypes.c_void_p, _I, _I, ctypes.c_double, _F32P, _I,
                                        _F32P, _I, ctypes.c_double, ctypes.c_void_p, _I, _F64P,
                                        ctypes.c_void_p, _I]
        l.oracle_error_stats.argtypes = [ctypes.c_int64, _F32P, _F64P, ctypes.c_void_p, _F64P]
        l.oracle_max_threads.restype = _I
        _cpu = l
    return _cpu


def max_threads() -> int:
    return cpu().oracle_max_threads()


def fill(rows: int, cols: int, seed: int, tag: int, dist: int) -> np.ndarray:
    X = np.empty((rows, cols), dtype=np.float32)
    if rows and cols:
        assert cpu().oracle_fill(X, rows, cols, cols, seed, tag, dist) == 0
    return X


def fill_rows(row_ids, cols: int, seed: int, tag: int, dist: int) -> np.ndarray:
    ids = np.ascontiguousarray(row_ids, dtype=np.int32)
    X = np.empty((len(ids), cols), dtype=np.float32)
    cpu().oracle_fill_rows(X, ids, len(ids), cols, seed, tag, dist)
    return X


def sgemm_basic(A: np.ndarray, B: np.ndarray, C: np.ndarray, alpha: float, beta: float,
                basic: bool = True, threads: int = 0) -> np.ndarray:
    """The reference's per-element arithmetic; returns a new array (C is not
    modified).  basic=True: kernel_basic's epilogue fma(acc, alpha, c*beta),
    C always read.  basic=False: the tiled kernels' fma(c, beta, acc*alpha),
    C not read when beta == 0."""
    m, k = A.shape
    n = B.shape[1]
    out = np.ascontiguousarray(C, dtype=np.float32).copy()
    A = np.ascontiguousarray(A, dtype=np.float32)
    B = np.ascontiguousarray(B, dtype=np.float32)
    cpu().oracle_sgemm_basic(m, n, k, alpha, A, max(k, 1), B, max(n, 1), beta, out, max(n, 1),
                             1 if basic else 0, threads)
    return out


def sgemm_basic_rows(row_ids, A: np.ndarray, B: np.ndarray, C_rows: np.ndarray, alpha: float,
                     beta: float, basic: bool = True, threads: int = 0) -> np.ndarray:
    ids = np.ascontiguousarray(row_ids, dtype=np.int32)
    m, k = A.shape
    n = B.shape[1]
    out = np.ascontiguousarray(C_rows, dtype=np.float32).copy()
    cpu().oracle_sgemm_basic_rows(len(ids), ids, n, k, alpha, np.ascontiguousarray(A), k,
                                  np.ascontiguousarray(B), n, beta, out, n,
                                  1 if basic else 0, threads)
    return out


def dgemm(A: np.ndarray, B: np.ndarray, C0: Optional[np.ndarray], alpha: float, beta: float,
          row_ids=None, threads: int = 0):
    """FP64 reference and magnitude for all rows (or the listed rows)."""
    m, k = A.shape
    n = B.shape[1]
    ids = None if row_ids is None else np.ascontiguousarray(row_ids, dtype=np.int32)
    nrows = m if ids is None else len(ids)
    ref = np.empty((nrows, n), dtype=np.float64)
    mag = np.empty((nrows, n), dtype=np.float64)
    c0p = None
    if C0 is not None:
        C0 = np.ascontiguousarray(C0, dtype=np.float32)
        c0p = C0.ctypes.data
    cpu().oracle_dgemm_rows(nrows, None if ids is None else ids.ctypes.data, n, k, alpha,
                            np.ascontiguousarray(A, dtype=np.float32), k,
                            np.ascontiguousarray(B, dtype=np.float32), n, beta, c0p, n, ref,
                            mag.ctypes.data, threads)
    return ref, mag


def error_stats(C: np.ndarray, ref: np.ndarray, mag: Optional[np.ndarray]) -> dict:
    out = np.zeros(5, dtype=np.float64)
    C = np.ascontiguousarray(C, dtype=np.float32)
    cpu().oracle_error_stats(C.size, C, np.ascontiguousarray(ref, dtype=np.float64),
                             None if mag is None else np.ascontiguousarray(mag).ctypes.data, out)
    return {"max_rel": out[0], "mean_rel": out[1], "max_componentwise": out[2],
            "n_rel": int(out[3]), "non_finite": int(out[4])}


# ----------------------------------------------------------------- GPU FP64 --

def gpu() -> ctypes.CDLL:
    global _gpu
    if _gpu is None:
        l = ctypes.CDLL(GPU_LIB)
        v = ctypes.c_void_p
        l.oracle_gpu_dgemm.argtypes = [_I, _I, _I, ctypes.c_double, v, _I, v, _I,
                                       ctypes.c_double, v, _I, v, v]
        l.oracle_gpu_error_stats.argtypes = [_I, _I, v, _I, v, v, _F64P]
        _gpu = l
    return _gpu


def gpu_reference(A, B, C0, alpha: float, beta: float):
    """(REF, MAG) as torch FP64 CUDA tensors: alpha*A@B + beta*C0 and
    |alpha||A||B| + |beta||C0|, for several error checks of one problem."""
    import torch

    m, k = A.shape
    n = B.shape[1]
    ref = torch.empty((m, n), dtype=torch.float64, device=A.device)
    mag = torch.empty((m, n), dtype=torch.float64, device=A.device)
    c0 = C0.data_ptr() if C0 is not None else None
    assert gpu().oracle_gpu_dgemm(m, n, k, alpha, A.data_ptr(), A.stride(0), B.data_ptr(),
                                  B.stride(0), beta, c0, n, ref.data_ptr(), mag.data_ptr()) == 0
    return ref, mag


def gpu_error_stats_vs(C, ref, mag) -> dict:
    """Error statistics of C (torch CUDA FP32) against gpu_reference's output."""
    m, n = C.shape
    out = np.zeros(5, dtype=np.float64)
    assert gpu().oracle_gpu_error_stats(m, n, C.data_ptr(), C.stride(0), ref.data_ptr(),
                                        mag.data_ptr(), out) == 0
    return {"max_rel": out[0], "mean_rel": out[1], "max_componentwise": out[2],
            "n_rel": int(out[3]), "non_finite": int(out[4])}


def gpu_error_stats(A, B, C0, C, alpha: float, beta: float) -> dict:
    """Full-matrix FP64 error of C (torch CUDA tensors) against alpha*A@B + beta*C0."""
    ref, mag = gpu_reference(A, B, C0, alpha, beta)
    out = gpu_error_stats_vs(C, ref, mag)
    del ref, mag
    return out


# -------------------------------------------------------- reference kernels --

def ref() -> ctypes.CDLL:
    """The reference's own sgemm()/sgemm_basic(), built from its sources."""
    global _ref
    if _ref is None:
        if not os.path.exists(REF_LIB):
            raise FileNotFoundError(f"{REF_LIB} not built (make -C oracle with the reference "
                                    "sources present)")
        l = ctypes.CDLL(REF_LIB)
        fp = ctypes.POINTER(ctypes.c_float)
        v = ctypes.c_void_p
        for name in ("ref_sgemm", "ref_sgemm_basic"):
            f = getattr(l, name)
            f.restype = None
            f.argtypes = [_I, _I, _I, fp, v, _I, v, _I, fp, v, _I]
        l.ref_sgemm_kernel_choice.argtypes = [_I, _I]
        l.ref_sgemm_kernel_choice.restype = _I
        _ref = l
    return _ref


def ref_sgemm(A, B, C, alpha: float, beta: float, basic: bool = False) -> None:
    """Run the reference's sgemm() (or sgemm_basic()) on torch CUDA tensors.

    The reference requires ldb == ldc == n (its kernels advance B and C by n);
    callers pass contiguous tensors.
    """
    m, k = A.shape
    n = B.shape[1]
    a = ctypes.c_float(alpha)
    b = ctypes.c_float(beta)
    f = ref().ref_sgemm_basic if basic else ref().ref_sgemm
    f(m, n, k, ctypes.byref(a), A.data_ptr(), A.stride(0), B.data_ptr(), B.stride(0),
      ctypes.byref(b), C.data_ptr(), C.stride(0))


def ref_variant(v: int) -> ctypes.CDLL:
    """The reference's sgemm() with its PTX macros redefined from outside:
    v = 1, 2, 3 a "memory" clobber on the shared loads, the shared stores, every
    macro; v = 4 a record of the shared addresses; v = 5 shared addresses
    rebased onto the 16 KB boundary the kernels' XOR double buffering assumes
    (test-only repair of sgemm_128x128x8)."""
    if v not in _ref_variants:
        path = os.path.join(HERE, "_ref", f"libref_sgemm_v{v}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} not built (make -C oracle REF_ROOT=...)")
        l = ctypes.CDLL(path)
        fp = ctypes.POINTER(ctypes.c_float)
        v_ = ctypes.c_void_p
        l.ref_sgemm.restype = None
        l.ref_sgemm.argtypes = [_I, _I, _I, fp, v_, _I, v_, _I, fp, v_, _I]
        l.ref_variant.restype = _I
        assert l.ref_variant() == v
        if v == 4:
            l.ref_probe_reset.restype = _I
            l.ref_probe_read.restype = _I
            l.ref_probe_read.argtypes = [ctypes.c_void_p]
        _ref_variants[v] = l
    return _ref_variants[v]


def ref_sgemm_variant(v: int, A, B, C, alpha: float, beta: float) -> None:
    """Run variant v of the reference's sgemm() on torch CUDA tensors
    (contiguous, ldb == ldc == n as the reference requires)."""
    m, k = A.shape
    n = B.shape[1]
    a = ctypes.c_float(alpha)
    b = ctypes.c_float(beta)
    ref_variant(v).ref_sgemm(m, n, k, ctypes.byref(a), A.data_ptr(), A.stride(0), B.data_ptr(),
                             B.stride(0), ctypes.byref(b), C.data_ptr(), C.stride(0))


# Variant 5's rebase (ref_sgemm_variant.cu REF_REBASE): the bytes by which the
# reference kernels' shared array sits past the 16 KB boundary they assume.
REF_REBASE = 1024


def ref_rebased_premise() -> bool:
    """Whether variant 5 may run here: both reference kernels' shared array
    starts REF_REBASE bytes past a 16 KB boundary, read from variant 4's record
    on a small problem of each kernel (main loop included).  With any other
    base the rebased addresses would not be the array's."""
    import torch
    for m, n in ((128, 128), (2560, 256)):  # sgemm_128x128x8, then sgemm_128x256x8
        A = torch.zeros(m, 16, device="cuda")
        B = torch.zeros(16, n, device="cuda")
        C = torch.zeros(m, n, device="cuda")
        addrs = ref_shared_addresses(A, B, C, 1.0, 0.0)
        if len(addrs) < 2 or addrs[0] % 16384 != REF_REBASE or addrs[1] - addrs[0] != 16384:
            return False
    return True


def ref_shared_addresses(A, B, C, alpha: float, beta: float) -> list:
    """Run variant 4 of the reference's sgemm() once and return the shared
    addresses its address-conversion macro produced for block (0, 0) thread 0,
    in call order."""
    import torch
    l = ref_variant(4)
    assert l.ref_probe_reset() == 0
    ref_sgemm_variant(4, A, B, C, alpha, beta)
    torch.cuda.synchronize()
    out = (ctypes.c_ulonglong * 16)()
    n = l.ref_probe_read(ctypes.addressof(out))
    assert n >= 0
    return [int(out[i]) for i in range(min(n, 16))]
