"""Host CBLAS, the CPU GEMM path hcBLAS's tests compare against (checker / baseline only).

hcBLAS's unit tests call ``cblas_{s,d,c,z}gemm`` from the system ``libblas``
(test/unit/hcblas_sgemm.cpp:28 and :252, linked at test/unit/CMakeLists.txt:30);
that library is an un-vendored, unpinned third-party dependency.  This image
ships OpenBLAS 0.3.30 inside the scipy wheel (``scipy.libs/libscipy_openblas-*.so``),
which exports the standard CBLAS entry points with a ``scipy_`` prefix.  This
module binds those with ctypes.  It is used (1) by tests/golden/make_golden.py to
produce golden vectors from a real CBLAS, and (2) by bench.py's CPU-baseline leg
and ``--impl reference`` arm to time the host CBLAS path.  The product library
never calls it.
"""
from __future__ import annotations

import ctypes
import glob
import os

import numpy as np

CblasRowMajor, CblasColMajor = 101, 102
CblasNoTrans, CblasTrans, CblasConjTrans = 111, 112, 113

_ORDER = {0: CblasRowMajor, 1: CblasColMajor}  # hcblasOrder RowMajor=0, ColMajor=1
_TRANS = {0: CblasNoTrans, 1: CblasTrans, 2: CblasConjTrans}

_lib = None
_path = None


def library_path():
    import scipy

    base = os.path.join(os.path.dirname(os.path.dirname(scipy.__file__)), "scipy.libs")
    cands = sorted(glob.glob(os.path.join(base, "libscipy_openblas-*.so")))
    if not cands:
        raise RuntimeError("no OpenBLAS build found next to scipy")
    return cands[0]


def _load():
    global _lib, _path
    if _lib is None:
        _path = library_path()
        lib = ctypes.CDLL(_path)
        ci, vp = ctypes.c_int, ctypes.c_void_p
        for name, scal in (("s", ctypes.c_float), ("d", ctypes.c_double)):
            f = getattr(lib, f"scipy_cblas_{name}gemm")
            f.restype = None
            f.argtypes = [ci, ci, ci, ci, ci, ci, scal, vp, ci, vp, ci, scal, vp, ci]
        for name in ("c", "z"):
            f = getattr(lib, f"scipy_cblas_{name}gemm")
            f.restype = None
            f.argtypes = [ci, ci, ci, ci, ci, ci, vp, vp, ci, vp, ci, vp, vp, ci]
        lib.scipy_openblas_set_num_threads.argtypes = [ci]
        lib.scipy_openblas_set_num_threads.restype = None
        lib.scipy_openblas_get_num_threads.restype = ci
        lib.scipy_openblas_get_config.restype = ctypes.c_char_p
        _lib = lib
    return _lib


def set_threads(n: int):
    _load().scipy_openblas_set_num_threads(int(n))


def get_threads() -> int:
    return int(_load().scipy_openblas_get_num_threads())


def config() -> str:
    return _load().scipy_openblas_get_config().decode()


def gemm(order, transa, transb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc,
         a_off=0, b_off=0, c_off=0):
    """In-place ``cblas_Xgemm`` on flat numpy buffers (C is modified)."""
    lib = _load()
    dt = np.dtype(A.dtype)
    pa = A.ctypes.data + a_off * dt.itemsize
    pb = B.ctypes.data + b_off * dt.itemsize
    pc = C.ctypes.data + c_off * dt.itemsize
    o, ta, tb = _ORDER[order], _TRANS[transa], _TRANS[transb]
    if dt == np.float32:
        lib.scipy_cblas_sgemm(o, ta, tb, M, N, K, float(alpha), pa, lda, pb, ldb, float(beta), pc, ldc)
    elif dt == np.float64:
        lib.scipy_cblas_dgemm(o, ta, tb, M, N, K, float(alpha), pa, lda, pb, ldb, float(beta), pc, ldc)
    elif dt == np.complex64:
        al = np.array([alpha], dtype=np.complex64)
        be = np.array([beta], dtype=np.complex64)
        lib.scipy_cblas_cgemm(o, ta, tb, M, N, K, al.ctypes.data, pa, lda, pb, ldb, be.ctypes.data, pc, ldc)
    elif dt == np.complex128:
        al = np.array([alpha], dtype=np.complex128)
        be = np.array([beta], dtype=np.complex128)
        lib.scipy_cblas_zgemm(o, ta, tb, M, N, K, al.ctypes.data, pa, lda, pb, ldb, be.ctypes.data, pc, ldc)
    else:
        raise TypeError(f"no CBLAS gemm for {dt}")
    return C
