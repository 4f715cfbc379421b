"""ctypes front-end of the CPU GEMM oracle (test infrastructure only).

Imported only by tests/, ``__graft_entry__.smoke()`` and bench.py's CPU
baseline leg, always as the checker.  The product library never calls it.

The oracle restates CBLAS xGEMM (the host path hcBLAS's unit tests compare
against, test/unit/hcblas_sgemm.cpp:252 ``cblas_sgemm(...)``) with binary64
accumulation for S/C/H and double-double accumulation for D/Z; see
gemm_oracle.c for the full statement.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")

S, D, C, Z, H = 0, 1, 2, 3, 4
ROW, COL = 0, 1  # hcblasOrder: RowMajor = 0, ColMajor = 1
OP_N, OP_T, OP_C = 0, 1, 2

_DTYPE_CODE = {
    np.dtype(np.float32): S,
    np.dtype(np.float64): D,
    np.dtype(np.complex64): C,
    np.dtype(np.complex128): Z,
    np.dtype(np.float16): H,
}

_lib = None


def build() -> str:
    """Compile the oracle with its Makefile (gcc, no GPU needed)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(
            os.path.join(_HERE, "gemm_oracle.c")
        ):
            build()
        lib = ctypes.CDLL(_LIB_PATH)
        i64 = ctypes.c_int64
        vp = ctypes.c_void_p
        lib.oracle_gemm.restype = ctypes.c_int
        lib.oracle_gemm.argtypes = [
            ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
            i64, i64, i64, vp, vp, i64, i64, vp, i64, i64, vp, vp, i64, i64,
            vp, ctypes.c_int,
        ]
        lib.oracle_half_to_double.restype = ctypes.c_double
        lib.oracle_half_to_double.argtypes = [ctypes.c_uint16]
        lib.oracle_double_to_half.restype = ctypes.c_uint16
        lib.oracle_double_to_half.argtypes = [ctypes.c_double]
        lib.oracle_rand_r_u02.restype = None
        lib.oracle_rand_r_u02.argtypes = [ctypes.POINTER(ctypes.c_uint), i64, vp]
        lib.oracle_rand_r_mod.restype = None
        lib.oracle_rand_r_mod.argtypes = [ctypes.POINTER(ctypes.c_uint), i64, ctypes.c_int, vp]
        _lib = lib
    return _lib


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def gemm(order, transa, transb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc,
         a_off=0, b_off=0, c_off=0, nthreads=0, want_ref=True):
    """C := alpha*op(A)*op(B) + beta*C on flat numpy buffers (CBLAS semantics).

    Returns ``(C_out, ref)``: ``C_out`` is a new flat array of C's dtype holding
    the updated C (rounded to the storage type), ``ref`` the high-precision
    result as a dense column-major M x N float64/complex128 array (or None).
    """
    lib = _load()
    A = np.ascontiguousarray(A).reshape(-1)
    B = np.ascontiguousarray(B).reshape(-1)
    C_out = np.array(C, copy=True).reshape(-1)
    code = _DTYPE_CODE[A.dtype]
    assert B.dtype == A.dtype and C_out.dtype == A.dtype
    al = np.array([complex(alpha).real, complex(alpha).imag], dtype=np.float64)
    be = np.array([complex(beta).real, complex(beta).imag], dtype=np.float64)
    ref = None
    if want_ref:
        if code in (2, 3):  # complex types
            ref = np.zeros((N, M), dtype=np.complex128)
        else:
            ref = np.zeros((N, M), dtype=np.float64)
    rc = lib.oracle_gemm(code, order, transa, transb, M, N, K, _ptr(al), _ptr(A), a_off, lda,
                         _ptr(B), b_off, ldb, _ptr(be), _ptr(C_out), c_off, ldc,
                         _ptr(ref) if ref is not None else None, nthreads)
    if rc != 0:
        raise ValueError("oracle_gemm rejected its arguments")
    if ref is not None:
        ref = ref.T  # (M, N) view of the column-major result
    return C_out, ref


def view_c(C_flat, order, M, N, ldc, c_off=0):
    """(M, N) logical view of a flat C buffer in the given storage order."""
    C_flat = np.asarray(C_flat).reshape(-1)
    if order == COL:
        return np.lib.stride_tricks.as_strided(
            C_flat[c_off:], shape=(M, N),
            strides=(C_flat.itemsize, C_flat.itemsize * ldc))
    return np.lib.stride_tricks.as_strided(
        C_flat[c_off:], shape=(M, N), strides=(C_flat.itemsize * ldc, C_flat.itemsize))


def normwise_rel_error(C_test, ref):
    """||C_test - ref||_F / ||ref||_F in binary64 (complex-aware)."""
    ct = np.asarray(C_test).astype(np.complex128 if np.iscomplexobj(ref) else np.float64)
    num = np.linalg.norm((ct - ref).reshape(-1))
    den = np.linalg.norm(np.asarray(ref).reshape(-1))
    return float(num / den) if den > 0 else float(num)


def compare_l2fe(reference, data):
    """hcBLAS's sgemmCompareL2fe (test/include/helper_functions.h:10-53)."""
    ref = np.asarray(reference, dtype=np.float64).reshape(-1)
    dat = np.asarray(data, dtype=np.float64).reshape(-1)
    nrm = float(np.dot(ref, ref))
    if abs(nrm) < 1e-7:
        return -1.0
    return float(np.sqrt(np.dot(ref - dat, ref - dat)) / np.sqrt(nrm))


def half_to_double(bits: int) -> float:
    return _load().oracle_half_to_double(bits)


def double_to_half(x: float) -> int:
    return _load().oracle_double_to_half(x)


# glibc's rand_r / srand+rand, used by the reference tests' input recipes
# (test/unit/hcblas_sgemm.cpp:32 global_seed = 100; test/unit/test_constants.h).
_libc = None


def _c():
    global _libc
    if _libc is None:
        _libc = ctypes.CDLL("libc.so.6")
        _libc.rand_r.restype = ctypes.c_int
        _libc.rand_r.argtypes = [ctypes.POINTER(ctypes.c_uint)]
        _libc.rand.restype = ctypes.c_int
        _libc.srand.argtypes = [ctypes.c_uint]
    return _libc


class RandR:
    """Stateful glibc rand_r stream, as the reference tests draw it."""

    RAND_MAX = 2147483647

    def __init__(self, seed: int):
        self.state = ctypes.c_uint(seed)

    def next(self) -> int:
        return _c().rand_r(ctypes.byref(self.state))

    def ints(self, n: int, mod: int) -> np.ndarray:
        out = np.empty(n, dtype=np.float64)
        _load().oracle_rand_r_mod(ctypes.byref(self.state), n, mod, out.ctypes.data)
        return out.astype(np.int64)

    def uniform02(self, n: int) -> np.ndarray:
        # static_cast<float>(rand_r(&seed)) / static_cast<float>(RAND_MAX / X), X = 2
        # (test/unit/hcblas_sgemm.cpp:222-243): computed in binary32.
        out = np.empty(n, dtype=np.float32)
        _load().oracle_rand_r_u02(ctypes.byref(self.state), n, out.ctypes.data)
        return out


def srand_rand(seed: int) -> int:
    """srand(seed); rand() -- the reference's shape-class generators."""
    c = _c()
    c.srand(seed)
    return c.rand()
