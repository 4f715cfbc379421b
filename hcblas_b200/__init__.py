"""hcblas_b200 -- Python binding of the hcBLAS GEMM drop-in for B200.

This module is a ctypes mirror of the library's C ABI (include/hcblas.h):
the same function names, argument order, argument meaning and status codes
as hcBLAS's C API (lib/include/hcblas.h of the reference), over the in-tree
shared object ``hcblas_b200/libhcblas.so`` (sm_100a kernels + C++ host
library).  There is no fallback: if the shared object is missing the import
of :func:`lib` raises, and every GEMM runs on the GPU or fails with a status.

Device memory is managed with :func:`am_alloc` / :func:`am_free` (the
library's stand-ins for ``hc::am_alloc`` / ``hc::am_free``) and moved with
:func:`hcblasSetMatrix` / :func:`hcblasGetMatrix`, exactly like the
reference's tests do.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("HCBLAS_B200_LIB") or os.path.join(_HERE, "libhcblas.so")

# hcblasStatus_t (lib/include/hcblas.h:56-64 of the reference)
HCBLAS_STATUS_SUCCESS = 0
HCBLAS_STATUS_NOT_INITIALIZED = 1
HCBLAS_STATUS_ALLOC_FAILED = 2
HCBLAS_STATUS_INVALID_VALUE = 3
HCBLAS_STATUS_MAPPING_ERROR = 4
HCBLAS_STATUS_EXECUTION_FAILED = 5
HCBLAS_STATUS_INTERNAL_ERROR = 6

# hcblasOperation_t (lib/include/hcblas.h:74-78)
HCBLAS_OP_N, HCBLAS_OP_T, HCBLAS_OP_C = 0, 1, 2

# hcblasOrder (lib/include/hcblaslib.h:47)
RowMajor, ColMajor = 0, 1

# math modes (extension)
HCBLAS_MATH_NATIVE, HCBLAS_MATH_SPLIT_BF16, HCBLAS_MATH_OZAKI_INT8 = 0, 1, 2
HCBLAS_MATH_OZAKI_F16 = 3
HCBLAS_MATH_OZAKI_CRT = 4

# every C-ABI entry point include/hcblas.h declares (checked by the tests)
EXPORTED = (
    "hcblasCreate", "hcblasDestroy", "hcblasSetAcclView", "hcblasGetAcclView",
    "hcblasSetStream", "hcblasSetVector", "hcblasGetVector", "hcblasSetMatrix",
    "hcblasGetMatrix", "hcblasSetMatrixAsync", "hcblasGetMatrixAsync", "hcblasSgemm", "hcblasDgemm", "hcblasCgemm", "hcblasZgemm",
    "hcblasHgemm", "hcblasSgemmBatched", "hcblasCgemmBatched", "hcblasDgemmBatched",
    "hcblasZgemmBatched", "hcblasHgemmBatched", "hcblasSgemmStridedBatched",
    "hcblasDgemmStridedBatched", "hcblasCgemmStridedBatched", "hcblasZgemmStridedBatched",
    "hcblasHgemmStridedBatched", "hcblasLibSgemm", "hcblasLibDgemm", "hcblasLibHgemm",
    "hcblasLibCgemm", "hcblasLibZgemm", "hcblasLibGemmBatched",
    "hcblasSetMathMode", "hcblasGetMathMode",
    "hcblasGetLastPath", "hcblasGetVersionString", "hcblasGetKernelLaunchCount",
    "hcblasGetDeviceError", "hcblasSetTuningParam",
    "hcblasSetProfiling", "hcblasGetProfile", "hcblas_am_alloc", "hcblas_am_free",
    "hcblas_am_copy", "hcblas_view_wait", "hcblas_device_count", "hcblas_current_device",
    "hcblasHgemmGrouped", "hcblasSgemmGrouped", "hcblasSgemv", "hcblasDgemv", "hcblasSgemvBatched",
    "hcblasDgemvBatched", "hcblasSger", "hcblasDger", "hcblasSgerBatched", "hcblasDgerBatched",
    "hcblasSetAccuracyTarget", "hcblasGetAccuracyTarget", "hcblasPlanEmulation",
    "hcblasSgemmSplitBF16NoAlloc", "hcblasSgemmSplitBF16NoAllocStatus",
    "hcblasDgemmGrouped", "hcblasCgemmGrouped", "hcblasZgemmGrouped",
)

# accuracy targets (extension)
HCBLAS_ACCURACY_DEFAULT, HCBLAS_ACCURACY_NATIVE = 0, -1


class GemmProblem(ctypes.Structure):
    """One problem of hcblasHgemmGrouped / hcblasSgemmGrouped (hcblasGemmProblem)."""
    _fields_ = [("transa", ctypes.c_ushort), ("transb", ctypes.c_ushort),
                ("m", ctypes.c_int), ("n", ctypes.c_int), ("k", ctypes.c_int),
                ("A", ctypes.c_void_p), ("lda", ctypes.c_int),
                ("B", ctypes.c_void_p), ("ldb", ctypes.c_int),
                ("C", ctypes.c_void_p), ("ldc", ctypes.c_int)]


class AcclView(ctypes.Structure):
    """hcblas_accl_view_t: (device ordinal, cudaStream_t)."""
    _fields_ = [("device_id", ctypes.c_int), ("stream", ctypes.c_void_p)]


class Complex64(ctypes.Structure):
    _fields_ = [("x", ctypes.c_float), ("y", ctypes.c_float)]


class Complex128(ctypes.Structure):
    _fields_ = [("x", ctypes.c_double), ("y", ctypes.c_double)]


class Half(ctypes.Structure):
    _fields_ = [("bits", ctypes.c_uint16)]


_lib = None


def lib():
    """Load libhcblas.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m hcblas_b200.build` "
                "(there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        st = ctypes.c_ushort  # hcblasStatus_t: unsigned short
        vp, ci, cll = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong
        op = ctypes.c_ushort
        H = ctypes.POINTER(ctypes.c_void_p)
        L.hcblasCreate.argtypes = [H, ctypes.POINTER(AcclView)]
        L.hcblasCreate.restype = st
        L.hcblasDestroy.argtypes = [H]
        L.hcblasDestroy.restype = st
        L.hcblasSetAcclView.argtypes = [vp, ctypes.POINTER(AcclView), vp]
        L.hcblasSetAcclView.restype = st
        L.hcblasGetAcclView.argtypes = [vp, ctypes.POINTER(ctypes.POINTER(AcclView)),
                                        ctypes.POINTER(vp)]
        L.hcblasGetAcclView.restype = st
        L.hcblasSetStream.argtypes = [vp, vp]
        L.hcblasSetStream.restype = st
        for n in ("hcblasSetVector", "hcblasGetVector"):
            f = getattr(L, n)
            f.argtypes = [vp, ci, ci, vp, ci, vp, ci]
            f.restype = st
        for n in ("hcblasSetMatrix", "hcblasGetMatrix"):
            f = getattr(L, n)
            f.argtypes = [vp, ci, ci, ci, vp, ci, vp, ci]
            f.restype = st
        for n in ("hcblasSetMatrixAsync", "hcblasGetMatrixAsync"):
            f = getattr(L, n)
            f.argtypes = [vp, ci, ci, ci, vp, ci, vp, ci, vp]
            f.restype = st
        for p in "SDCZH":
            f = getattr(L, f"hcblas{p}gemm")
            f.argtypes = [vp, op, op, ci, ci, ci, vp, vp, ci, vp, ci, vp, vp, ci]
            f.restype = st
            f = getattr(L, f"hcblas{p}gemmBatched")
            f.argtypes = [vp, op, op, ci, ci, ci, vp, vp, ci, vp, ci, vp, vp, ci, ci]
            f.restype = st
            f = getattr(L, f"hcblas{p}gemmStridedBatched")
            f.argtypes = [vp, op, op, ci, ci, ci, vp, vp, ci, cll, vp, ci, cll, vp, vp, ci, cll, ci]
            f.restype = st
        i64, ch = ctypes.c_int64, ctypes.c_char
        for p in "SDH":
            f = getattr(L, f"hcblasLib{p}gemm")
            f.argtypes = [vp, ci, ch, ch, ci, ci, ci, vp, vp, i64, vp, i64, vp, vp, i64,
                          i64, i64, i64]
            f.restype = ci
        for p in "CZ":
            f = getattr(L, f"hcblasLib{p}gemm")
            f.argtypes = [vp, ci, ch, ch, ci, ci, ci, vp, vp, i64, i64, vp, i64, i64, vp, vp,
                          i64, i64]
            f.restype = ci
        L.hcblasLibGemmBatched.argtypes = [vp, ci, ci, ch, ch, ci, ci, ci, vp, vp, i64, i64, vp,
                                           i64, i64, vp, vp, i64, i64, i64, i64, i64, ci]
        L.hcblasLibGemmBatched.restype = ci
        L.hcblasSetMathMode.argtypes = [vp, ci, ci]
        L.hcblasSetMathMode.restype = st
        L.hcblasGetMathMode.argtypes = [vp, ctypes.POINTER(ci), ctypes.POINTER(ci)]
        L.hcblasGetMathMode.restype = st
        L.hcblasGetLastPath.argtypes = [vp]
        L.hcblasGetLastPath.restype = ctypes.c_char_p
        L.hcblasGetVersionString.argtypes = []
        L.hcblasGetVersionString.restype = ctypes.c_char_p
        L.hcblasGetKernelLaunchCount.argtypes = []
        L.hcblasGetKernelLaunchCount.restype = ctypes.c_longlong
        L.hcblasSetTuningParam.argtypes = [vp, ctypes.c_char_p, ci]
        L.hcblasSetTuningParam.restype = st
        L.hcblasGetDeviceError.argtypes = [vp]
        L.hcblasGetDeviceError.restype = ci
        L.hcblasSetProfiling.argtypes = [vp, ci]
        L.hcblasSetProfiling.restype = st
        L.hcblasGetProfile.argtypes = [vp, ctypes.c_char_p, ci]
        L.hcblasGetProfile.restype = ci
        L.hcblas_am_alloc.argtypes = [ctypes.c_size_t, ci, ctypes.c_uint]
        L.hcblas_am_alloc.restype = vp
        L.hcblas_am_free.argtypes = [vp]
        L.hcblas_am_free.restype = ci
        L.hcblas_am_copy.argtypes = [AcclView, vp, vp, ctypes.c_size_t]
        L.hcblas_am_copy.restype = ci
        L.hcblas_view_wait.argtypes = [AcclView]
        L.hcblas_view_wait.restype = ci
        L.hcblas_device_count.argtypes = []
        L.hcblas_device_count.restype = ci
        L.hcblas_current_device.argtypes = []
        L.hcblas_current_device.restype = ci
        L.hcblasHgemmGrouped.argtypes = [vp, ci, vp, vp, vp]
        L.hcblasHgemmGrouped.restype = st
        L.hcblasSgemmGrouped.argtypes = [vp, ci, vp, vp, vp]
        L.hcblasSgemmGrouped.restype = st
        for p in "SD":
            f = getattr(L, f"hcblas{p}gemv")
            f.argtypes = [vp, op, ci, ci, vp, vp, ci, vp, ci, vp, vp, ci]
            f.restype = st
            f = getattr(L, f"hcblas{p}gemvBatched")
            f.argtypes = [vp, op, ci, ci, vp, vp, ci, vp, ci, vp, vp, ci, ci]
            f.restype = st
            f = getattr(L, f"hcblas{p}ger")
            f.argtypes = [vp, ci, ci, vp, vp, ci, vp, ci, vp, ci]
            f.restype = st
            f = getattr(L, f"hcblas{p}gerBatched")
            f.argtypes = [vp, ci, ci, vp, vp, ci, vp, ci, vp, ci, ci]
            f.restype = st
        _lib = L
    return _lib


# ------------------------------------------------------------------ handle --


def peak_probe(kind, iters=0):
    """TFLOP/s of one arithmetic pipe measured by the library's issue-rate
    probe: kind 0 = FP32 FMA (f32x2), 1 = FP64 FMA, 2 = FP64 mma.sync
    m16n8k4 (the pipes the native SGEMM, the FP64 SIMT kernel and the DMMA
    DGEMM run on); iters per chain, 0 for the default.  None on failure."""
    L = lib()
    f = L.hcbk_peak_probe
    f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    f.restype = ctypes.c_int
    out = ctypes.c_double(0.0)
    return out.value if f(int(kind), int(iters), ctypes.byref(out)) == 0 else None

def hcblasCreate(device: int = 0, stream: int | None = None):
    """Returns ``(status, handle)``; the handle is a raw pointer (int)."""
    h = ctypes.c_void_p()
    view = AcclView(device, stream)
    s = lib().hcblasCreate(ctypes.byref(h), ctypes.byref(view))
    return s, h.value


def hcblasDestroy(handle):
    h = ctypes.c_void_p(handle)
    return lib().hcblasDestroy(ctypes.byref(h))


def hcblasSetStream(handle, stream):
    return lib().hcblasSetStream(handle, stream)


def hcblasSetMathMode(handle, mode, param=0):
    return lib().hcblasSetMathMode(handle, mode, param)


def hcblasGetLastPath(handle) -> str:
    return lib().hcblasGetLastPath(handle).decode()


def hcblasSetAccuracyTarget(handle, bits: int) -> int:
    f = lib().hcblasSetAccuracyTarget
    f.argtypes = [ctypes.c_void_p, ctypes.c_int]
    f.restype = ctypes.c_ushort
    return f(handle, bits)


def plan_emulation(mode: int, param: int, bits: int, dtype: str, k: int):
    """(status, count, model_bits) of hcblasPlanEmulation; dtype 's', 'd',
    'c' or 'z'."""
    f = lib().hcblasPlanEmulation
    f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_longlong,
                  ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)]
    f.restype = ctypes.c_ushort
    c, mb = ctypes.c_int(0), ctypes.c_double(0.0)
    s = f(mode, param, bits, "sdcz".index(dtype), k, ctypes.byref(c), ctypes.byref(mb))
    return s, c.value, mb.value


def set_tuning(handle, name: str, value: int):
    return lib().hcblasSetTuningParam(handle, name.encode(), int(value))


def device_error(handle) -> int:
    """Sync the handle's stream; return and clear a tensor-core timeout code."""
    return int(lib().hcblasGetDeviceError(handle))


def kernel_launch_count() -> int:
    return int(lib().hcblasGetKernelLaunchCount())


def set_profiling(handle, on: bool):
    return lib().hcblasSetProfiling(handle, 1 if on else 0)


def get_profile(handle) -> dict:
    """{kernel name: (launches, total_ms)} from the handle's event records."""
    n = lib().hcblasGetProfile(handle, None, 0)
    buf = ctypes.create_string_buffer(max(n + 1, 1))
    lib().hcblasGetProfile(handle, buf, len(buf))
    out = {}
    for line in buf.value.decode().splitlines():
        name, cnt, ms = line.split()
        out[name] = (int(cnt), float(ms))
    return out


# ------------------------------------------------------------------ memory --

def am_alloc(nbytes: int, device: int = 0) -> int:
    p = lib().hcblas_am_alloc(nbytes, device, 0)
    if not p:
        raise MemoryError(f"hcblas_am_alloc({nbytes}) failed")
    return p


def am_free(ptr: int):
    return lib().hcblas_am_free(ptr)


def hcblasSetMatrix(handle, rows, cols, elem_size, host_ptr, lda, dev_ptr, ldb):
    return lib().hcblasSetMatrix(handle, rows, cols, elem_size, host_ptr, lda, dev_ptr, ldb)


def hcblasGetMatrix(handle, rows, cols, elem_size, dev_ptr, lda, host_ptr, ldb):
    return lib().hcblasGetMatrix(handle, rows, cols, elem_size, dev_ptr, lda, host_ptr, ldb)


def hcblasSetMatrixAsync(handle, rows, cols, elem_size, host_ptr, lda, dev_ptr, ldb, stream):
    """hcblasSetMatrix enqueued on `stream` (a cudaStream_t as int; 0 = the
    handle's stream) without waiting; host memory should be pinned."""
    return lib().hcblasSetMatrixAsync(handle, rows, cols, elem_size, host_ptr, lda, dev_ptr, ldb,
                                      stream)


def hcblasGetMatrixAsync(handle, rows, cols, elem_size, dev_ptr, lda, host_ptr, ldb, stream):
    """hcblasGetMatrix enqueued on `stream` without waiting."""
    return lib().hcblasGetMatrixAsync(handle, rows, cols, elem_size, dev_ptr, lda, host_ptr, ldb,
                                      stream)


class DeviceArray:
    """A device copy of a flat numpy array (allocated with am_alloc)."""

    def __init__(self, handle, host: np.ndarray | None = None, *, nbytes: int = 0,
                 dtype=None, device: int = 0):
        self.handle = handle
        if host is not None:
            host = np.ascontiguousarray(host)
            self.dtype, self.size = host.dtype, host.size
            nbytes = host.nbytes
        else:
            self.dtype = np.dtype(dtype)
            self.size = nbytes // self.dtype.itemsize
        self.nbytes = nbytes
        self.ptr = am_alloc(max(nbytes, 1), device)
        if host is not None:
            self.upload(host)

    _CHUNK = 1 << 30  # bytes per hcblasSetMatrix / hcblasGetMatrix call (int sizes)

    def upload(self, host: np.ndarray):
        host = np.ascontiguousarray(host)
        assert host.nbytes == self.nbytes
        for off in range(0, host.nbytes, self._CHUNK):
            nb = min(self._CHUNK, host.nbytes - off)
            s = hcblasSetMatrix(self.handle, nb, 1, 1, host.ctypes.data + off, nb,
                                self.ptr + off, nb)
            if s != HCBLAS_STATUS_SUCCESS:
                raise RuntimeError(f"hcblasSetMatrix failed: {s}")

    def download(self) -> np.ndarray:
        out = np.empty(self.size, dtype=self.dtype)
        for off in range(0, self.nbytes, self._CHUNK):
            nb = min(self._CHUNK, self.nbytes - off)
            s = hcblasGetMatrix(self.handle, nb, 1, 1, self.ptr + off, nb, out.ctypes.data + off,
                                nb)
            if s != HCBLAS_STATUS_SUCCESS:
                raise RuntimeError(f"hcblasGetMatrix failed: {s}")
        return out

    def free(self):
        if self.ptr:
            am_free(self.ptr)
            self.ptr = 0

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


# -------------------------------------------------------------------- GEMM --

_PREFIX = {np.dtype(np.float32): "S", np.dtype(np.float64): "D",
           np.dtype(np.complex64): "C", np.dtype(np.complex128): "Z",
           np.dtype(np.float16): "H"}


def scalar_bytes(dtype, value):
    """Host scalar buffer holding alpha/beta in the storage type."""
    dt = np.dtype(dtype)
    return np.array([value], dtype=dt)


def gemm(handle, transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc):
    """hcblas{S,D,C,Z,H}gemm on device pointers; the prefix follows ``A.dtype``.

    ``A``, ``B``, ``C`` are :class:`DeviceArray` objects.
    """
    p = _PREFIX[np.dtype(A.dtype)]
    al = scalar_bytes(A.dtype, alpha)
    be = scalar_bytes(A.dtype, beta)
    f = getattr(lib(), f"hcblas{p}gemm")
    return f(handle, transa, transb, m, n, k, al.ctypes.data, A.ptr, lda, B.ptr, ldb,
             be.ctypes.data, C.ptr, ldc)


def lib_gemm(handle, order, type_a, type_b, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc,
             a_off=0, b_off=0, c_off=0):
    """Hcblaslibrary::hcblas_Xgemm through its C shim (hcblasLib{S,D,H,C,Z}gemm).

    ``type_a``/``type_b`` are 'n', 't' or 'c'; ``order`` RowMajor/ColMajor;
    ``A``, ``B``, ``C`` are :class:`DeviceArray`.  Returns 0 (HCBLAS_SUCCEEDS)
    or -1 (HCBLAS_INVALID).
    """
    dt = np.dtype(A.dtype)
    p = _PREFIX[dt]
    al = scalar_bytes(dt, alpha)
    be = scalar_bytes(dt, beta)
    f = getattr(lib(), f"hcblasLib{p}gemm")
    ta, tb = type_a.encode(), type_b.encode()
    if p in "CZ":
        return f(handle, order, ta, tb, M, N, K, al.ctypes.data, A.ptr, a_off, lda, B.ptr,
                 b_off, ldb, be.ctypes.data, C.ptr, c_off, ldc)
    return f(handle, order, ta, tb, M, N, K, al.ctypes.data, A.ptr, lda, B.ptr, ldb,
             be.ctypes.data, C.ptr, ldc, a_off, b_off, c_off)


def gemm_strided_batched(handle, transa, transb, m, n, k, alpha, A, lda, sA, B, ldb, sB,
                         beta, C, ldc, sC, batch):
    p = _PREFIX[np.dtype(A.dtype)]
    al = scalar_bytes(A.dtype, alpha)
    be = scalar_bytes(A.dtype, beta)
    f = getattr(lib(), f"hcblas{p}gemmStridedBatched")
    return f(handle, transa, transb, m, n, k, al.ctypes.data, A.ptr, lda, sA, B.ptr, ldb, sB,
             be.ctypes.data, C.ptr, ldc, sC, batch)


def gemm_batched(handle, transa, transb, m, n, k, alpha, Aarr_dev, lda, Barr_dev, ldb, beta,
                 Carr_dev, ldc, batch, dtype):
    """hcblas{S,D,C,Z,H}gemmBatched with device-resident pointer arrays."""
    p = _PREFIX[np.dtype(dtype)]
    al = scalar_bytes(dtype, alpha)
    be = scalar_bytes(dtype, beta)
    f = getattr(lib(), f"hcblas{p}gemmBatched")
    return f(handle, transa, transb, m, n, k, al.ctypes.data, Aarr_dev, lda, Barr_dev, ldb,
             be.ctypes.data, Carr_dev, ldc, batch)


def hgemm_grouped(handle, problems, alpha: float, beta: float) -> int:
    """hcblasHgemmGrouped over a list of GemmProblem (device pointers inside)."""
    arr = (GemmProblem * len(problems))(*problems)
    a = np.array([alpha], dtype=np.float16).view(np.uint16)
    b = np.array([beta], dtype=np.float16).view(np.uint16)
    return lib().hcblasHgemmGrouped(handle, len(problems), ctypes.cast(arr, ctypes.c_void_p),
                                    a.ctypes.data, b.ctypes.data)


def sgemm_grouped(handle, problems, alpha: float, beta: float) -> int:
    """hcblasSgemmGrouped (f32 problems on the split-BF16 tensor-core path)."""
    arr = (GemmProblem * len(problems))(*problems)
    a = np.array([alpha], dtype=np.float32)
    b = np.array([beta], dtype=np.float32)
    return lib().hcblasSgemmGrouped(handle, len(problems), ctypes.cast(arr, ctypes.c_void_p),
                                    a.ctypes.data, b.ctypes.data)


def gemv(handle, trans, m, n, alpha, A, lda, x, incx, beta, y, incy, batch=None):
    """hcblas{S,D}gemv[Batched] on DeviceArrays; the prefix follows ``A.dtype``."""
    p = _PREFIX[np.dtype(A.dtype)]
    al, be = scalar_bytes(A.dtype, alpha), scalar_bytes(A.dtype, beta)
    if batch is None:
        return getattr(lib(), f"hcblas{p}gemv")(handle, trans, m, n, al.ctypes.data, A.ptr, lda,
                                                 x.ptr, incx, be.ctypes.data, y.ptr, incy)
    return getattr(lib(), f"hcblas{p}gemvBatched")(handle, trans, m, n, al.ctypes.data, A.ptr,
                                                    lda, x.ptr, incx, be.ctypes.data, y.ptr, incy,
                                                    batch)


def ger(handle, m, n, alpha, x, incx, y, incy, A, lda, batch=None):
    """hcblas{S,D}ger[Batched] on DeviceArrays; the prefix follows ``A.dtype``."""
    p = _PREFIX[np.dtype(A.dtype)]
    al = scalar_bytes(A.dtype, alpha)
    if batch is None:
        return getattr(lib(), f"hcblas{p}ger")(handle, m, n, al.ctypes.data, x.ptr, incx, y.ptr,
                                                incy, A.ptr, lda)
    return getattr(lib(), f"hcblas{p}gerBatched")(handle, m, n, al.ctypes.data, x.ptr, incx,
                                                   y.ptr, incy, A.ptr, lda, batch)
