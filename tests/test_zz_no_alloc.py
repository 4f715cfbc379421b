"""hcblasSgemmSplitBF16NoAlloc: the split-BF16 SGEMM entry point that
allocates nothing (its scratch is a static device array of the library).

Collected last on purpose: it must give the same answers whether it runs in a
fresh process (its first call then performs the per-device set-up) or after
every other GPU test has used the handle-based paths.  Two calls in a row,
with different inputs, shapes and transposes, are each checked against the
handle-based entry point (hcblasSgemm under HCBLAS_MATH_SPLIT_BF16 with the
same number of terms) and against the CPU oracle, with the tolerance of the
split-BF16 tests:
  * 6 products: 2 gamma_{K+2}(f32) || |alpha||A||B| + |beta||C| ||_F
  * 3 products: (2^-15 + 2 gamma_{K+2}(f32)) || |alpha||A||B| ||_F
                + 2 gamma_{K+2}(f32) || |beta||C| ||_F
The second call also shows that the reused scratch carries nothing over.
After each call hcblasSgemmSplitBF16NoAllocStatus must report no pipeline
timeout.  The fresh-process case runs in a child interpreter whose first GEMM
call is the no-allocation entry point.
"""
import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest

import hcblas_b200 as hb
from oracle import oracle as O

pytestmark = pytest.mark.gpu

U32 = 2.0 ** -24
OPS = {0: hb.HCBLAS_OP_N, 1: hb.HCBLAS_OP_T}


def g32(K):
    return (K + 2) * U32 / (1 - (K + 2) * U32)


def op_dense(X, trans, rows, cols, ld):
    """op(X) as a dense (rows x cols) float64 array, X column-major."""
    if trans == 0:
        return X[: ld * cols].reshape(cols, ld)[:, :rows].T.astype(np.float64)
    return X[: ld * rows].reshape(rows, ld)[:, :cols].astype(np.float64)


def entry():
    f = hb.lib().hcblasSgemmSplitBF16NoAlloc
    vp, ci, op = ctypes.c_void_p, ctypes.c_int, ctypes.c_ushort
    f.argtypes = [vp, op, op, ci, ci, ci, vp, vp, ci, vp, ci, vp, vp, ci, ci]
    f.restype = ctypes.c_ushort
    return f


def status():
    f = hb.lib().hcblasSgemmSplitBF16NoAllocStatus
    f.argtypes = [ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f(None)


def bound_of(terms, K, alpha, beta, Ad, Bd, Cd):
    ab = abs(alpha) * (np.abs(Ad) @ np.abs(Bd))
    cc = abs(beta) * np.abs(Cd)
    if terms == 6:
        return 2 * g32(K) * np.linalg.norm(ab + cc)
    return (2.0 ** -15 + 2 * g32(K)) * np.linalg.norm(ab) + 2 * g32(K) * np.linalg.norm(cc)


def make(rng, ta, tb, M, N, K):
    lda = (M if ta == 0 else K) + 3
    ldb = (K if tb == 0 else N) + 5
    ldc = M + 2
    A = rng.standard_normal(lda * (K if ta == 0 else M)).astype(np.float32)
    B = rng.standard_normal(ldb * (N if tb == 0 else K)).astype(np.float32)
    C = rng.standard_normal(ldc * N).astype(np.float32)
    return A, lda, B, ldb, C, ldc


@pytest.mark.parametrize("terms", [3, 6])
def test_no_alloc_matches_handle_path(handle, terms):
    f = entry()
    rng = np.random.default_rng(2024 + terms)
    calls = [(1, 0, 300, 200, 700, 1.25, -0.5), (0, 1, 256, 384, 1000, 0.75, 2.0)]
    for ta, tb, M, N, K, alpha, beta in calls:  # two calls in a row
        A, lda, B, ldb, C, ldc = make(rng, ta, tb, M, N, K)
        al = np.array([alpha], np.float32)
        be = np.array([beta], np.float32)
        dA, dB = hb.DeviceArray(handle, A), hb.DeviceArray(handle, B)
        dC_new, dC_old = hb.DeviceArray(handle, C), hb.DeviceArray(handle, C)

        st = f(None, OPS[ta], OPS[tb], M, N, K, al.ctypes.data, dA.ptr, lda, dB.ptr, ldb,
               be.ctypes.data, dC_new.ptr, ldc, terms)
        assert st == hb.HCBLAS_STATUS_SUCCESS, st
        assert status() == 0
        got_new = dC_new.download()

        assert hb.hcblasSetMathMode(handle, hb.HCBLAS_MATH_SPLIT_BF16, terms) == 0
        try:
            st = hb.lib().hcblasSgemm(handle, OPS[ta], OPS[tb], M, N, K, al.ctypes.data,
                                      dA.ptr, lda, dB.ptr, ldb, be.ctypes.data, dC_old.ptr, ldc)
            assert st == hb.HCBLAS_STATUS_SUCCESS, st
            assert hb.hcblasGetLastPath(handle).startswith(f"tc.split_bf16x{terms}")
            assert hb.device_error(handle) == 0
        finally:
            hb.hcblasSetMathMode(handle, hb.HCBLAS_MATH_NATIVE, 0)
        got_old = dC_old.download()

        Ad, Bd = op_dense(A, ta, M, K, lda), op_dense(B, tb, K, N, ldb)
        Cd = C[: ldc * N].reshape(N, ldc)[:, :M].T.astype(np.float64)
        bound = bound_of(terms, K, alpha, beta, Ad, Bd, Cd)
        view = lambda X: X[: ldc * N].reshape(N, ldc)[:, :M].T.astype(np.float64)
        _, ref = O.gemm(O.COL, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc)
        assert np.linalg.norm(view(got_new) - view(got_old)) <= bound
        assert np.linalg.norm(view(got_new) - ref) <= bound
        # padding between columns of C is untouched
        pad_new = got_new[: ldc * N].reshape(N, ldc)[:, M:]
        assert np.array_equal(pad_new, C[: ldc * N].reshape(N, ldc)[:, M:])


def test_no_alloc_rejects_oversize_and_bad_args(handle):
    f = entry()
    one = np.array([1.0], np.float32)
    fake = ctypes.c_void_p(16)  # never dereferenced: rejected before any launch
    # 4096 x 4096 x 4096 at 3 terms needs 2 * (32 + 32) MiB > 64 MiB
    assert f(None, 0, 0, 4096, 4096, 4096, one.ctypes.data, fake, 4096, fake, 4096,
             one.ctypes.data, fake, 4096, 3) == hb.HCBLAS_STATUS_INVALID_VALUE
    assert f(None, 0, 0, 8, 8, 8, one.ctypes.data, fake, 8, fake, 8, one.ctypes.data, fake, 8,
             4) == hb.HCBLAS_STATUS_INVALID_VALUE
    assert f(None, 0, 0, -1, 8, 8, one.ctypes.data, fake, 8, fake, 8, one.ctypes.data, fake, 8,
             3) == hb.HCBLAS_STATUS_INVALID_VALUE
    assert f(None, 0, 0, 0, 8, 8, one.ctypes.data, fake, 8, fake, 8, one.ctypes.data, fake, 8,
             3) == hb.HCBLAS_STATUS_EXECUTION_FAILED
    # the largest sizes: each operand's planes alone exceed the scratch, and
    # their byte counts summed over the planes would wrap a 64-bit size
    big = 2 ** 31 - 1
    for terms in (3, 6):
        assert f(None, 0, 0, big, big, big, one.ctypes.data, fake, big, fake, big,
                 one.ctypes.data, fake, big, terms) == hb.HCBLAS_STATUS_INVALID_VALUE


def _fresh_process_case():
    """Body of the child process: the no-allocation entry point is the
    first GEMM this process calls, so its first call performs the per-device
    set-up; two calls in a row, each checked against the oracle."""
    s, h = hb.hcblasCreate(0)
    assert s == hb.HCBLAS_STATUS_SUCCESS
    f = entry()
    rng = np.random.default_rng(77)
    try:
        for ta, tb, M, N, K, alpha, beta, terms in [(0, 1, 200, 130, 300, 1.0, 0.5, 6),
                                                    (1, 0, 96, 257, 520, -0.5, 0.0, 3)]:
            A, lda, B, ldb, C, ldc = make(rng, ta, tb, M, N, K)
            al, be = np.array([alpha], np.float32), np.array([beta], np.float32)
            dA, dB, dC = hb.DeviceArray(h, A), hb.DeviceArray(h, B), hb.DeviceArray(h, C)
            st = f(None, OPS[ta], OPS[tb], M, N, K, al.ctypes.data, dA.ptr, lda, dB.ptr, ldb,
                   be.ctypes.data, dC.ptr, ldc, terms)
            assert st == hb.HCBLAS_STATUS_SUCCESS, st
            assert status() == 0
            got = dC.download()
            Ad, Bd = op_dense(A, ta, M, K, lda), op_dense(B, tb, K, N, ldb)
            Cd = C[: ldc * N].reshape(N, ldc)[:, :M].T.astype(np.float64)
            _, ref = O.gemm(O.COL, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc)
            view = got[: ldc * N].reshape(N, ldc)[:, :M].T.astype(np.float64)
            err = np.linalg.norm(view - ref)
            assert err <= bound_of(terms, K, alpha, beta, Ad, Bd, Cd), err
    finally:
        hb.hcblasDestroy(h)
    print("fresh-process no-allocation calls ok")


def test_no_alloc_in_fresh_process():
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c",
                        "import tests.test_zz_no_alloc as t; t._fresh_process_case()"],
                       cwd=root, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "fresh-process no-allocation calls ok" in r.stdout
