"""Grouped GEMM for FP64, complex FP32 and complex FP64 problems
(hcblasDgemmGrouped / hcblasCgemmGrouped / hcblasZgemmGrouped): uneven
problems with mixed (conjugate) transposes and arbitrary leading dimensions in
one persistent CUDA-core launch, each checked against the CPU oracle
(double-double for D/Z) with the plain-arithmetic bound
    ||C_gpu - C_ref||_F <= 2 gamma_{K+2}(u) || |alpha||A||B| + |beta||C| ||_F.
Also: alpha == 0, the reuse of the uploaded table by an identical follow-up
call, and the status rules of the grouped entry points.
"""
import ctypes

import numpy as np
import pytest

import hcblas_b200 as hb
from oracle import oracle as O

pytestmark = pytest.mark.gpu

U = {"d": 2.0 ** -53, "c": 2.0 ** -24, "z": 2.0 ** -53}
DT = {"d": np.float64, "c": np.complex64, "z": np.complex128}


def gam(K, u):
    return (K + 2) * u / (1 - (K + 2) * u)


def op_dense(X, trans, rows, cols, ld):
    if trans == 0:
        return X[: ld * cols].reshape(cols, ld)[:, :rows].T
    Y = X[: ld * rows].reshape(rows, ld)[:, :cols]
    return np.conj(Y) if trans == 2 else Y


def rand(rng, dt, n):
    v = rng.uniform(-1, 1, n)
    if np.issubdtype(dt, np.complexfloating):
        v = v + 1j * rng.uniform(-1, 1, n)
    return v.astype(dt)


def make(handle, rng, kind, count, lo=8, hi=300):
    dt = DT[kind]
    ops = (0, 1) if kind == "d" else (0, 1, 2)
    probs, host, dev = [], [], []
    for _ in range(count):
        ta, tb = int(rng.choice(ops)), int(rng.choice(ops))
        M, N, K = (int(np.exp(rng.uniform(np.log(lo), np.log(hi + 1)))) for _ in range(3))
        lda = (M if ta == 0 else K) + int(rng.integers(0, 5))
        ldb = (K if tb == 0 else N) + int(rng.integers(0, 5))
        ldc = M + int(rng.integers(0, 3))
        A = rand(rng, dt, lda * (K if ta == 0 else M))
        B = rand(rng, dt, ldb * (N if tb == 0 else K))
        C = rand(rng, dt, ldc * N)
        dA, dB, dC = (hb.DeviceArray(handle, X) for X in (A, B, C))
        probs.append(hb.GemmProblem(ta, tb, M, N, K, dA.ptr, lda, dB.ptr, ldb, dC.ptr, ldc))
        host.append((ta, tb, M, N, K, A, lda, B, ldb, C, ldc))
        dev.append((dA, dB, dC))
    return (hb.GemmProblem * count)(*probs), host, dev


def call(handle, kind, arr, alpha, beta):
    f = {"d": hb.lib().hcblasDgemmGrouped, "c": hb.lib().hcblasCgemmGrouped,
         "z": hb.lib().hcblasZgemmGrouped}[kind]
    if kind == "d":
        al, be = np.array([alpha], np.float64), np.array([beta], np.float64)
    else:
        ct = np.float32 if kind == "c" else np.float64
        al = np.array([complex(alpha).real, complex(alpha).imag], ct)
        be = np.array([complex(beta).real, complex(beta).imag], ct)
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_void_p]
    f.restype = ctypes.c_ushort
    n = len(arr) if arr is not None else 0
    return f(handle, n, ctypes.cast(arr, ctypes.c_void_p) if arr is not None else None,
             al.ctypes.data, be.ctypes.data)


def check(kind, host, dev, alpha, beta):
    for (ta, tb, M, N, K, A, lda, B, ldb, C, ldc), (_, _, dC) in zip(host, dev):
        got = dC.download()
        _, ref = O.gemm(O.COL, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc)
        gv = O.view_c(got, O.COL, M, N, ldc)
        Ad, Bd = op_dense(A, ta, M, K, lda), op_dense(B, tb, K, N, ldb)
        cc = abs(beta) * np.abs(O.view_c(C, O.COL, M, N, ldc))
        bound = 2 * gam(K, U[kind]) * np.linalg.norm(abs(alpha) * (np.abs(Ad) @ np.abs(Bd)) + cc)
        err = np.linalg.norm(gv - ref)
        assert err <= bound, (kind, ta, tb, M, N, K, err, bound)
        # the leading-dimension padding of C is untouched
        assert np.array_equal(got[: ldc * N].reshape(N, ldc)[:, M:],
                              C[: ldc * N].reshape(N, ldc)[:, M:])


@pytest.mark.parametrize("kind", ["d", "c", "z"])
def test_grouped_dcz_uneven(handle, kind):
    rng = np.random.default_rng({"d": 11, "c": 12, "z": 13}[kind])
    arr, host, dev = make(handle, rng, kind, 40)
    alpha, beta = (1.5, -0.5) if kind == "d" else ((1 + 0.5j), (0.5 - 0.25j))
    launches0 = hb.kernel_launch_count()
    assert call(handle, kind, arr, alpha, beta) == 0
    assert hb.device_error(handle) == 0
    assert hb.kernel_launch_count() - launches0 == 1  # one persistent launch
    assert hb.hcblasGetLastPath(handle) == f"simt.{kind}.grouped"
    check(kind, host, dev, alpha, beta)
    # an identical follow-up call reuses the table: same results from the same inputs
    for (_, _, _, _, _, _, _, _, _, C, _), (_, _, dC) in zip(host, dev):
        dC.upload(C)
    assert call(handle, kind, arr, alpha, beta) == 0
    check(kind, host, dev, alpha, beta)


def test_grouped_d_alpha_zero(handle):
    """alpha == 0: C_i := beta C_i, A and B not referenced."""
    rng = np.random.default_rng(14)
    arr, host, dev = make(handle, rng, "d", 12)
    assert call(handle, "d", arr, 0.0, 2.0) == 0
    assert hb.device_error(handle) == 0
    for (ta, tb, M, N, K, A, lda, B, ldb, C, ldc), (_, _, dC) in zip(host, dev):
        gv = O.view_c(dC.download(), O.COL, M, N, ldc)
        assert np.array_equal(gv, 2.0 * O.view_c(C, O.COL, M, N, ldc))


def test_grouped_dcz_status_rules(handle):
    L = hb.lib()
    one = np.array([1.0, 0.0])
    assert call(None, "d", None, 1.0, 0.0) == hb.HCBLAS_STATUS_NOT_INITIALIZED
    assert call(handle, "z", None, 1.0, 0.0) == hb.HCBLAS_STATUS_SUCCESS  # count 0
    bad = (hb.GemmProblem * 1)(hb.GemmProblem(0, 0, -1, 4, 4, 16, 4, 16, 4, 16, 4))
    assert call(handle, "c", bad, 1.0, 0.0) == hb.HCBLAS_STATUS_INVALID_VALUE
    empty = (hb.GemmProblem * 1)(hb.GemmProblem(0, 0, 0, 4, 4, 16, 4, 16, 4, 16, 4))
    assert call(handle, "d", empty, 1.0, 0.0) == hb.HCBLAS_STATUS_EXECUTION_FAILED
    f = L.hcblasZgemmGrouped
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_void_p]
    assert f(handle, -1, None, one.ctypes.data, one.ctypes.data) == \
        hb.HCBLAS_STATUS_INVALID_VALUE
    assert f(handle, 1, ctypes.cast(empty, ctypes.c_void_p), None, one.ctypes.data) == \
        hb.HCBLAS_STATUS_INVALID_VALUE
