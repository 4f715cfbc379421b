"""Strided batches of CRT (Ozaki scheme II) DGEMMs in one pass per kernel.

hcblasDgemmStridedBatched under HCBLAS_MATH_OZAKI_CRT with a norm-scaled plan
(an explicit moduli count below the full width, or the native-accuracy
target) runs the row scales, the residues, one modular GEMM over every
(element, modulus) plane and the combine once for the whole batch (path
`tc.crt_m<n>.batched`).  Every kernel computes exactly what it computes for a
single GEMM, so each element must equal, bit for bit, the same GEMM made by
itself; the oracle check bounds the error as the single-call tests do.  A
workspace limit splits the batch into passes of a few elements, which must
change nothing either.  The full-width plan (moduli count 0 with no accuracy
target) keeps one emulated call per element.
"""
import numpy as np
import pytest

import hcblas_b200 as hb
from oracle import oracle as O

pytestmark = pytest.mark.gpu

N_, T_ = 0, 1


def _dense(X, trans, rows, cols, ld):
    """op(X) as a dense rows x cols array from column-major storage."""
    if trans == N_:
        return X[: ld * cols].reshape(cols, ld)[:, :rows].T
    return X[: ld * rows].reshape(rows, ld)[:, :cols]


def _case(rng, ta, tb, M, N, K, batch, pad=5):
    lda = (M if ta == N_ else K) + pad
    ldb = (K if tb == N_ else N) + pad
    ldc = M + pad
    sA = lda * (K if ta == N_ else M) + 3
    sB = ldb * (N if tb == N_ else K) + 7
    sC = ldc * N + 11
    A = rng.standard_normal(sA * batch)
    B = rng.standard_normal(sB * batch)
    C = rng.standard_normal(sC * batch)
    return (lda, ldb, ldc, sA, sB, sC), A, B, C


def _run_batched(h, ta, tb, M, N, K, lds, A, B, C, alpha, beta, batch):
    lda, ldb, ldc, sA, sB, sC = lds
    dA, dB, dC = (hb.DeviceArray(h, X) for X in (A, B, C))
    s = hb.gemm_strided_batched(h, ta, tb, M, N, K, alpha, dA, lda, sA, dB, ldb, sB, beta,
                                dC, ldc, sC, batch)
    assert s == hb.HCBLAS_STATUS_SUCCESS
    assert hb.device_error(h) == 0
    return dC.download(), hb.hcblasGetLastPath(h)


def _run_each(h, ta, tb, M, N, K, lds, A, B, C, alpha, beta, batch):
    lda, ldb, ldc, sA, sB, sC = lds
    out = C.copy()
    for i in range(batch):
        dA = hb.DeviceArray(h, A[i * sA:(i + 1) * sA])
        dB = hb.DeviceArray(h, B[i * sB:(i + 1) * sB])
        dC = hb.DeviceArray(h, C[i * sC:(i + 1) * sC])
        assert hb.gemm(h, ta, tb, M, N, K, alpha, dA, lda, dB, ldb, beta, dC, ldc) == 0
        out[i * sC:(i + 1) * sC] = dC.download()
    assert hb.device_error(h) == 0
    return out, hb.hcblasGetLastPath(h)


@pytest.mark.parametrize("ta,tb,M,N,K,batch", [
    (N_, T_, 128, 128, 128, 24),   # the strided 128^3 batch shape
    (T_, N_, 37, 53, 91, 9),       # ragged, K-contiguous operands
    (N_, N_, 200, 64, 300, 5),
    (T_, T_, 64, 150, 77, 6),
])
def test_batched_crt_equals_single_calls(handle, ta, tb, M, N, K, batch):
    rng = np.random.default_rng(900 + M + N + K)
    lds, A, B, C = _case(rng, ta, tb, M, N, K, batch)
    alpha, beta = 0.75, -0.5
    assert hb.hcblasSetMathMode(handle, hb.HCBLAS_MATH_OZAKI_CRT, 14) == 0
    try:
        got, path = _run_batched(handle, ta, tb, M, N, K, lds, A, B, C, alpha, beta, batch)
        assert path == "tc.crt_m14.batched", path
        ref_each, path1 = _run_each(handle, ta, tb, M, N, K, lds, A, B, C, alpha, beta, batch)
        assert path1 == "tc.crt_m14", path1
    finally:
        hb.hcblasSetMathMode(handle, hb.HCBLAS_MATH_NATIVE, 0)
    assert np.array_equal(got, ref_each)  # C outside the M x N windows included
    # against the double-double oracle: the single-call tests' bound
    lda, ldb, ldc, sA, sB, sC = lds
    for i in (0, batch - 1):
        Ai, Bi, Ci = A[i * sA:(i + 1) * sA], B[i * sB:(i + 1) * sB], C[i * sC:(i + 1) * sC]
        _, ref = O.gemm(O.COL, ta, tb, M, N, K, alpha, Ai, lda, Bi, ldb, beta, Ci, ldc)
        gv = O.view_c(got[i * sC:(i + 1) * sC], O.COL, M, N, ldc)
        bound = 2.0 ** -50 * np.linalg.norm(
            abs(alpha) * np.abs(_dense(Ai, ta, M, K, lda)) @ np.abs(_dense(Bi, tb, K, N, ldb)) +
            abs(beta) * np.abs(O.view_c(Ci, O.COL, M, N, ldc)))
        assert np.linalg.norm(gv - ref) <= bound, i


def test_batched_crt_in_passes(handle):
    """A workspace limit of a few elements per pass gives the same bits."""
    rng = np.random.default_rng(77)
    M, N, K, batch = 96, 112, 160, 11
    lds, A, B, C = _case(rng, N_, T_, M, N, K, batch)
    assert hb.hcblasSetMathMode(handle, hb.HCBLAS_MATH_OZAKI_CRT, 14) == 0
    try:
        whole, path = _run_batched(handle, N_, T_, M, N, K, lds, A, B, C, 1.0, 0.25, batch)
        assert path == "tc.crt_m14.batched"
        # 14 moduli of 96 x 160 and 112 x 160 int8 planes and a 96 x 112 C plane
        # per element: about 0.9 MiB; 3 MiB holds three elements per pass
        assert hb.set_tuning(handle, "workspace_mb", 3) == 0
        parts, path = _run_batched(handle, N_, T_, M, N, K, lds, A, B, C, 1.0, 0.25, batch)
        assert path == "tc.crt_m14.batched"
    finally:
        hb.set_tuning(handle, "workspace_mb", 0)
        hb.hcblasSetMathMode(handle, hb.HCBLAS_MATH_NATIVE, 0)
    assert np.array_equal(whole, parts)


def test_batched_crt_native_accuracy_target(handle):
    """The accuracy target "native" plans 14 norm-scaled moduli: batched."""
    rng = np.random.default_rng(78)
    M, N, K, batch = 128, 128, 128, 8
    lds, A, B, C = _case(rng, N_, T_, M, N, K, batch, pad=0)
    assert hb.hcblasSetMathMode(handle, hb.HCBLAS_MATH_OZAKI_CRT, 0) == 0
    assert hb.hcblasSetAccuracyTarget(handle, hb.HCBLAS_ACCURACY_NATIVE) == 0
    try:
        got, path = _run_batched(handle, N_, T_, M, N, K, lds, A, B, C, 1.0, 0.0, batch)
        assert path.startswith("tc.crt_m") and path.endswith(".batched"), path
    finally:
        hb.hcblasSetAccuracyTarget(handle, hb.HCBLAS_ACCURACY_DEFAULT)
        hb.hcblasSetMathMode(handle, hb.HCBLAS_MATH_NATIVE, 0)
    lda, ldb, ldc, sA, sB, sC = lds
    worst = 0.0
    for i in range(batch):
        _, ref = O.gemm(O.COL, N_, T_, M, N, K, 1.0, A[i * sA:(i + 1) * sA], lda,
                        B[i * sB:(i + 1) * sB], ldb, 0.0, C[i * sC:(i + 1) * sC], ldc)
        gv = O.view_c(got[i * sC:(i + 1) * sC], O.COL, M, N, ldc)
        worst = max(worst, O.normwise_rel_error(gv, ref))
    assert worst < 1e-15, worst


def test_full_width_plan_stays_per_element(handle):
    rng = np.random.default_rng(79)
    M, N, K, batch = 64, 48, 96, 3
    lds, A, B, C = _case(rng, N_, N_, M, N, K, batch)
    assert hb.hcblasSetMathMode(handle, hb.HCBLAS_MATH_OZAKI_CRT, 0) == 0
    try:
        got, path = _run_batched(handle, N_, N_, M, N, K, lds, A, B, C, 1.0, 1.0, batch)
        assert path.startswith("tc.crt_m") and not path.endswith(".batched"), path
    finally:
        hb.hcblasSetMathMode(handle, hb.HCBLAS_MATH_NATIVE, 0)
    lda, ldb, ldc, sA, sB, sC = lds
    for i in range(batch):
        _, ref = O.gemm(O.COL, N_, N_, M, N, K, 1.0, A[i * sA:(i + 1) * sA], lda,
                        B[i * sB:(i + 1) * sB], ldb, 1.0, C[i * sC:(i + 1) * sC], ldc)
        gv = O.view_c(got[i * sC:(i + 1) * sC], O.COL, M, N, ldc)
        assert O.normwise_rel_error(gv, ref) < 1e-15, i
