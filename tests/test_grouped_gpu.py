"""Grouped HGEMM (hcblasHgemmGrouped): many uneven problems in one persistent
tcgen05 launch, checked problem by problem against the CPU oracle.

Tolerance per problem (f16 storage of C, f32 accumulation):
    ||C_gpu - C_ref||_F <= 2^-11 ||C_ref||_F + 2 gamma_{K+2}(f32) || |alpha||A||B| + |beta||C| ||_F
Shapes follow the grouped-batch workload (M, N, K log-uniform integers, mixed
N/T) at sizes the oracle finishes quickly.
"""
import numpy as np
import pytest

import hcblas_b200 as hb
from oracle import oracle as O

pytestmark = pytest.mark.gpu

U32 = 2.0 ** -24


def g32(K):
    return (K + 2) * U32 / (1 - (K + 2) * U32)


def op_dense(X, trans, rows, cols, ld):
    if trans == 0:
        return X[: ld * cols].reshape(cols, ld)[:, :rows].T.astype(np.float64)
    return X[: ld * rows].reshape(rows, ld)[:, :cols].astype(np.float64)


def loguniform(rng, lo, hi):
    return int(np.exp(rng.uniform(np.log(lo), np.log(hi + 1))))


def make_problems(handle, rng, count, lo=16, hi=600, align=8, misalign=(), dtype=np.float16,
                  pad=None):
    probs, host, dev = [], [], []
    for i in range(count):
        ta, tb = int(rng.integers(0, 2)), int(rng.integers(0, 2))
        M, N, K = (loguniform(rng, lo, hi) for _ in range(3))
        ra, rb = (M if ta == 0 else K), (K if tb == 0 else N)
        rnd = lambda v: -(-v // align) * align
        lda = rnd(ra) + (1 if i in misalign else 0)
        ldb = rnd(rb)
        if pad is not None:  # arbitrary leading dimensions
            lda, ldb = ra + int(rng.integers(0, pad)), rb + int(rng.integers(0, pad))
        ldc = M + int(rng.integers(0, 3))
        A = rng.uniform(-1, 1, lda * (K if ta == 0 else M)).astype(dtype)
        B = rng.uniform(-1, 1, ldb * (N if tb == 0 else K)).astype(dtype)
        C = rng.uniform(-1, 1, ldc * N).astype(dtype)
        dA, dB, dC = (hb.DeviceArray(handle, X) for X in (A, B, C))
        probs.append(hb.GemmProblem(ta, tb, M, N, K, dA.ptr, lda, dB.ptr, ldb, dC.ptr, ldc))
        host.append((ta, tb, M, N, K, A, lda, B, ldb, C, ldc))
        dev.append((dA, dB, dC))
    return probs, host, dev


def check(host, dev, alpha, beta):
    worst = 0.0
    for (ta, tb, M, N, K, A, lda, B, ldb, C, ldc), (_, _, dC) in zip(host, dev):
        got = dC.download()
        _, ref = O.gemm(O.COL, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc)
        gv = O.view_c(got, O.COL, M, N, ldc).astype(np.float64)
        Ad, Bd = np.abs(op_dense(A, ta, M, K, lda)), np.abs(op_dense(B, tb, K, N, ldb))
        cc = abs(beta) * np.abs(O.view_c(C, O.COL, M, N, ldc).astype(np.float64))
        bound = 2.0 ** -11 * np.linalg.norm(ref) + \
            2 * g32(K) * np.linalg.norm(abs(alpha) * (Ad @ Bd) + cc)
        err = np.linalg.norm(gv - ref)
        assert err <= bound, (ta, tb, M, N, K, err, bound)
        # columns of C beyond row M (ld padding) are untouched
        assert np.array_equal(got[: ldc * N].reshape(N, ldc)[:, M:],
                              C[: ldc * N].reshape(N, ldc)[:, M:])
        worst = max(worst, err / max(bound, 1e-30))
    return worst


def test_grouped_uneven_mixed_transposes(handle):
    rng = np.random.default_rng(3)
    probs, host, dev = make_problems(handle, rng, 48)
    assert hb.hgemm_grouped(handle, probs, 1.0, 0.5) == 0
    assert hb.device_error(handle) == 0
    assert hb.hcblasGetLastPath(handle) == "tc.h.grouped"
    check(host, dev, 1.0, 0.5)


def test_grouped_reuses_plan_with_new_data(handle):
    """A second call with the same problem array reuses the device table; the
    results must follow the new matrix contents."""
    rng = np.random.default_rng(4)
    probs, host, dev = make_problems(handle, rng, 20, lo=16, hi=300)
    assert hb.hgemm_grouped(handle, probs, 1.0, 0.0) == 0
    new_host = []
    for (ta, tb, M, N, K, A, lda, B, ldb, C, ldc), (dA, dB, dC) in zip(host, dev):
        A2 = rng.uniform(-1, 1, A.size).astype(np.float16)
        C2 = rng.uniform(-1, 1, C.size).astype(np.float16)
        dA.upload(A2)
        dC.upload(C2)
        new_host.append((ta, tb, M, N, K, A2, lda, B, ldb, C2, ldc))
    assert hb.hgemm_grouped(handle, probs, -0.75, 1.25) == 0
    assert hb.device_error(handle) == 0
    check(new_host, dev, -0.75, 1.25)


def test_grouped_unaligned_problems_fall_back(handle):
    rng = np.random.default_rng(5)
    probs, host, dev = make_problems(handle, rng, 12, lo=16, hi=200, misalign=(2, 7))
    assert hb.hgemm_grouped(handle, probs, 1.0, 1.0) == 0
    assert hb.device_error(handle) == 0
    assert hb.hcblasGetLastPath(handle) == "tc.h.grouped+single"
    check(host, dev, 1.0, 1.0)


def test_grouped_alpha_zero_scales_c(handle):
    rng = np.random.default_rng(6)
    probs, host, dev = make_problems(handle, rng, 6, lo=16, hi=100)
    assert hb.hgemm_grouped(handle, probs, 0.0, 0.5) == 0
    for (ta, tb, M, N, K, A, lda, B, ldb, C, ldc), (_, _, dC) in zip(host, dev):
        got = O.view_c(dC.download(), O.COL, M, N, ldc)
        want = (0.5 * O.view_c(C, O.COL, M, N, ldc).astype(np.float32)).astype(np.float16)
        assert np.array_equal(got, want)


def test_grouped_status_rules(handle):
    rng = np.random.default_rng(7)
    probs, _, dev = make_problems(handle, rng, 3, lo=16, hi=64)
    assert hb.hgemm_grouped(handle, [], 1.0, 0.0) == hb.HCBLAS_STATUS_SUCCESS
    bad = [hb.GemmProblem(0, 0, -1, 8, 8, probs[0].A, 8, probs[0].B, 8, probs[0].C, 8)]
    assert hb.hgemm_grouped(handle, probs + bad, 1.0, 0.0) == hb.HCBLAS_STATUS_INVALID_VALUE
    empty = [hb.GemmProblem(0, 0, 8, 0, 8, probs[0].A, 8, probs[0].B, 8, probs[0].C, 8)]
    assert hb.hgemm_grouped(handle, probs + empty, 1.0, 0.0) == \
        hb.HCBLAS_STATUS_EXECUTION_FAILED
    L = hb.lib()
    assert L.hcblasHgemmGrouped(handle, -1, None, None, None) == hb.HCBLAS_STATUS_INVALID_VALUE
    assert L.hcblasHgemmGrouped(None, 1, None, None, None) == hb.HCBLAS_STATUS_NOT_INITIALIZED


@pytest.mark.parametrize("ta,tb", [(0, 0), (1, 0), (0, 1), (1, 1)])
def test_strided_batched_hgemm_is_grouped(handle, ta, tb):
    """hcblasHgemmStridedBatched with TMA-addressable strides runs as one
    grouped launch (one table entry per batch element)."""
    rng = np.random.default_rng(40 + 2 * ta + tb)
    M, N, K, batch = 128, 96, 72, 24
    lda = (M if ta == 0 else K) + 8
    ldb = (K if tb == 0 else N) + 16
    ldc = M + 3
    sA = lda * (K if ta == 0 else M) + 64
    sB = ldb * (N if tb == 0 else K) + 8
    sC = ldc * N + 5
    A = rng.uniform(-1, 1, sA * batch).astype(np.float16)
    B = rng.uniform(-1, 1, sB * batch).astype(np.float16)
    C = rng.uniform(-1, 1, sC * batch).astype(np.float16)
    dA, dB, dC = (hb.DeviceArray(handle, X) for X in (A, B, C))
    s = hb.gemm_strided_batched(handle, ta, tb, M, N, K, 0.5, dA, lda, sA, dB, ldb, sB, -1.0, dC,
                                ldc, sC, batch)
    assert s == hb.HCBLAS_STATUS_SUCCESS
    assert hb.device_error(handle) == 0
    assert hb.hcblasGetLastPath(handle) == "tc.h.grouped"
    got = dC.download()
    for i in range(batch):
        Ai, Bi, Ci = A[i * sA:(i + 1) * sA], B[i * sB:(i + 1) * sB], C[i * sC:(i + 1) * sC]
        _, ref = O.gemm(O.COL, ta, tb, M, N, K, 0.5, Ai, lda, Bi, ldb, -1.0, Ci, ldc)
        gv = O.view_c(got[i * sC:(i + 1) * sC], O.COL, M, N, ldc).astype(np.float64)
        Ad, Bd = np.abs(op_dense(Ai, ta, M, K, lda)), np.abs(op_dense(Bi, tb, K, N, ldb))
        cc = np.abs(O.view_c(Ci, O.COL, M, N, ldc).astype(np.float64))
        bound = 2.0 ** -11 * np.linalg.norm(ref) + 2 * g32(K) * np.linalg.norm(0.5 * (Ad @ Bd) + cc)
        assert np.linalg.norm(gv - ref) <= bound, i
        assert np.array_equal(got[i * sC + ldc * N:(i + 1) * sC], C[i * sC + ldc * N:(i + 1) * sC])


# ------------------------------------------------- grouped FP32 (split-BF16)

def check_f32(host, dev, alpha, beta, rel=0.0):
    """Per problem: the plain-FP32 normwise bound
        ||C_gpu - C_ref||_F <= gamma_{K+2}(f32) || |alpha||A||B| + |beta||C| ||_F
    (+ rel ||C_ref||_F for the 3-term split, whose planes carry ~16 bits)."""
    for (ta, tb, M, N, K, A, lda, B, ldb, C, ldc), (_, _, dC) in zip(host, dev):
        got = dC.download()
        _, ref = O.gemm(O.COL, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc)
        gv = O.view_c(got, O.COL, M, N, ldc).astype(np.float64)
        Ad, Bd = np.abs(op_dense(A, ta, M, K, lda)), np.abs(op_dense(B, tb, K, N, ldb))
        cc = abs(beta) * np.abs(O.view_c(C, O.COL, M, N, ldc).astype(np.float64))
        bound = g32(K) * np.linalg.norm(abs(alpha) * (Ad @ Bd) + cc) + rel * np.linalg.norm(ref)
        err = np.linalg.norm(gv - ref)
        assert err <= bound, (ta, tb, M, N, K, err, bound)
        assert np.array_equal(got[: ldc * N].reshape(N, ldc)[:, M:],
                              C[: ldc * N].reshape(N, ldc)[:, M:])


def test_sgemm_grouped_split_uneven_any_leading_dimension(handle):
    """f32 problems with unpadded, odd leading dimensions and mixed
    transposes, all in one packing launch and one grouped tensor-core launch;
    6 products keep every problem within the plain FP32 bound."""
    rng = np.random.default_rng(30)
    probs, host, dev = make_problems(handle, rng, 40, lo=8, hi=400, dtype=np.float32, pad=4)
    assert hb.sgemm_grouped(handle, probs, 1.25, 0.5) == 0
    assert hb.device_error(handle) == 0
    assert hb.hcblasGetLastPath(handle) == "tc.s.grouped_split_bf16x6"
    check_f32(host, dev, 1.25, 0.5)


def test_sgemm_grouped_split3_and_plan_reuse(handle):
    """The 3-term split under HCBLAS_MATH_SPLIT_BF16 param 3; a second call
    with the same problem array reuses the plan but packs the new contents."""
    rng = np.random.default_rng(31)
    probs, host, dev = make_problems(handle, rng, 16, lo=16, hi=300, dtype=np.float32, pad=3)
    assert hb.hcblasSetMathMode(handle, hb.HCBLAS_MATH_SPLIT_BF16, 3) == 0
    try:
        assert hb.sgemm_grouped(handle, probs, 1.0, 0.0) == 0
        assert hb.hcblasGetLastPath(handle) == "tc.s.grouped_split_bf16x3"
        new_host = []
        for (ta, tb, M, N, K, A, lda, B, ldb, C, ldc), (dA, dB, dC) in zip(host, dev):
            A2 = rng.uniform(-1, 1, A.size).astype(np.float32)
            dA.upload(A2)
            dC.upload(C)
            new_host.append((ta, tb, M, N, K, A2, lda, B, ldb, C, ldc))
        assert hb.sgemm_grouped(handle, probs, -0.5, 2.0) == 0
        assert hb.device_error(handle) == 0
    finally:
        hb.hcblasSetMathMode(handle, hb.HCBLAS_MATH_NATIVE, 0)
    check_f32(new_host, dev, -0.5, 2.0, rel=2.0 ** -14)


def test_sgemm_grouped_alpha_zero_and_status(handle):
    rng = np.random.default_rng(32)
    probs, host, dev = make_problems(handle, rng, 5, lo=8, hi=90, dtype=np.float32, pad=2)
    assert hb.sgemm_grouped(handle, probs, 0.0, 0.5) == 0
    for (ta, tb, M, N, K, A, lda, B, ldb, C, ldc), (_, _, dC) in zip(host, dev):
        got = O.view_c(dC.download(), O.COL, M, N, ldc)
        assert np.array_equal(got, 0.5 * O.view_c(C, O.COL, M, N, ldc))
    assert hb.sgemm_grouped(handle, [], 1.0, 0.0) == hb.HCBLAS_STATUS_SUCCESS
    bad = [hb.GemmProblem(0, 0, 4, -1, 4, probs[0].A, 8, probs[0].B, 8, probs[0].C, 8)]
    assert hb.sgemm_grouped(handle, probs + bad, 1.0, 0.0) == hb.HCBLAS_STATUS_INVALID_VALUE
    L = hb.lib()
    assert L.hcblasSgemmGrouped(None, 1, None, None, None) == hb.HCBLAS_STATUS_NOT_INITIALIZED


@pytest.mark.parametrize("ctas,c_tma", [(1, 1), (2, 1), (1, 0), (2, 0)])
def test_grouped_kernel_configurations(handle, ctas, c_tma):
    """Both shapes of the grouped kernel (one CTA per SM with a 6-stage ring,
    two with 3 stages each), with C written through TMA boxes or by direct
    stores, give results within the bound, beta != 0, ld padding untouched."""
    rng = np.random.default_rng(40 + ctas + 2 * c_tma)
    probs, host, dev = make_problems(handle, rng, 40)
    assert hb.set_tuning(handle, "grouped_ctas", ctas) == 0
    assert hb.set_tuning(handle, "grouped_c_tma", c_tma) == 0
    try:
        assert hb.hgemm_grouped(handle, probs, 0.75, -1.5) == 0
        assert hb.device_error(handle) == 0
    finally:
        hb.set_tuning(handle, "grouped_ctas", 2)
        hb.set_tuning(handle, "grouped_c_tma", 1)
    check(host, dev, 0.75, -1.5)
