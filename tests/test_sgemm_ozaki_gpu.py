"""GPU parity of SGEMM on the INT8 Ozaki-I path (HCBLAS_MATH_OZAKI_INT8 on an
FP32 call): the FP32 operands are widened exactly to FP64, split into s int8
slices of 7 bits per row / column exponent, the slice-group products summed
exactly in INT32 on the int8 tensor cores, weighted in FP64 and rounded once
into the FP32 C.  Checked against the FP64 oracle: with s = 4 (28 bits per
entry, above FP32's 24) the error must not exceed the plain FP32 kernel's on
the same call; s = 3 must stay within the element-wise slice bound."""
import numpy as np
import pytest

import hcblas_b200 as hb
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TCH = {0: "n", 1: "t"}


@pytest.fixture(scope="module")
def handle():
    s, h = hb.hcblasCreate(0)
    assert s == 0
    yield h
    hb.hcblasDestroy(h)


def run(handle, mode, param, order, ta, tb, M, N, K, alpha, beta, A, lda, B, ldb, C, ldc):
    assert hb.hcblasSetMathMode(handle, mode, param) == 0
    try:
        dA, dB, dC = (hb.DeviceArray(handle, X) for X in (A, B, C))
        assert hb.lib_gemm(handle, order, TCH[ta], TCH[tb], M, N, K, alpha, dA, lda, dB, ldb,
                           beta, dC, ldc) == 0
        assert hb.device_error(handle) == 0
        return dC.download(), hb.hcblasGetLastPath(handle)
    finally:
        hb.hcblasSetMathMode(handle, hb.HCBLAS_MATH_NATIVE, 0)


CASES = [(O.COL, 1, 0, 300, 260, 1000), (O.COL, 0, 1, 129, 77, 64), (O.ROW, 0, 0, 256, 200, 513),
         (O.COL, 1, 1, 500, 96, 2048)]


def make(rng, order, ta, tb, M, N, K):
    """N(0,1) * 2^e with e ~ U{-8..8} per row of op(A) / column of op(B)"""
    ea = np.exp2(rng.integers(-8, 9, M))
    eb = np.exp2(rng.integers(-8, 9, N))
    Ad = rng.standard_normal((M, K)) * ea[:, None]
    Bd = rng.standard_normal((K, N)) * eb[None, :]
    C = rng.standard_normal(M * N).astype(np.float32)

    def store(X, t, ld_major):
        S = X if t == 0 else X.T
        return (np.asfortranarray(S).reshape(-1, order="F") if order == O.COL
                else np.ascontiguousarray(S).reshape(-1)).astype(np.float32), ld_major
    A, lda = store(Ad, ta, None)
    B, ldb = store(Bd, tb, None)
    if order == O.COL:
        lda = M if ta == 0 else K
        ldb = K if tb == 0 else N
        ldc = M
    else:
        lda = K if ta == 0 else M
        ldb = N if tb == 0 else K
        ldc = N
    return A, lda, B, ldb, C, ldc


@pytest.mark.parametrize("s", [3, 4])
def test_sgemm_ozaki_int8_vs_oracle(handle, s):
    rng = np.random.default_rng(80 + s)
    for order, ta, tb, M, N, K in CASES:
        A, lda, B, ldb, C, ldc = make(rng, order, ta, tb, M, N, K)
        alpha, beta = 1.0, 1.0
        _, ref = O.gemm(order, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc)
        got, path = run(handle, hb.HCBLAS_MATH_OZAKI_INT8, s, order, ta, tb, M, N, K, alpha, beta,
                        A, lda, B, ldb, C, ldc)
        assert path == f"tc.sozaki_i8_s{s}", path
        plain, _ = run(handle, hb.HCBLAS_MATH_NATIVE, 0, order, ta, tb, M, N, K, alpha, beta,
                       A, lda, B, ldb, C, ldc)
        err = O.normwise_rel_error(O.view_c(got, order, M, N, ldc), ref)
        err_plain = O.normwise_rel_error(O.view_c(plain, order, M, N, ldc), ref)
        if s == 4:
            assert err <= err_plain, (order, ta, tb, M, N, K, err, err_plain)
        else:
            # 21 bits per entry relative to its row / column maximum
            assert err <= 64 * 2.0 ** -21, (order, ta, tb, M, N, K, err)
