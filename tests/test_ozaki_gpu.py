"""GPU parity of the Ozaki-scheme DGEMM (INT8 slices on tcgen05) against the
double-double oracle.

Bound (a-priori, per element).  With e_m, f_n the row/column exponents
(|A(m,k)| < 2^e_m, |B(k,n)| < 2^f_n) and s slices of 7 bits:
  representation: |A - A_s| < 2^(e_m - 7s), same for B      -> 2 * 2^-7s
  dropped products a_i b_j with i + j >= s                 -> (s+1) * 2^-7s
so |C - C_s| <= |alpha| * K * (s+3) * 2^(e_m + f_n - 7s) + (s+2) u |C_s|.
The test uses the Frobenius norm of that elementwise bound.
"""
import numpy as np
import pytest

import hcblas_b200 as hb
from oracle import oracle as O
from tests.test_gemm_gpu import make_case, TCH

pytestmark = pytest.mark.gpu


def frexp_exp(x):
    _, e = np.frexp(np.max(np.abs(x)) if np.size(x) else 0.0)
    return e


def ozaki_bound(order, ta, tb, M, N, K, alpha, A, lda, B, ldb, s, ref):
    from tests.test_gemm_gpu import op_dense
    Ad = op_dense(A, order, ta, M, K, lda, 0)
    Bd = op_dense(B, order, tb, K, N, ldb, 0)
    ea = np.frexp(np.max(np.abs(Ad), axis=1))[1].astype(np.float64)
    eb = np.frexp(np.max(np.abs(Bd), axis=0))[1].astype(np.float64)
    scale = np.exp2(ea[:, None] + eb[None, :] - 7 * s)
    elem = abs(alpha) * K * (s + 3) * scale
    return np.linalg.norm(elem) + (s + 2) * 2.0 ** -53 * np.linalg.norm(ref)


def run_ozaki(handle, s, order, ta, tb, M, N, K, alpha, beta, A, lda, B, ldb, C, ldc):
    assert hb.hcblasSetMathMode(handle, hb.HCBLAS_MATH_OZAKI_INT8, s) == 0
    try:
        dA, dB, dC = (hb.DeviceArray(handle, X) for X in (A, B, C))
        rc = hb.lib_gemm(handle, order, TCH[ta], TCH[tb], M, N, K, alpha, dA, lda, dB, ldb, beta,
                         dC, ldc)
        assert rc == 0
        assert hb.device_error(handle) == 0
        path = hb.hcblasGetLastPath(handle)
        return dC.download(), path
    finally:
        hb.hcblasSetMathMode(handle, hb.HCBLAS_MATH_NATIVE, 0)


@pytest.mark.parametrize("s", [3, 4, 5, 6, 7, 8])
def test_ozaki_slices_vs_dd_oracle(handle, s):
    rng = np.random.default_rng(500 + s)
    cases = [(O.COL, 0, 1, 300, 200, 500), (O.COL, 1, 0, 129, 77, 64), (O.ROW, 0, 0, 256, 256, 1000),
             (O.COL, 1, 1, 1000, 130, 257)]
    for order, ta, tb, M, N, K in cases:
        A, lda, B, ldb, C, ldc = make_case(rng, "d", order, ta, tb, M, N, K)
        alpha, beta = 1.5, -0.25
        got, path = run_ozaki(handle, s, order, ta, tb, M, N, K, alpha, beta, A, lda, B, ldb, C, ldc)
        assert path == f"tc.ozaki_s{s}", path
        _, ref = O.gemm(order, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc)
        gv = O.view_c(got, order, M, N, ldc)
        err = np.linalg.norm(gv - ref)
        bound = ozaki_bound(order, ta, tb, M, N, K, alpha, A, lda, B, ldb, s, ref)
        assert err <= bound, (s, order, ta, tb, M, N, K, err, bound)


def test_ozaki_hard_exponent_range(handle):
    """Entries N(0,1) * 2^e, e ~ U{-20..20} per row of A and per column of B."""
    rng = np.random.default_rng(1)
    M = N = K = 512
    A = (rng.standard_normal((M, K)) * np.exp2(rng.integers(-20, 21, M))[:, None])
    B = (rng.standard_normal((K, N)) * np.exp2(rng.integers(-20, 21, N))[None, :])
    Af = np.asfortranarray(A).reshape(-1, order="F")
    Bf = np.asfortranarray(B).reshape(-1, order="F")
    C = np.zeros(M * N)
    _, ref = O.gemm(O.COL, 0, 0, M, N, K, 1.0, Af, M, Bf, K, 0.0, C, M)
    errs = {}
    for s in (5, 6, 7, 8):
        got, _ = run_ozaki(handle, s, O.COL, 0, 0, M, N, K, 1.0, 0.0, Af, M, Bf, K, C, M)
        errs[s] = O.normwise_rel_error(O.view_c(got, O.COL, M, N, M), ref)
        bound = ozaki_bound(O.COL, 0, 0, M, N, K, 1.0, Af, M, Bf, K, s, ref)
        assert np.linalg.norm(O.view_c(got, O.COL, M, N, M) - ref) <= bound
    print("ozaki hard-range normwise errors:", errs)
    assert errs[8] < errs[6] < errs[5]


def test_ozaki_special_rows(handle):
    rng = np.random.default_rng(4)
    M, N, K = 64, 48, 80
    A = rng.standard_normal(M * K)
    B = rng.standard_normal(K * N)
    A[3 + np.arange(K) * M] = 0.0       # row 3 of A all zero
    A[5 + 7 * M] = np.nan               # row 5 holds a NaN
    C = np.ones(M * N)
    got, _ = run_ozaki(handle, 7, O.COL, 0, 0, M, N, K, 1.0, 0.5, A, M, B, K, C, M)
    gv = O.view_c(got, O.COL, M, N, M)
    assert np.all(np.isnan(gv[5, :]))
    assert np.all(gv[3, :] == 0.5)
    ok = np.ones(M, bool)
    ok[5] = False
    A0 = np.nan_to_num(A)
    _, ref = O.gemm(O.COL, 0, 0, M, N, K, 1.0, A0, M, B, K, 0.5, C, M)
    ref_ok = ref[ok]
    bound = ozaki_bound(O.COL, 0, 0, M, N, K, 1.0, A0, M, B, K, 7, ref)
    assert np.linalg.norm(gv[ok] - ref_ok) <= bound


def test_ozaki_k_split(handle):
    """K beyond one launch's INT32-exact range (~16.6k for s = 8) is split."""
    rng = np.random.default_rng(6)
    M, N, K = 40, 36, 17000
    A, lda, B, ldb, C, ldc = make_case(rng, "d", O.COL, 1, 0, M, N, K)
    got, path = run_ozaki(handle, 8, O.COL, 1, 0, M, N, K, 1.0, 1.0, A, lda, B, ldb, C, ldc)
    _, ref = O.gemm(O.COL, 1, 0, M, N, K, 1.0, A, lda, B, ldb, 1.0, C, ldc)
    err = np.linalg.norm(O.view_c(got, O.COL, M, N, ldc) - ref)
    assert err <= ozaki_bound(O.COL, 1, 0, M, N, K, 1.0, A, lda, B, ldb, 8, ref)


def test_ozaki_vs_native_accuracy(handle):
    """Config of the headline: col-major N/T, N(0,1); report errors of native
    FP64 and Ozaki s = 6, 7, 8 against the double-double oracle."""
    rng = np.random.default_rng(1)
    M = N = K = 1024
    A = rng.standard_normal(M * K)
    B = rng.standard_normal(N * K)
    C = np.zeros(M * N)
    _, ref = O.gemm(O.COL, 0, 1, M, N, K, 1.0, A, M, B, N, 0.0, C, M)
    dA, dB, dC = (hb.DeviceArray(handle, X) for X in (A, B, C))
    assert hb.lib_gemm(handle, O.COL, "n", "t", M, N, K, 1.0, dA, M, dB, N, 0.0, dC, M) == 0
    errs = {"native": O.normwise_rel_error(O.view_c(dC.download(), O.COL, M, N, M), ref)}
    for s in (6, 7, 8):
        got, _ = run_ozaki(handle, s, O.COL, 0, 1, M, N, K, 1.0, 0.0, A, M, B, N, C, M)
        errs[s] = O.normwise_rel_error(O.view_c(got, O.COL, M, N, M), ref)
    print("native vs ozaki normwise errors:", errs)
    assert errs[8] <= errs["native"] * 4
