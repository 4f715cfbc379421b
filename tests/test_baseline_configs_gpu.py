"""Parity at the benchmark configurations themselves (full sizes), through the
C ABI, on sampled output columns against the CPU oracle (double-double for
D/Z, binary64 for S/C/H).  Every matched-error claim of the benchmark is
asserted here:

  C1  SGEMM row-major NN 1024^3, alpha 1, beta 0.5, U[-1,1) seed 0: plain
      FP32 within gamma_{K+2} || |A||B| + |beta C| ||.
  C2  DGEMM col-major NT 4096^3, N(0,1) seed 1, and the hard variant
      N(0,1) 2^e, e ~ U{-20..20} per row of A / column of op(B): the CRT
      path with the accuracy target "native" (no moduli count given) takes
      14 moduli and is no less accurate than the native FP64 kernel; its
      error meets the planner's model (normalised RMS <= 2^-53); Ozaki-I at
      5, 6 and 7 slices stays within its a-priori bound.
  C3  SGEMM col-major TN, alpha = beta = 1, N(0,1) 2^e with e ~ U{-8..8} per
      row/column, seed 2, at 8192^3 and 8192 x 8192 x 256: split-BF16 with 6
      products is no less accurate than plain FP32.
  C4  batched: 16 sampled problems of the strided 512 x 128^3 f16 batch and
      of the 4096-problem uneven grouped sets (f16, and f32 on the split-BF16
      path) within their bounds.
  C5  CGEMM / ZGEMM col-major CN 2048^3, alpha (1, 0.5), beta (0.5, -0.25),
      N(0,1) parts seed 4: ZGEMM CRT with the native target (14 moduli) no
      less accurate than native FP64; CGEMM 3M split-BF16 x6 no less accurate
      than plain 4M FP32.

Sampled columns keep the oracle to seconds; the GPU computes the whole
product.  The reference's own tests use the same normwise measure
(test/unit/hcblas_sgemm.cpp:260-261, helper_functions.h:10-53).
"""
import numpy as np
import pytest

import hcblas_b200 as hb
from oracle import oracle as O
from tests.test_ozaki_gpu import ozaki_bound

pytestmark = pytest.mark.gpu

U64, U32 = 2.0 ** -53, 2.0 ** -24
MATH = {"native": hb.HCBLAS_MATH_NATIVE, "split": hb.HCBLAS_MATH_SPLIT_BF16,
        "ozaki": hb.HCBLAS_MATH_OZAKI_INT8, "crt": hb.HCBLAS_MATH_OZAKI_CRT}
TCH = {0: "n", 1: "t", 2: "c"}


def g(K, u):
    return (K + 2) * u / (1 - (K + 2) * u)


def op_b_cols(B, tb, K, ldb, cols):
    """op(B)[:, cols] as a dense K x len(cols) column-major flat array."""
    if tb == 0:
        return np.ascontiguousarray(B.reshape(-1, ldb)[cols, :K]).reshape(-1)
    sub = B.reshape(K, ldb)[:, cols].T  # (ncols, K): column j of op(B) is row j of B
    sub = np.conj(sub) if tb == 2 else sub
    return np.ascontiguousarray(sub).reshape(-1)


def sampled_ref(ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, cols):
    """Oracle of C[:, cols] (M x len(cols)) and the dense op(B)[:, cols]."""
    Bs = op_b_cols(B, tb, K, ldb, cols)
    Cs = (np.zeros(M * len(cols), A.dtype) if C is None else
          np.ascontiguousarray(C.reshape(-1, ldc)[cols, :M]).reshape(-1))
    _, ref = O.gemm(O.COL, ta, 0, M, len(cols), K, alpha, A, lda, Bs, K, beta, Cs, M)
    return ref, Bs.reshape(len(cols), K).T


def op_a_dense(A, ta, M, K, lda):
    if ta == 0:
        return A.reshape(-1, lda)[:K, :M].T
    X = A.reshape(-1, lda)[:M, :K]
    return np.conj(X) if ta == 2 else X


def run(handle, kind, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, mode="native",
        param=0, accuracy=0):
    """One C-ABI call; returns (C on the host as M x N view, path)."""
    assert hb.hcblasSetMathMode(handle, MATH[mode], param) == 0
    assert hb.hcblasSetAccuracyTarget(handle, accuracy) == 0
    try:
        dA, dB = hb.DeviceArray(handle, A), hb.DeviceArray(handle, B)
        dC = hb.DeviceArray(handle, C) if C is not None else hb.DeviceArray(
            handle, np.zeros(ldc * N, A.dtype))
        rc = hb.lib_gemm(handle, O.COL, TCH[ta], TCH[tb], M, N, K, alpha, dA, lda, dB, ldb, beta,
                         dC, ldc)
        assert rc == 0
        assert hb.device_error(handle) == 0
        path = hb.hcblasGetLastPath(handle)
        out = dC.download()
        for X in (dA, dB, dC):
            X.free()
    finally:
        hb.hcblasSetMathMode(handle, hb.HCBLAS_MATH_NATIVE, 0)
        hb.hcblasSetAccuracyTarget(handle, 0)
    return O.view_c(out, O.COL, M, N, ldc), path


def rel(got_cols, ref):
    return O.normwise_rel_error(got_cols, ref)


# ------------------------------------------------------------------- C1 --

def test_c1_sgemm_rowmajor_nn_1024(handle):
    rng = np.random.default_rng(0)
    n = 1024
    A = rng.uniform(-1, 1, n * n).astype(np.float32)
    B = rng.uniform(-1, 1, n * n).astype(np.float32)
    C = rng.uniform(-1, 1, n * n).astype(np.float32)
    dA, dB, dC = (hb.DeviceArray(handle, X) for X in (A, B, C))
    assert hb.lib_gemm(handle, O.ROW, "n", "n", n, n, n, 1.0, dA, n, dB, n, 0.5, dC, n) == 0
    got = O.view_c(dC.download(), O.ROW, n, n, n)
    _, ref = O.gemm(O.ROW, 0, 0, n, n, n, 1.0, A, n, B, n, 0.5, C, n)
    Ad, Bd = A.reshape(n, n).astype(np.float64), B.reshape(n, n).astype(np.float64)
    bound = g(n, U32) * np.linalg.norm(np.abs(Ad) @ np.abs(Bd) + 0.5 * np.abs(
        C.reshape(n, n).astype(np.float64)))
    err = np.linalg.norm(got - ref)
    print(f"C1 path {hb.hcblasGetLastPath(handle)} normwise {rel(got, ref):.3e}")
    assert err <= bound
    assert rel(got, ref) < 1e-5  # the reference test's L2 criterion


# ------------------------------------------------------------------- C2 --

def c2_inputs(hard):
    """The benchmark's own inputs: A column-major M x K (lda = M), B
    column-major N x K (op(B) = B^T, ldb = N)."""
    M = N = K = 4096
    if not hard:
        rng = np.random.default_rng(1)
        return M, N, K, rng.standard_normal(M * K), rng.standard_normal(N * K)
    hr = np.random.default_rng(11)
    A = (hr.standard_normal((K, M)) * np.exp2(hr.integers(-20, 21, M))[None, :]).reshape(-1)
    B = (hr.standard_normal((K, N)) * np.exp2(hr.integers(-20, 21, N))[None, :]).reshape(-1)
    return M, N, K, A, B


@pytest.mark.parametrize("hard", [False, True], ids=["normal", "hard_2e"])
def test_c2_dgemm_nt_4096_matched_error(handle, hard):
    M, N, K, A, B = c2_inputs(hard)
    cols = np.random.default_rng(5).choice(N, 16, replace=False)
    ref, Bs = sampled_ref(0, 1, M, N, K, 1.0, A, M, B, N, 0.0, None, M, cols)
    errs = {}
    got, path = run(handle, "d", 0, 1, M, N, K, 1.0, A, M, B, N, 0.0, None, M)
    errs["native"] = rel(got[:, cols], ref)
    # the planner: accuracy target "native", no moduli count given
    st, count, mbits = hb.plan_emulation(hb.HCBLAS_MATH_OZAKI_CRT, 0, -1, "d", K)
    assert st == 0 and count == 14 and mbits >= 53
    got, path = run(handle, "d", 0, 1, M, N, K, 1.0, A, M, B, N, 0.0, None, M, "crt",
                    accuracy=hb.HCBLAS_ACCURACY_NATIVE)
    assert path == "tc.crt_m14", path
    errs["crt_native_target"] = rel(got[:, cols], ref)
    # the model behind the plan: RMS of e_ij / (||a_i|| ||b_j||) <= 2^-53
    row_norms = np.linalg.norm(A.reshape(K, M), axis=0)
    col_norms = np.linalg.norm(Bs, axis=0)
    nrms = np.sqrt(np.mean(((got[:, cols] - ref) / (row_norms[:, None] * col_norms[None, :])) ** 2))
    assert nrms <= 2.0 ** -53, nrms
    for s in (5, 6, 7):
        got, path = run(handle, "d", 0, 1, M, N, K, 1.0, A, M, B, N, 0.0, None, M, "ozaki", s)
        assert path == f"tc.ozaki_i8_s{s}", path
        errs[f"ozaki_s{s}"] = rel(got[:, cols], ref)
        Bsub = np.ascontiguousarray(Bs).reshape(-1)  # B' = op(B)[:, cols]^T, ncols x K col-major
        bound = ozaki_bound(O.COL, 0, 1, M, len(cols), K, 1.0, A, M, Bsub, len(cols), s, ref)
        assert np.linalg.norm(got[:, cols] - ref) <= bound, (s, bound)
    print(f"C2 {'hard' if hard else 'normal'} normwise errors:", errs)
    assert errs["crt_native_target"] <= errs["native"], errs


# ------------------------------------------------------------------- C3 --

@pytest.mark.parametrize("K", [8192, 256])
def test_c3_sgemm_tn_split_matches_plain(handle, K):
    rng = np.random.default_rng(2)  # the benchmark's own inputs
    M = N = 8192
    # op(A) = A^T: A is K x M column-major (lda = K), row m of op(A) scaled by 2^e_m
    A = (rng.standard_normal((M, K)) * np.exp2(rng.integers(-8, 9, M))[:, None]).astype(
        np.float32).reshape(-1)
    # op(B) = B: K x N column-major (ldb = K), column n scaled by 2^e_n
    B = (rng.standard_normal((N, K)) * np.exp2(rng.integers(-8, 9, N))[:, None]).astype(
        np.float32).reshape(-1)
    C = rng.standard_normal(M * N).astype(np.float32)
    cols = np.random.default_rng(6).choice(N, 8, replace=False)
    ref, Bs = sampled_ref(1, 0, M, N, K, 1.0, A, K, B, K, 1.0, C, M, cols)
    errs = {}
    for mode, param in (("native", 0), ("split", 6)):
        got, path = run(handle, "s", 1, 0, M, N, K, 1.0, A, K, B, K, 1.0, C, M, mode, param)
        errs[path] = rel(got[:, cols], ref)
    print(f"C3 K={K} normwise errors:", errs)
    plain = [v for k, v in errs.items() if k.startswith("simt")][0]
    split = [v for k, v in errs.items() if k.startswith("tc.split_bf16x6")][0]
    assert split <= plain, errs
    Ad = op_a_dense(A, 1, M, K, K).astype(np.float64)
    Cd = C.reshape(N, M)[cols, :].T.astype(np.float64)
    bound = 2 * g(K, U32) * np.linalg.norm(np.abs(Ad) @ np.abs(Bs.astype(np.float64)) + np.abs(Cd))
    assert split * np.linalg.norm(ref) <= bound


# ------------------------------------------------------------------- C5 --

def c5_inputs(dtype):
    rng = np.random.default_rng(4)
    n = 2048
    A = (rng.standard_normal(n * n) + 1j * rng.standard_normal(n * n)).astype(dtype)
    B = (rng.standard_normal(n * n) + 1j * rng.standard_normal(n * n)).astype(dtype)
    C = (rng.standard_normal(n * n) + 1j * rng.standard_normal(n * n)).astype(dtype)
    return n, A, B, C


def test_c5_zgemm_cn_crt_native_target(handle):
    n, A, B, C = c5_inputs(np.complex128)
    alpha, beta = (1 + 0.5j), (0.5 - 0.25j)
    cols = np.random.default_rng(7).choice(n, 16, replace=False)
    ref, _ = sampled_ref(2, 0, n, n, n, alpha, A, n, B, n, beta, C, n, cols)
    got, _ = run(handle, "z", 2, 0, n, n, n, alpha, A, n, B, n, beta, C, n)
    native = rel(got[:, cols], ref)
    st, count, _ = hb.plan_emulation(hb.HCBLAS_MATH_OZAKI_CRT, 0, -1, "z", n)
    assert st == 0 and count == 14
    got, path = run(handle, "z", 2, 0, n, n, n, alpha, A, n, B, n, beta, C, n, "crt",
                    accuracy=hb.HCBLAS_ACCURACY_NATIVE)
    assert path == "tc.zcrt3m_m14", path
    crt = rel(got[:, cols], ref)
    print(f"C5 ZGEMM native {native:.3e} crt14 {crt:.3e}")
    assert crt <= native


def test_c5_cgemm_cn_split3m_matches_plain(handle):
    n, A, B, C = c5_inputs(np.complex64)
    alpha, beta = (1 + 0.5j), (0.5 - 0.25j)
    cols = np.random.default_rng(7).choice(n, 16, replace=False)
    ref, _ = sampled_ref(2, 0, n, n, n, alpha, A, n, B, n, beta, C, n, cols)
    got, _ = run(handle, "c", 2, 0, n, n, n, alpha, A, n, B, n, beta, C, n)
    plain = rel(got[:, cols], ref)
    got, path = run(handle, "c", 2, 0, n, n, n, alpha, A, n, B, n, beta, C, n, "split", 6)
    assert path.startswith("tc.csplit3m_bf16x6"), path
    split = rel(got[:, cols], ref)
    print(f"C5 CGEMM plain 4M {plain:.3e} split 3M x6 {split:.3e}")
    assert split <= plain


# ------------------------------------------------------------------- C4 --

def test_c4a_strided_hgemm_512x128(handle):
    rng = np.random.default_rng(5)
    n, b = 128, 512
    A = rng.uniform(-1, 1, n * n * b).astype(np.float16)
    B = rng.uniform(-1, 1, n * n * b).astype(np.float16)
    dA, dB = hb.DeviceArray(handle, A), hb.DeviceArray(handle, B)
    dC = hb.DeviceArray(handle, np.zeros(n * n * b, np.float16))
    assert hb.gemm_strided_batched(handle, 0, 0, n, n, n, 1.0, dA, n, n * n, dB, n, n * n, 0.0,
                                   dC, n, n * n, b) == 0
    assert hb.device_error(handle) == 0
    assert hb.hcblasGetLastPath(handle) == "tc.h.grouped"
    got = dC.download()
    for i in np.random.default_rng(9).choice(b, 16, replace=False):
        sl = slice(i * n * n, (i + 1) * n * n)
        _, ref = O.gemm(O.COL, 0, 0, n, n, n, 1.0, A[sl], n, B[sl], n, 0.0,
                        np.zeros(n * n, np.float16), n)
        Ad = A[sl].astype(np.float64).reshape(n, n).T
        Bd = B[sl].astype(np.float64).reshape(n, n).T
        bound = (2.0 ** -11 + g(n, U32)) * np.linalg.norm(np.abs(Ad) @ np.abs(Bd))
        gv = O.view_c(got[sl].astype(np.float64), O.COL, n, n, n)
        assert np.linalg.norm(gv - ref) <= bound, i


@pytest.mark.parametrize("dtype", [np.float16, np.float32], ids=["f16", "f32_split"])
def test_c4b_grouped_4096_uneven_sampled(handle, dtype):
    import bench_cases
    name = "hgemm_grouped_4096" if dtype == np.float16 else "sgemm_grouped_4096"
    call, (dev, arr) = bench_cases.CASES[name](handle)
    call()
    assert hb.device_error(handle) == 0
    u_out = 2.0 ** -11 if dtype == np.float16 else 0.0
    worst = 0.0
    for i in np.random.default_rng(8).choice(len(arr), 16, replace=False):
        p = arr[int(i)]
        dA, dB, dC = dev[3 * int(i):3 * int(i) + 3]
        Ah = dA.download().astype(np.float64)
        Bh = dB.download().astype(np.float64)
        got = dC.download().astype(np.float64)
        _, ref = O.gemm(O.COL, p.transa, p.transb, p.m, p.n, p.k, 1.0, Ah, p.lda, Bh, p.ldb, 0.0,
                        np.zeros(p.m * p.n), p.m)
        Ad = op_a_dense(Ah, p.transa, p.m, p.k, p.lda)
        Bd = op_a_dense(Bh, 1 - p.transb, p.n, p.k, p.ldb).T  # op(B) = (op'(B^T))^T
        bound = (u_out + 2 * g(p.k, U32)) * np.linalg.norm(np.abs(Ad) @ np.abs(Bd))
        err = np.linalg.norm(O.view_c(got, O.COL, p.m, p.n, p.m) - ref)
        worst = max(worst, err / bound)
        assert err <= bound, (int(i), p.m, p.n, p.k, p.transa, p.transb, err, bound)
    print(f"C4b {np.dtype(dtype)} worst error / bound over 16 problems: {worst:.3g}")
