"""GPU parity of the tcgen05 tensor-core paths against the CPU oracle.

HGEMM (f16 storage, f32 accumulation in TMEM): every op(A) x op(B), ragged
shapes; tolerance
    ||C_gpu - C_ref||_F <= 2^-11 ||C_ref||_F + 2 gamma_{K+2}(f32) || |A||B| + |beta||C| ||_F
(one f16 rounding of each output plus f32 accumulation).

Split-BF16 SGEMM:
  * 6 products (three-way split, 24 significant bits): the plain FP32 bound
    2 gamma_{K+2}(f32) || |alpha||A||B| + |beta||C| ||_F;
  * 3 products (hi/lo, ~16 bits, lo*lo dropped): each operand carries a
    representation error <= 2^-17 |x| and the dropped term is <= 2^-18 |xy|,
    so the bound is (2^-15 + 2 gamma_{K+2}(f32)) || |alpha||A||B| ||_F +
    gamma(f32) |beta| ||C||_F.
Every call also checks the device error flag (a timed-out pipeline wait).
"""
import numpy as np
import pytest

import hcblas_b200 as hb
from oracle import oracle as O
from tests.test_gemm_gpu import error_bound, make_case, op_dense, TCH

pytestmark = pytest.mark.gpu

U32 = 2.0 ** -24


def g32(K):
    return (K + 2) * U32 / (1 - (K + 2) * U32)


def mag(order, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc):
    Ad = np.abs(op_dense(A, order, ta, M, K, lda, 0))
    Bd = np.abs(op_dense(B, order, tb, K, N, ldb, 0))
    ab = abs(alpha) * (Ad @ Bd)
    cc = abs(beta) * np.abs(O.view_c(C, order, M, N, ldc).astype(np.float64)) if beta else 0 * ab
    return ab, cc


def run(handle, kind, order, ta, tb, M, N, K, alpha, beta, rng, ld_align=8):
    # leading dimensions rounded to 8 elements: TMA needs 16-byte strides
    A, lda, B, ldb, C, ldc = make_case(rng, kind, order, ta, tb, M, N, K, ld_align=ld_align)
    dA, dB, dC = (hb.DeviceArray(handle, X) for X in (A, B, C))
    rc = hb.lib_gemm(handle, order, TCH[ta], TCH[tb], M, N, K, alpha, dA, lda, dB, ldb, beta, dC,
                     ldc)
    assert rc == 0
    assert hb.device_error(handle) == 0
    path = hb.hcblasGetLastPath(handle)
    got = dC.download()
    _, ref = O.gemm(order, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc)
    gv = O.view_c(got, order, M, N, ldc).astype(np.float64)
    err = np.linalg.norm(gv - ref)
    return err, ref, path, (A, lda, B, ldb, C, ldc)


HSHAPES = [(128, 128, 64), (256, 512, 128), (1000, 777, 333), (129, 65, 17), (3000, 2500, 200)]


@pytest.fixture
def pair_mode(handle, request):
    """tc_pair tuning knob: 0 = single-CTA kernels, 2 = CTA pairs
    (tcgen05 cta_group::2) for every shape; restored to auto afterwards."""
    assert hb.set_tuning(handle, "tc_pair", request.param) == 0
    yield request.param
    hb.set_tuning(handle, "tc_pair", 1)


@pytest.mark.parametrize("pair_mode", [0, 2], indirect=True)
@pytest.mark.parametrize("ta,tb", [(0, 0), (0, 1), (1, 0), (1, 1)])
def test_hgemm_tc_ops(handle, ta, tb, pair_mode):
    rng = np.random.default_rng(40 + 2 * ta + tb)
    for (M, N, K) in HSHAPES:
        for order in (O.COL, O.ROW):
            err, ref, path, (A, lda, B, ldb, C, ldc) = run(handle, "h", order, ta, tb, M, N, K,
                                                           1.0, 0.5, rng)
            assert path.startswith("tc.h"), path
            assert path.endswith(".pair") == (pair_mode == 2), path
            ab, cc = mag(order, ta, tb, M, N, K, 1.0, A, lda, B, ldb, 0.5, C, ldc)
            bound = 2.0 ** -11 * np.linalg.norm(ref) + 2 * g32(K) * np.linalg.norm(ab + cc)
            assert err <= bound, (M, N, K, order, ta, tb, err, bound, path)


def test_hgemm_odd_ld_falls_back_to_simt(handle):
    """Unpadded odd shapes (ld = 129, 333, ...) are not TMA-addressable."""
    rng = np.random.default_rng(8)
    for (M, N, K) in [(129, 65, 17), (1000, 777, 333)]:
        err, ref, path, (A, lda, B, ldb, C, ldc) = run(handle, "h", O.COL, 0, 0, M, N, K, 1.0,
                                                       0.5, rng, ld_align=1)
        assert path.startswith("simt.h"), path
        ab, cc = mag(O.COL, 0, 0, M, N, K, 1.0, A, lda, B, ldb, 0.5, C, ldc)
        assert err <= 2.0 ** -11 * np.linalg.norm(ref) + 2 * g32(K) * np.linalg.norm(ab + cc)


def test_hgemm_misaligned_falls_back(handle):
    rng = np.random.default_rng(3)
    M, N, K = 200, 100, 50
    A = rng.standard_normal((M + 1) * K).astype(np.float16)  # lda = M + 1: not 16-byte strided
    B = rng.standard_normal(K * N).astype(np.float16)
    C = rng.standard_normal(M * N).astype(np.float16)
    dA, dB, dC = (hb.DeviceArray(handle, X) for X in (A, B, C))
    assert hb.lib_gemm(handle, O.COL, "n", "n", M, N, K, 1.0, dA, M + 1, dB, K, 0.0, dC, M) == 0
    assert hb.hcblasGetLastPath(handle).startswith("simt.h")
    _, ref = O.gemm(O.COL, 0, 0, M, N, K, 1.0, A, M + 1, B, K, 0.0, C, M)
    got = O.view_c(dC.download(), O.COL, M, N, M).astype(np.float64)
    assert np.linalg.norm(got - ref) <= 2.0 ** -10 * np.linalg.norm(ref)


SSHAPES = [(256, 256, 256), (1000, 700, 300), (130, 200, 1000), (2048, 2048, 64)]


@pytest.mark.parametrize("pair_mode", [0, 2], indirect=True)
@pytest.mark.parametrize("terms", [3, 6])
@pytest.mark.parametrize("ta,tb", [(0, 0), (0, 1), (1, 0), (1, 1)])
def test_split_bf16_sgemm(handle, terms, ta, tb, pair_mode):
    rng = np.random.default_rng(100 + terms + 2 * ta + tb)
    assert hb.hcblasSetMathMode(handle, hb.HCBLAS_MATH_SPLIT_BF16, terms) == 0
    try:
        for (M, N, K) in SSHAPES:
            for order in (O.COL, O.ROW):
                alpha, beta = 1.25, -0.5
                err, ref, path, (A, lda, B, ldb, C, ldc) = run(handle, "s", order, ta, tb, M, N, K,
                                                               alpha, beta, rng)
                assert path.startswith(f"tc.split_bf16x{terms}"), path
                assert (".pair" in path) == (pair_mode == 2), path
                ab, cc = mag(order, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc)
                if terms == 6:
                    bound = 2 * g32(K) * np.linalg.norm(ab + cc)
                else:
                    bound = (2.0 ** -15 + 2 * g32(K)) * np.linalg.norm(ab) + \
                        2 * g32(K) * np.linalg.norm(cc)
                assert err <= bound, (terms, M, N, K, order, ta, tb, err, bound)
    finally:
        hb.hcblasSetMathMode(handle, hb.HCBLAS_MATH_NATIVE, 0)


def test_split_bf16_pack_paths_agree(handle):
    """The K-contiguous pack (packed f32x2 Veltkamp splits where the values
    allow, integer rounding elsewhere) and the MN-contiguous pack (integer
    rounding throughout) must produce the same bf16 planes: the same matrix
    stored both ways round (op N vs op T) gives bit-identical C, with zeros,
    subnormals, values near 2^-100 and 2^110 and beyond mixed in."""
    rng = np.random.default_rng(77)
    M, N, K = 192, 160, 200
    Ad = (rng.standard_normal((M, K)) * np.exp2(rng.integers(-30, 31, (M, K)))).astype(np.float32)
    special = np.array([0.0, -0.0, 1e-40, -3e-39, 2.0 ** -100, -(2.0 ** -101), 2.0 ** 109,
                        -(2.0 ** 110), 2.0 ** 115, 1.5 * 2.0 ** -99, 3.0, -7.0], np.float32)
    idx = rng.choice(M * K, 600, replace=False)
    Ad.reshape(-1)[idx] = special[rng.integers(0, special.size, idx.size)]
    Bd = rng.standard_normal((K, N)).astype(np.float32)
    A_n = np.asfortranarray(Ad).reshape(-1, order="F")    # column-major M x K, op N
    A_t = np.asfortranarray(Ad.T).reshape(-1, order="F")  # column-major K x M, op T
    B_n = np.asfortranarray(Bd).reshape(-1, order="F")
    assert hb.hcblasSetMathMode(handle, hb.HCBLAS_MATH_SPLIT_BF16, 6) == 0
    try:
        outs = []
        for A, ta, lda in ((A_n, "n", M), (A_t, "t", K)):
            dA, dB = hb.DeviceArray(handle, A), hb.DeviceArray(handle, B_n)
            dC = hb.DeviceArray(handle, np.zeros(M * N, np.float32))
            assert hb.lib_gemm(handle, O.COL, ta, "n", M, N, K, 1.0, dA, lda, dB, K, 0.0, dC,
                               M) == 0
            assert hb.device_error(handle) == 0
            outs.append(dC.download())
    finally:
        hb.hcblasSetMathMode(handle, hb.HCBLAS_MATH_NATIVE, 0)
    assert np.array_equal(outs[0].view(np.uint32), outs[1].view(np.uint32))


def test_split_bf16_accuracy_vs_plain(handle):
    """Report (and bound) the split-BF16 error next to plain FP32 at K = 2048,
    entries N(0,1) * 2^e, e ~ U{-8..8} per row of A / column of B."""
    rng = np.random.default_rng(2)
    M = N = 512
    K = 2048
    A = (rng.standard_normal((K, M)) * 2.0 ** rng.integers(-8, 9, M)[None, :]).astype(np.float32)
    B = (rng.standard_normal((K, N)) * 2.0 ** rng.integers(-8, 9, N)[None, :]).astype(np.float32)
    A = np.asfortranarray(A).reshape(-1, order="F")
    B = np.asfortranarray(B).reshape(-1, order="F")
    C = rng.standard_normal(M * N).astype(np.float32)
    _, ref = O.gemm(O.COL, 1, 0, M, N, K, 1.0, A, K, B, K, 1.0, C, M)
    errs = {}
    for mode, param in ((hb.HCBLAS_MATH_NATIVE, 0), (hb.HCBLAS_MATH_SPLIT_BF16, 3),
                        (hb.HCBLAS_MATH_SPLIT_BF16, 6)):
        hb.hcblasSetMathMode(handle, mode, param)
        dA, dB, dC = (hb.DeviceArray(handle, X) for X in (A, B, C))
        assert hb.lib_gemm(handle, O.COL, "t", "n", M, N, K, 1.0, dA, K, dB, K, 1.0, dC, M) == 0
        got = O.view_c(dC.download(), O.COL, M, N, M)
        errs[(mode, param)] = O.normwise_rel_error(got, ref)
    hb.hcblasSetMathMode(handle, hb.HCBLAS_MATH_NATIVE, 0)
    print("normwise errors:", errs)
    plain = errs[(0, 0)]
    # six products carry all 24 bits and promote TMEM chunks with IEEE adds:
    # no worse than plain FP32 SGEMM
    assert errs[(1, 6)] <= plain
    # three products are bounded by the 16-bit hi/lo representation
    assert errs[(1, 3)] <= 2.0 ** -16


# ------------------------------------------------------------ CGEMM 3M --
# T1 = Ar Br, T2 = Ai Bi, T3 = (Ar+Ai)(Br+Bi) each carry the split-BF16 error
# of one real product (6 terms: the FP32 bound; 3 terms: + 2^-15 relative)
# and the f32 sum Ar + Ai one more rounding; Re = T1 - T2, Im = T3 - T1 - T2.
# Elementwise bound on |dRe| + |dIm|:
#   (e + 4 u) |alpha| (|Ar||Br| + |Ai||Bi| + (|Ar|+|Ai|)(|Br|+|Bi|)) + 4u |beta||C|
# with e = 2 gamma_{K+2} (6 terms) or 2^-15 + 2 gamma_{K+2} (3 terms).

@pytest.mark.parametrize("terms", [3, 6])
@pytest.mark.parametrize("ta,tb", [(2, 0), (0, 0), (1, 2), (2, 1)])
def test_cgemm_split3m(handle, terms, ta, tb):
    rng = np.random.default_rng(300 + 10 * terms + 3 * ta + tb)
    assert hb.hcblasSetMathMode(handle, hb.HCBLAS_MATH_SPLIT_BF16, terms) == 0
    try:
        for order, (M, N, K) in ((O.COL, (300, 200, 500)), (O.ROW, (129, 77, 1000)),
                                 (O.COL, (64, 256, 33))):
            alpha, beta = (1 + 0.5j), (0.5 - 0.25j)
            A, lda, B, ldb, C, ldc = make_case(rng, "c", order, ta, tb, M, N, K)
            dA, dB, dC = (hb.DeviceArray(handle, X) for X in (A, B, C))
            rc = hb.lib_gemm(handle, order, TCH[ta], TCH[tb], M, N, K, alpha, dA, lda, dB, ldb,
                             beta, dC, ldc)
            assert rc == 0
            assert hb.device_error(handle) == 0
            assert hb.hcblasGetLastPath(handle) == f"tc.csplit3m_bf16x{terms}"
            got = dC.download()
            _, ref = O.gemm(order, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc)
            Ad = op_dense(A, order, ta, M, K, lda, 0)
            Bd = op_dense(B, order, tb, K, N, ldb, 0)
            ar, ai, br, bi = np.abs(Ad.real), np.abs(Ad.imag), np.abs(Bd.real), np.abs(Bd.imag)
            mag = ar @ br + ai @ bi + (ar + ai) @ (br + bi)
            e = 2 * g32(K) + (2.0 ** -15 if terms == 3 else 0.0)
            cc = np.abs(O.view_c(C, order, M, N, ldc))
            bound = (e + 4 * U32) * abs(alpha) * np.linalg.norm(mag) + \
                4 * U32 * abs(beta) * np.linalg.norm(cc)
            err = np.linalg.norm(O.view_c(got, order, M, N, ldc).astype(np.complex128) - ref)
            assert err <= bound, (terms, order, ta, tb, M, N, K, err, bound)
    finally:
        hb.hcblasSetMathMode(handle, hb.HCBLAS_MATH_NATIVE, 0)


@pytest.mark.parametrize("kind,M,ldc", [("h", 18, 24), ("h", 50, 56), ("h", 200, 208),
                                        ("s", 18, 20), ("s", 45, 48)])
def test_tc_epilogue_keeps_ld_padding(handle, kind, M, ldc):
    """C rows between M and ldc are never written (tensor stores are used only
    where a column is a whole number of 16-byte chunks), on the single-problem
    tensor-core kernel (HGEMM; split-BF16 SGEMM) and on the grouped kernel."""
    rng = np.random.default_rng(M + ldc)
    N, K = 70, 96
    dt = np.float16 if kind == "h" else np.float32
    lda = -(-M // 8) * 8  # a leading dimension TMA can address
    A = rng.uniform(-1, 1, lda * K).astype(dt)
    B = rng.uniform(-1, 1, K * N).astype(dt)
    C = rng.uniform(-1, 1, ldc * N).astype(dt)
    mode = hb.HCBLAS_MATH_NATIVE if kind == "h" else hb.HCBLAS_MATH_SPLIT_BF16
    assert hb.hcblasSetMathMode(handle, mode, 6 if kind == "s" else 0) == 0
    try:
        dA, dB, dC = (hb.DeviceArray(handle, X) for X in (A, B, C))
        assert hb.lib_gemm(handle, O.COL, "n", "n", M, N, K, 1.0, dA, lda, dB, K, 0.5, dC,
                           ldc) == 0
        assert hb.device_error(handle) == 0
        assert hb.hcblasGetLastPath(handle).startswith("tc."), hb.hcblasGetLastPath(handle)
        got = dC.download()
    finally:
        hb.hcblasSetMathMode(handle, hb.HCBLAS_MATH_NATIVE, 0)
    assert np.array_equal(got.reshape(N, ldc)[:, M:], C.reshape(N, ldc)[:, M:])
    _, ref = O.gemm(O.COL, 0, 0, M, N, K, 1.0, A, lda, B, K, 0.5, C, ldc)
    tol = 2e-3 if kind == "h" else 1e-5
    assert O.normwise_rel_error(O.view_c(got, O.COL, M, N, ldc).astype(np.float64), ref) < tol
    if kind == "h":  # the grouped kernel on the same problem
        dC.upload(C)
        p = hb.GemmProblem(0, 0, M, N, K, dA.ptr, lda, dB.ptr, K, dC.ptr, ldc)
        assert hb.hgemm_grouped(handle, [p], 1.0, 0.5) == 0
        assert hb.hcblasGetLastPath(handle) == "tc.h.grouped"
        got = dC.download()
        assert np.array_equal(got.reshape(N, ldc)[:, M:], C.reshape(N, ldc)[:, M:])
        assert O.normwise_rel_error(O.view_c(got, O.COL, M, N, ldc).astype(np.float64),
                                    ref) < tol
