"""Batched GEMMs on the persistent grouped tensor-core kernels.

* Pointer-array HGEMM batches (hcblasHgemmBatched, and the class-API form
  with row-major order, offsets and batch offsets): the problem table is built
  on the GPU from the device-resident pointer arrays (tensor-map addresses
  replaced in place), the grouped kernel walks every problem's tiles, and
  entries whose A or B TMA cannot address are computed by the CUDA-core pass.
* Pointer-array and strided SGEMM batches under HCBLAS_MATH_SPLIT_BF16: one
  pack launch and one grouped GEMM launch for the whole batch, the operand
  and C pointers of a pointer-array batch patched in on the GPU.
Bounds per problem: f16 C, f32 accumulation
    ||C - C_ref|| <= 2^-11 ||C_ref|| + 2 gamma_{K+2}(f32) || |alpha||A||B| + |beta||C| ||;
split-BF16 with 6 products: 2 gamma_{K+2}(f32) || |alpha||A||B| + |beta||C| ||.
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


def ptr_array(handle, ptrs):
    return hb.DeviceArray(handle, np.array(ptrs, dtype=np.uint64))


def make_batch(handle, rng, dt, batch, ta, tb, M, N, K, lda, ldb, ldc, shift=()):
    """Separate device allocations per problem; entries in `shift` start one
    element past their allocation (2 or 4 bytes: not 16-byte aligned)."""
    host, dev, pa, pb, pc = [], [], [], [], []
    esz = np.dtype(dt).itemsize
    for i in range(batch):
        A = rng.uniform(-1, 1, lda * (K if ta == 0 else M) + 1).astype(dt)
        B = rng.uniform(-1, 1, ldb * (N if tb == 0 else K) + 1).astype(dt)
        C = rng.uniform(-1, 1, ldc * N + 1).astype(dt)
        dA, dB, dC = (hb.DeviceArray(handle, X) for X in (A, B, C))
        o = 1 if i in shift else 0
        host.append((A[o:], B[o:], C[o:]))
        dev.append((dA, dB, dC, o))
        pa.append(dA.ptr + o * esz)
        pb.append(dB.ptr + o * esz)
        pc.append(dC.ptr + o * esz)
    return host, dev, ptr_array(handle, pa), ptr_array(handle, pb), ptr_array(handle, pc)


def check_f16(host, dev, ta, tb, M, N, K, lda, ldb, ldc, alpha, beta, sample):
    for i in sample:
        A, B, C = host[i]
        dA, dB, dC, o = dev[i]
        got = dC.download()[o:]
        _, ref = O.gemm(O.COL, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc)
        gv = O.view_c(got, O.COL, M, N, ldc).astype(np.float64)
        Ad, Bd = np.abs(op_dense(A, ta, M, K, lda)), np.abs(op_dense(B, tb, K, N, ldb))
        cc = abs(beta) * np.abs(O.view_c(C, O.COL, M, N, ldc).astype(np.float64))
        bound = 2.0 ** -11 * np.linalg.norm(ref) + \
            2 * g32(K) * np.linalg.norm(abs(alpha) * (Ad @ Bd) + cc)
        assert np.linalg.norm(gv - ref) <= bound, (i, np.linalg.norm(gv - ref), bound)
        # the leading-dimension padding of C is untouched
        assert np.array_equal(got[: ldc * N].reshape(N, ldc)[:, M:],
                              C[: ldc * N].reshape(N, ldc)[:, M:])


def test_hgemm_batched_ptr_512x128(handle):
    """The uniform batch of the benchmark (512 x 128^3, f16) through
    hcblasHgemmBatched: one table build, one grouped launch, one CUDA-core
    pass for flagged entries (none here)."""
    rng = np.random.default_rng(21)
    n, b = 128, 512
    host, dev, pA, pB, pC = make_batch(handle, rng, np.float16, b, 0, 0, n, n, n, n, n, n)
    launches0 = hb.kernel_launch_count()
    assert hb.gemm_batched(handle, 0, 0, n, n, n, 1.0, pA.ptr, n, pB.ptr, n, 0.0, pC.ptr, n, b,
                           np.float16) == 0
    assert hb.device_error(handle) == 0
    assert hb.kernel_launch_count() - launches0 == 3
    assert hb.hcblasGetLastPath(handle) == "tc.h.grouped.ptr"
    check_f16(host, dev, 0, 0, n, n, n, n, n, n, 1.0, 0.0,
              np.random.default_rng(9).choice(b, 16, replace=False))


@pytest.mark.parametrize("ta,tb,ldc_pad", [(0, 1, 0), (1, 0, 3), (1, 1, 8)])
def test_hgemm_batched_ptr_misaligned_and_beta(handle, ta, tb, ldc_pad):
    """Some entries start 2 bytes past a 16-byte boundary (the CUDA-core pass
    computes them); beta != 0 reads C by TMA when ldc allows it, by plain
    loads when it does not; N = 72 takes two tile widths' worth of padding
    decisions (64 + 8)."""
    rng = np.random.default_rng(22 + ta + 2 * tb)
    M, N, K, b = 200, 72, 136, 24
    lda = (M if ta == 0 else K) + 8
    ldb = (K if tb == 0 else N) + 16
    ldc = M + ldc_pad
    shift = {3, 7, 19}
    host, dev, pA, pB, pC = make_batch(handle, rng, np.float16, b, ta, tb, M, N, K, lda, ldb,
                                       ldc, shift)
    assert hb.gemm_batched(handle, ta, tb, M, N, K, 1.25, pA.ptr, lda, pB.ptr, ldb, -0.5, pC.ptr,
                           ldc, b, np.float16) == 0
    assert hb.device_error(handle) == 0
    assert hb.hcblasGetLastPath(handle) == "tc.h.grouped.ptr"
    check_f16(host, dev, ta, tb, M, N, K, lda, ldb, ldc, 1.25, -0.5, range(b))


def test_hgemm_batched_ptr_class_api_row_major_offsets(handle):
    """hcblasLibGemmBatched (dtype 4 = H), row-major, element offsets and
    batch offsets: matrix i is X[i] + xOffset + i * X_batchOffset."""
    rng = np.random.default_rng(23)
    M, N, K, b = 96, 160, 80, 6
    L = hb.lib()
    # row-major A (M x K, lda = K), B^T (op B = T: B is N x K, ldb = K), C (M x N, ldc = N)
    aoff, boff, coff = 8, 16, 24           # keep A/B 16-byte aligned
    A = rng.uniform(-1, 1, aoff + M * K * b).astype(np.float16)
    B = rng.uniform(-1, 1, boff + N * K * b).astype(np.float16)
    C = rng.uniform(-1, 1, coff + M * N * b).astype(np.float16)
    dA, dB, dC = (hb.DeviceArray(handle, X) for X in (A, B, C))
    pA, pB, pC = (ptr_array(handle, [d.ptr] * b) for d in (dA, dB, dC))
    one = np.array([1.0], np.float16).view(np.uint16)
    half = np.array([0.5], np.float16).view(np.uint16)
    rc = L.hcblasLibGemmBatched(handle, 4, 0, b"n", b"t", M, N, K, one.ctypes.data, pA.ptr, K,
                                M * K, pB.ptr, K, N * K, half.ctypes.data, pC.ptr, N, M * N,
                                aoff, boff, coff, b)
    assert rc == 0
    assert hb.device_error(handle) == 0
    assert hb.hcblasGetLastPath(handle) == "tc.h.grouped.ptr"
    got = dC.download()
    for i in range(b):
        _, ref = O.gemm(O.ROW, 0, 1, M, N, K, 1.0, A[aoff + i * M * K:], K,
                        B[boff + i * N * K:], K, 0.5, C[coff + i * M * N:], N)
        gv = O.view_c(got[coff + i * M * N:], O.ROW, M, N, N).astype(np.float64)
        Ad = np.abs(A[aoff + i * M * K: aoff + (i + 1) * M * K].reshape(M, K).astype(np.float64))
        Bd = np.abs(B[boff + i * N * K: boff + (i + 1) * N * K].reshape(N, K).astype(np.float64))
        cc = 0.5 * np.abs(C[coff + i * M * N: coff + (i + 1) * M * N].reshape(M, N))
        bound = 2.0 ** -11 * np.linalg.norm(ref) + 2 * g32(K) * np.linalg.norm(Ad @ Bd.T + cc)
        assert np.linalg.norm(gv - ref) <= bound, i


def split_bound(A, B, C, ta, tb, M, N, K, lda, ldb, ldc, alpha, beta):
    Ad, Bd = np.abs(op_dense(A, ta, M, K, lda)), np.abs(op_dense(B, tb, K, N, ldb))
    cc = abs(beta) * np.abs(O.view_c(C, O.COL, M, N, ldc).astype(np.float64))
    return 2 * g32(K) * np.linalg.norm(abs(alpha) * (Ad @ Bd) + cc)


def test_sgemm_batched_ptr_split(handle):
    rng = np.random.default_rng(24)
    M, N, K, b = 150, 130, 300, 40
    ta, tb = 1, 0
    lda, ldb, ldc = K + 3, K + 1, M + 2
    host, dev, pA, pB, pC = make_batch(handle, rng, np.float32, b, ta, tb, M, N, K, lda, ldb,
                                       ldc, shift={5})
    assert hb.hcblasSetMathMode(handle, hb.HCBLAS_MATH_SPLIT_BF16, 6) == 0
    try:
        launches0 = hb.kernel_launch_count()
        assert hb.gemm_batched(handle, ta, tb, M, N, K, 0.75, pA.ptr, lda, pB.ptr, ldb, 0.25,
                               pC.ptr, ldc, b, np.float32) == 0
        assert hb.device_error(handle) == 0
        assert hb.hcblasGetLastPath(handle) == "tc.s.grouped_split_bf16x6"
        assert hb.kernel_launch_count() - launches0 == 3  # patch, pack, grouped GEMM
    finally:
        hb.hcblasSetMathMode(handle, hb.HCBLAS_MATH_NATIVE, 0)
    for i in range(b):
        A, B, C = host[i]
        dA, dB, dC, o = dev[i]
        got = dC.download()[o:]
        _, ref = O.gemm(O.COL, ta, tb, M, N, K, 0.75, A, lda, B, ldb, 0.25, C, ldc)
        gv = O.view_c(got, O.COL, M, N, ldc).astype(np.float64)
        assert np.linalg.norm(gv - ref) <= split_bound(A, B, C, ta, tb, M, N, K, lda, ldb, ldc,
                                                       0.75, 0.25), i


def test_sgemm_strided_split_one_grouped_launch(handle):
    rng = np.random.default_rng(25)
    M, N, K, b = 128, 128, 128, 64
    sA, sB, sC = M * K + 4, K * N + 8, M * N + 12
    A = rng.uniform(-1, 1, sA * b).astype(np.float32)
    B = rng.uniform(-1, 1, sB * b).astype(np.float32)
    C = rng.uniform(-1, 1, sC * b).astype(np.float32)
    dA, dB, dC = (hb.DeviceArray(handle, X) for X in (A, B, C))
    assert hb.hcblasSetMathMode(handle, hb.HCBLAS_MATH_SPLIT_BF16, 6) == 0
    try:
        launches0 = hb.kernel_launch_count()
        assert hb.gemm_strided_batched(handle, 0, 1, M, N, K, 1.0, dA, M, sA, dB, N, sB, 0.5, dC,
                                       M, sC, b) == 0
        assert hb.device_error(handle) == 0
        assert hb.hcblasGetLastPath(handle) == "tc.s.grouped_split_bf16x6"
        assert hb.kernel_launch_count() - launches0 == 2  # pack, grouped GEMM
    finally:
        hb.hcblasSetMathMode(handle, hb.HCBLAS_MATH_NATIVE, 0)
    got = dC.download()
    for i in np.random.default_rng(3).choice(b, 12, replace=False):
        Ai, Bi, Ci = A[i * sA:(i + 1) * sA], B[i * sB:(i + 1) * sB], C[i * sC:(i + 1) * sC]
        _, ref = O.gemm(O.COL, 0, 1, M, N, K, 1.0, Ai, M, Bi, N, 0.5, Ci, M)
        gv = O.view_c(got[i * sC:], O.COL, M, N, M).astype(np.float64)
        assert np.linalg.norm(gv - ref) <= split_bound(Ai, Bi, Ci, 0, 1, M, N, K, M, N, M, 1.0,
                                                       0.5), i
        assert np.array_equal(got[i * sC + M * N:(i + 1) * sC], Ci[M * N:])
