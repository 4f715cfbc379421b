"""GPU parity of the plain GEMM paths against the CPU oracle and the golden
fixtures, through the C ABI (libhcblas.so via ctypes).

Tolerances (stated per test): integer-valued recipes must match exactly, as
the reference's EXPECT_EQ tests do (test/unit/hcblas_dgemm.cpp:258); float
results must satisfy the normwise forward-error bound of a plain GEMM,
    ||C_gpu - C_ref||_F <= gamma_{K+2} * || |alpha| |op(A)| |op(B)| + |beta| |C| ||_F,
gamma_n = n u / (1 - n u), u the unit roundoff of the compute type (x4 for
complex arithmetic), plus u_storage * ||C_ref||_F for FP16 outputs.
"""
import ctypes
import os

import numpy as np
import pytest

import hcblas_b200 as hb
from oracle import oracle as O
from tests.conftest import GOLDEN

pytestmark = pytest.mark.gpu

NP = {"s": np.float32, "d": np.float64, "c": np.complex64, "z": np.complex128, "h": np.float16}
UNIT = {"s": 2.0 ** -24, "d": 2.0 ** -53, "c": 2.0 ** -24, "z": 2.0 ** -53, "h": 2.0 ** -24}
TCH = {0: "n", 1: "t", 2: "c"}


def gamma(kind, K):
    u = UNIT[kind]
    g = (K + 2) * u / (1 - (K + 2) * u)
    return g * (4 if kind in "cz" else 1)


def op_dense(X, order, trans, rows, cols, ld, off):
    """op(X) as a dense (rows x cols) float64/complex128 array."""
    X = np.asarray(X).reshape(-1)
    r0, c0 = (rows, cols) if trans == 0 else (cols, rows)
    V = O.view_c(X, order, r0, c0, ld, off).astype(np.complex128 if np.iscomplexobj(X) else np.float64)
    if trans == 0:
        return V
    return V.T.conj() if trans == 2 else V.T


def error_bound(kind, order, ta, tb, M, N, K, alpha, A, lda, ao, B, ldb, bo, beta, C, ldc, co, ref):
    mag = np.zeros((M, N))
    if abs(alpha) != 0:  # alpha == 0: A and B are not referenced
        Ad = np.abs(op_dense(A, order, ta, M, K, lda, ao))
        Bd = np.abs(op_dense(B, order, tb, K, N, ldb, bo))
        mag = mag + abs(alpha) * (Ad @ Bd)
    if abs(beta) != 0:  # beta == 0: C is not referenced
        mag = mag + abs(beta) * np.abs(O.view_c(C, order, M, N, ldc, co).astype(np.complex128))
    bound = gamma(kind, K) * np.linalg.norm(mag)
    if kind == "h":
        bound += 2.0 ** -11 * np.linalg.norm(ref) + 2.0 ** -24 * np.linalg.norm(mag)
    return bound


def rand_op(rng, kind, n):
    v = rng.standard_normal(n)
    if kind in "cz":
        v = v + 1j * rng.standard_normal(n)
    return v.astype(NP[kind])


def make_case(rng, kind, order, ta, tb, M, N, K, pad=0, offs=(0, 0, 0), ld_align=1):
    """Random operands for one GEMM; ld = rows (+pad), rounded up to ld_align."""
    ar, ac = (M, K) if ta == 0 else (K, M)
    br, bc = (K, N) if tb == 0 else (N, K)
    up = lambda v: -(-v // ld_align) * ld_align
    lda = up((ar if order == O.COL else ac) + pad)
    ldb = up((br if order == O.COL else bc) + pad)
    ldc = up((M if order == O.COL else N) + pad)
    na = offs[0] + lda * (ac if order == O.COL else ar)
    nb = offs[1] + ldb * (bc if order == O.COL else br)
    nc = offs[2] + ldc * (N if order == O.COL else M)
    return (rand_op(rng, kind, na), lda, rand_op(rng, kind, nb), ldb, rand_op(rng, kind, nc), ldc)


def run_and_check(handle, kind, order, ta, tb, M, N, K, alpha, beta, A, lda, B, ldb, C, ldc,
                  offs=(0, 0, 0), expect_path=None):
    dA, dB, dC = (hb.DeviceArray(handle, X) for X in (A, B, C))
    rc = hb.lib_gemm(handle, order, TCH[ta], TCH[tb], M, N, K, alpha, dA, lda, dB, ldb, beta, dC,
                     ldc, *offs)
    assert rc == 0, f"hcblasLib gemm returned {rc}"
    got = dC.download()
    path = hb.hcblasGetLastPath(handle)
    if expect_path:
        assert path.startswith(expect_path), path
    ref_c, ref = O.gemm(order, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, *offs)
    # entries outside the M x N window are untouched
    mask = np.ones(C.size, bool)
    view_idx = O.view_c(np.arange(C.size), order, M, N, ldc, offs[2])
    mask[view_idx.reshape(-1)] = False
    assert np.array_equal(got[mask], C[mask])
    gv = O.view_c(got, order, M, N, ldc, offs[2])
    err = np.linalg.norm((gv.astype(ref.dtype) - ref).reshape(-1))
    bound = error_bound(kind, order, ta, tb, M, N, K, alpha, A, lda, offs[0], B, ldb, offs[1],
                        beta, C, ldc, offs[2], ref)
    assert err <= bound, (kind, order, ta, tb, M, N, K, err, bound, path)
    return err / max(np.linalg.norm(ref), 1e-300), path


# ------------------------------------------------------------ golden chains --

@pytest.mark.parametrize("kind", "sdcz")
def test_int_chain_exact(handle, kind):
    """Integer recipes of the reference tests, replayed on one device C buffer."""
    f = np.load(os.path.join(GOLDEN, f"int_chain_{kind}.npz"))
    M, N, K = int(f["M"]), int(f["N"]), int(f["K"])
    dA, dB, dC = (hb.DeviceArray(handle, f[x]) for x in ("A", "B", "C"))
    for step, expect in zip(f["steps"], f["states"]):
        order, ta, tb, lda, ldb, ldc, ar, ai, br, bi = [int(v) for v in step]
        alpha = complex(ar, ai) if kind in "cz" else float(ar)
        beta = complex(br, bi) if kind in "cz" else float(br)
        rc = hb.lib_gemm(handle, order, TCH[ta], TCH[tb], M, N, K, alpha, dA, lda, dB, ldb,
                         beta, dC, ldc)
        assert rc == 0
        got = dC.download()
        assert np.array_equal(got, expect), (step.tolist(), hb.hcblasGetLastPath(handle))


def test_float_cases_vs_openblas(handle):
    """Seeded float cases with offsets / padded ld / NaN C under beta = 0."""
    f = np.load(os.path.join(GOLDEN, "float_cases.npz"))
    for row in f["meta"]:
        idx, kind_i, order, ta, tb, M, N, K, lda, ldb, ldc, ao, bo, co = [int(v) for v in row]
        kind = "sdcz"[kind_i]
        key = f"c{idx:03d}"
        A, B, C, out = f[key + "_A"], f[key + "_B"], f[key + "_C"], f[key + "_out"]
        alpha, beta = complex(f[key + "_alpha"][0]), complex(f[key + "_beta"][0])
        if kind in "sd":
            alpha, beta = alpha.real, beta.real
        dA, dB, dC = (hb.DeviceArray(handle, X) for X in (A, B, C))
        rc = hb.lib_gemm(handle, order, TCH[ta], TCH[tb], M, N, K, alpha, dA, lda, dB, ldb, beta,
                         dC, ldc, ao, bo, co)
        assert rc == 0
        got = dC.download()
        gv = O.view_c(got, order, M, N, ldc, co)
        ov = O.view_c(out, order, M, N, ldc, co)
        assert np.all(np.isfinite(gv))
        err = np.linalg.norm((gv.astype(np.complex128) - ov).reshape(-1))
        assert err <= 2 * gamma(kind, K) * np.linalg.norm(np.abs(ov).reshape(-1)) * 4, (key, err)


def test_capi_ones_and_destroy(built_lib):
    """test/unit-api/test-blas.cpp:1851-1937 through the C API."""
    f = np.load(os.path.join(GOLDEN, "capi_ones.npz"))
    M, N, K = int(f["M"]), int(f["N"]), int(f["K"])
    s, h = hb.hcblasCreate(0)
    assert s == hb.HCBLAS_STATUS_SUCCESS
    L = hb.lib()
    dA = hb.am_alloc(4 * M * K)
    dB = hb.am_alloc(4 * K * N)
    dC = hb.am_alloc(4 * M * N)
    A, B, C = f["A"], f["B"], f["C"]
    assert hb.hcblasSetMatrix(h, M, K, 4, A.ctypes.data, 1, dA, 1) == 0
    assert hb.hcblasSetMatrix(h, K, N, 4, B.ctypes.data, 1, dB, 1) == 0
    assert hb.hcblasSetMatrix(h, M, N, 4, C.ctypes.data, 1, dC, 1) == 0
    al = np.array([2.0], np.float32)
    be = np.array([2.0], np.float32)
    s = L.hcblasSgemm(h, 0, 0, M, N, K, al.ctypes.data, dA, M, dB, K, be.ctypes.data, dC, M)
    assert s == hb.HCBLAS_STATUS_SUCCESS
    out = np.zeros(M * N, np.float32)
    assert hb.hcblasGetMatrix(h, M, N, 4, dC, 1, out.ctypes.data, 1) == 0
    assert np.array_equal(out, f["out"])
    assert hb.hcblasDestroy(h) == hb.HCBLAS_STATUS_SUCCESS
    # a destroyed handle reports NOT_INITIALIZED (test-blas.cpp:1922-1926)
    s = L.hcblasSgemm(None, 0, 0, M, N, K, al.ctypes.data, dA, M, dB, K, be.ctypes.data, dC, M)
    assert s == hb.HCBLAS_STATUS_NOT_INITIALIZED
    for p in (dA, dB, dC):
        hb.am_free(p)


def test_status_codes(handle):
    """Status KATs of test/unit/hcblas_sgemm.cpp:34-195 through the C API."""
    L = hb.lib()
    M, N, K = 189, 9, 19
    # every operand buffer holds 200 x 200 floats: enough for any op with ld = 200
    dA, dB, dC = (hb.am_alloc(4 * 200 * 200) for _ in range(3))
    one = np.ones(1, np.float32)
    p1 = one.ctypes.data
    S = hb.HCBLAS_STATUS_SUCCESS
    for ta in (0, 1, 2):
        for tb in (0, 1, 2):
            assert L.hcblasSgemm(handle, ta, tb, M, N, K, p1, dA, 200, dB, 200, p1, dC, 200) == S
    E = hb.HCBLAS_STATUS_EXECUTION_FAILED
    assert L.hcblasSgemm(handle, 0, 0, M, N, K, p1, None, M, dB, K, p1, dC, M) == E
    assert L.hcblasSgemm(handle, 0, 0, M, N, K, p1, dA, M, None, K, p1, dC, M) == E
    assert L.hcblasSgemm(handle, 0, 0, M, N, K, p1, dA, M, dB, K, p1, None, M) == E
    assert L.hcblasSgemm(handle, 0, 0, 0, N, K, p1, dA, M, dB, K, p1, dC, M) == E
    assert L.hcblasSgemm(handle, 0, 0, M, 0, K, p1, dA, M, dB, K, p1, dC, M) == E
    assert L.hcblasSgemm(handle, 0, 0, M, N, 0, p1, dA, M, dB, K, p1, dC, M) == E
    V = hb.HCBLAS_STATUS_INVALID_VALUE
    assert L.hcblasSgemm(handle, 0, 0, -1, N, K, p1, dA, M, dB, K, p1, dC, M) == V
    assert L.hcblasDgemm(handle, 0, 0, M, -2, K, p1, dA, M, dB, K, p1, dC, M) == V
    assert L.hcblasSgemmBatched(handle, 0, 0, M, N, K, p1, dA, M, dB, K, p1, dC, M, -1) == V
    # class API: HCBLAS_INVALID (-1) for the same quick-return cases
    assert L.hcblasLibSgemm(handle, 1, b"n", b"n", M, N, K, p1, None, M, dB, K, p1, dC, M, 0, 0, 0) == -1
    assert L.hcblasLibSgemm(handle, 0, b"t", b"n", M, N, 0, p1, dA, M, dB, K, p1, dC, M, 0, 0, 0) == -1
    assert L.hcblasLibSgemm(handle, 0, b"t", b"t", M, N, K, p1, dA, M, dB, K, p1, dC, M, 0, 0, 0) == 0
    for p in (dA, dB, dC):
        hb.am_free(p)


# ------------------------------------------------------ oracle parity sweep --

SHAPES = [(1, 1, 1), (3, 5, 7), (17, 13, 11), (64, 64, 64), (65, 63, 129), (128, 128, 8),
          (129, 257, 33), (200, 70, 300)]


@pytest.mark.parametrize("kind", "sdczh")
def test_sweep_shapes_ops_orders(handle, kind):
    rng = np.random.default_rng(1000 + "sdczh".index(kind))
    ops = (0, 1, 2) if kind in "cz" else (0, 1)
    alpha = (1.25 - 0.5j) if kind in "cz" else 1.25
    beta = (0.5 + 0.25j) if kind in "cz" else -0.75
    if kind == "h":
        alpha, beta = 1.0, 0.5
    for si, (M, N, K) in enumerate(SHAPES):
        for order in (O.COL, O.ROW):
            for ta in ops:
                for tb in ops:
                    pad = (si + ta + tb) % 3
                    offs = ((si * 3) % 5, (si * 7) % 4, (si + order) % 3)
                    A, lda, B, ldb, C, ldc = make_case(rng, kind, order, ta, tb, M, N, K, pad, offs)
                    run_and_check(handle, kind, order, ta, tb, M, N, K, alpha, beta, A, lda, B,
                                  ldb, C, ldc, offs)


@pytest.mark.parametrize("kind", "sdczh")
def test_large_tile_ragged(handle, kind):
    """Shapes that take the large-tile kernels, with ragged edges."""
    rng = np.random.default_rng(77)
    M, N, K = (1537, 1409, 77) if kind not in "cz" else (1031, 1223, 45)
    for order, ta, tb in ((O.COL, 0, 0), (O.COL, 1, 1), (O.ROW, 0, 1), (O.COL, 1, 0)):
        A, lda, B, ldb, C, ldc = make_case(rng, kind, order, ta, tb, M, N, K)
        run_and_check(handle, kind, order, ta, tb, M, N, K, 1.0, 0.5, A, lda, B, ldb, C, ldc)


@pytest.mark.parametrize("kind", "sdcz")
def test_alpha_zero_and_beta_zero(handle, kind):
    rng = np.random.default_rng(5)
    M, N, K = 70, 33, 19
    A, lda, B, ldb, C, ldc = make_case(rng, kind, O.COL, 0, 1, M, N, K)
    # alpha = 0: C := beta * C, A and B never read (NaN A must not leak)
    A_nan = A.copy()
    A_nan[:] = np.nan
    run_and_check(handle, kind, O.COL, 0, 1, M, N, K, 0.0, 0.5, A_nan, lda, B, ldb, C, ldc,
                  expect_path="scale")
    # beta = 0: C is not read (NaN C must not leak)
    C_nan = C.copy()
    C_nan[:] = np.nan
    run_and_check(handle, kind, O.COL, 0, 1, M, N, K, 1.5, 0.0, A, lda, B, ldb, C_nan, ldc)
    # alpha = beta = 0: zeros
    run_and_check(handle, kind, O.COL, 0, 1, M, N, K, 0.0, 0.0, A_nan, lda, B, ldb, C_nan, ldc)


def test_sgemm_reference_recipe_l2(handle):
    """test/unit/hcblas_sgemm.cpp:222-261 recipe (U[0,2), rand_r seed 100),
    shape classes vvsmall..regular (4, 48, 777, 1133), L2 error < 1e-5."""
    f = np.load(os.path.join(GOLDEN, "sgemm_recipe.npz"))
    for i, s in enumerate(f["shapes"]):
        M = N = K = int(s)
        al, be = (float(v) for v in f[f"s{i}_ab"])
        dA, dB, dC = (hb.DeviceArray(handle, f[f"s{i}_{x}"]) for x in "ABC")
        assert hb.lib_gemm(handle, O.COL, "n", "n", M, N, K, al, dA, M, dB, K, be, dC, M) == 0
        assert O.compare_l2fe(f[f"s{i}_out"], dC.download()) < float(f["tolerance"])
    rr = O.RandR(100)
    for s in (777, 1133):
        M = N = K = s
        al = float(np.float32(rr.next()) / np.float32(O.RandR.RAND_MAX * 1.172))
        be = float(np.float32(rr.next()) / np.float32(O.RandR.RAND_MAX * 3.414))
        A, B, C = rr.uniform02(M * K), rr.uniform02(K * N), rr.uniform02(M * N)
        for order, ta, tb in ((O.COL, 0, 0), (O.COL, 0, 1), (O.COL, 1, 0), (O.COL, 1, 1),
                              (O.ROW, 0, 0)):
            dA, dB, dC = (hb.DeviceArray(handle, X) for X in (A, B, C))
            assert hb.lib_gemm(handle, order, TCH[ta], TCH[tb], M, N, K, al, dA, M, dB, K, be,
                               dC, M) == 0
            ref, _ = O.gemm(order, ta, tb, M, N, K, al, A, M, B, K, be, C, M, want_ref=False)
            assert O.compare_l2fe(ref, dC.download()) < 1e-5


# -------------------------------------------------------------- batched --

def _ptr_array(handle, ptrs):
    arr = np.array(ptrs, dtype=np.uint64)
    return hb.DeviceArray(handle, arr)


@pytest.mark.parametrize("kind", "sdcz")
def test_pointer_array_batched_exact(handle, kind):
    """test/unit/hcblas_sgemm.cpp:1612-1729: 64 x (189x9x19), integer data, exact."""
    M, N, K, batch = 189, 9, 19, 64
    rr = O.RandR(100)
    dt = NP[kind]
    As, Bs, Cs = [], [], []
    for _ in range(batch):
        if kind in "cz":
            A = (rr.ints(M * K, 10) + 1j * rr.ints(M * K, 20)).astype(dt)
            B = (rr.ints(K * N, 15) + 1j * rr.ints(K * N, 25)).astype(dt)
            C = (rr.ints(M * N, 18) + 1j * rr.ints(M * N, 28)).astype(dt)
        else:
            A = rr.ints(M * K, 100).astype(dt)
            B = rr.ints(K * N, 15).astype(dt)
            C = rr.ints(M * N, 25).astype(dt)
        As.append(A)
        Bs.append(B)
        Cs.append(C)
    dAs = [hb.DeviceArray(handle, x) for x in As]
    dBs = [hb.DeviceArray(handle, x) for x in Bs]
    dCs = [hb.DeviceArray(handle, x) for x in Cs]
    pA = _ptr_array(handle, [d.ptr for d in dAs])
    pB = _ptr_array(handle, [d.ptr for d in dBs])
    pC = _ptr_array(handle, [d.ptr for d in dCs])
    alpha = (1 + 1j) if kind in "cz" else 1.0
    beta = (1 + 1j) if kind in "cz" else 1.0
    s = hb.gemm_batched(handle, 0, 0, M, N, K, alpha, pA.ptr, M, pB.ptr, K, beta, pC.ptr, M,
                        batch, dt)
    assert s == hb.HCBLAS_STATUS_SUCCESS
    for i in range(batch):
        exp, _ = O.gemm(O.COL, 0, 0, M, N, K, alpha, As[i], M, Bs[i], K, beta, Cs[i], M,
                        want_ref=False)
        assert np.array_equal(dCs[i].download(), exp), i


@pytest.mark.parametrize("kind", "sdczh")
def test_strided_batched_vs_oracle(handle, kind):
    rng = np.random.default_rng(31)
    M, N, K, batch = 70, 45, 33, 9
    dt = NP[kind]
    sA, sB, sC = M * K + 5, K * N + 3, M * N + 7
    A = rand_op(rng, kind, sA * batch)
    B = rand_op(rng, kind, sB * batch)
    C = rand_op(rng, kind, sC * batch)
    dA, dB, dC = (hb.DeviceArray(handle, X) for X in (A, B, C))
    alpha = (0.5 + 1j) if kind in "cz" else 0.5
    beta = (1 - 0.5j) if kind in "cz" else 2.0
    s = hb.gemm_strided_batched(handle, 1, 0, M, N, K, alpha, dA, K, sA, dB, K, sB, beta, dC, M,
                                sC, batch)
    assert s == hb.HCBLAS_STATUS_SUCCESS
    got = dC.download()
    for i in range(batch):
        Ai, Bi, Ci = A[i * sA:(i + 1) * sA], B[i * sB:(i + 1) * sB], C[i * sC:(i + 1) * sC]
        _, ref = O.gemm(O.COL, 1, 0, M, N, K, alpha, Ai, K, Bi, K, beta, Ci, M)
        gv = O.view_c(got[i * sC:(i + 1) * sC], O.COL, M, N, M)
        err = np.linalg.norm((gv.astype(ref.dtype) - ref).reshape(-1))
        bound = error_bound(kind, O.COL, 1, 0, M, N, K, alpha, Ai, K, 0, Bi, K, 0, beta, Ci, M,
                            0, ref)
        assert err <= bound, (i, err, bound)
        # the stride gaps are untouched
        assert np.array_equal(got[i * sC + M * N:(i + 1) * sC], C[i * sC + M * N:(i + 1) * sC])


def test_class_batched_row_major(handle):
    """Row-major pointer-array batch (a silent no-op in the reference,
    sgemm_array_wrapper.cpp:113-151) computes here, with batch offsets."""
    rng = np.random.default_rng(9)
    M, N, K, batch = 33, 20, 17, 5
    L = hb.lib()
    A = rng.standard_normal(M * K * batch + 8).astype(np.float32)
    B = rng.standard_normal(K * N * batch + 8).astype(np.float32)
    C = rng.standard_normal(M * N * batch + 8).astype(np.float32)
    dA, dB, dC = (hb.DeviceArray(handle, X) for X in (A, B, C))
    pA = _ptr_array(handle, [dA.ptr] * batch)
    pB = _ptr_array(handle, [dB.ptr] * batch)
    pC = _ptr_array(handle, [dC.ptr] * batch)
    al = np.array([1.5], np.float32)
    be = np.array([-0.5], np.float32)
    rc = L.hcblasLibGemmBatched(handle, 0, 0, b"n", b"t", M, N, K, al.ctypes.data, pA.ptr, K,
                                M * K, pB.ptr, K, K * N, be.ctypes.data, pC.ptr, N, M * N, 3, 2,
                                1, batch)
    assert rc == 0
    got = dC.download()
    for i in range(batch):
        _, ref = O.gemm(O.ROW, 0, 1, M, N, K, 1.5, A[i * M * K:], K, B[i * K * N:], K, -0.5,
                        C[i * M * N:], N, 3, 2, 1)
        gv = O.view_c(got[i * M * N:], O.ROW, M, N, N, 1)
        assert np.linalg.norm(gv - ref) <= gamma("s", K) * 10 * np.linalg.norm(ref)


def test_set_get_matrix_strided(handle):
    rng = np.random.default_rng(3)
    rows, cols, lda, ldb = 37, 11, 40, 45
    A = rng.standard_normal(lda * cols)
    dB = hb.am_alloc(8 * ldb * cols)
    zero = np.zeros(ldb * cols)
    assert hb.hcblasSetMatrix(handle, ldb * cols, 1, 8, zero.ctypes.data, ldb * cols, dB,
                              ldb * cols) == 0
    assert hb.hcblasSetMatrix(handle, rows, cols, 8, A.ctypes.data, lda, dB, ldb) == 0
    out = np.full(lda * cols, -1.0)
    assert hb.hcblasGetMatrix(handle, rows, cols, 8, dB, ldb, out.ctypes.data, lda) == 0
    for j in range(cols):
        assert np.array_equal(out[j * lda:j * lda + rows], A[j * lda:j * lda + rows])
        assert np.all(out[j * lda + rows:(j + 1) * lda] == -1.0)
    assert hb.hcblasSetMatrix(handle, -1, cols, 8, A.ctypes.data, lda, dB, ldb) == \
        hb.HCBLAS_STATUS_INVALID_VALUE
    hb.am_free(dB)


def test_set_get_matrix_async_on_a_stream(handle):
    """The asynchronous copies enqueue on the given stream (pinned host
    memory) and complete once that stream is synchronised; bad sizes are
    rejected before anything is enqueued."""
    import torch
    rng = np.random.default_rng(4)
    rows, cols, lda, ldb = 300, 70, 301, 304
    pin = lambda n: torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
    A = pin(lda * cols)
    A[:] = rng.standard_normal(lda * cols)
    out = pin(lda * cols)
    out[:] = -1.0
    dB = hb.am_alloc(8 * ldb * cols)
    s = torch.cuda.Stream()
    assert hb.hcblasSetMatrixAsync(handle, rows, cols, 8, A.ctypes.data, lda, dB, ldb,
                                   s.cuda_stream) == 0
    assert hb.hcblasGetMatrixAsync(handle, rows, cols, 8, dB, ldb, out.ctypes.data, lda,
                                   s.cuda_stream) == 0
    s.synchronize()
    for j in range(cols):
        assert np.array_equal(out[j * lda:j * lda + rows], A[j * lda:j * lda + rows])
        assert np.all(out[j * lda + rows:(j + 1) * lda] == -1.0)
    assert hb.hcblasSetMatrixAsync(handle, rows, -1, 8, A.ctypes.data, lda, dB, ldb,
                                   s.cuda_stream) == hb.HCBLAS_STATUS_INVALID_VALUE
    hb.am_free(dB)


@pytest.mark.parametrize("ta,tb", [(0, 0), (0, 1), (1, 0), (1, 1)])
def test_dgemm_dmma_matches_fma_path(handle, ta, tb):
    """Native DGEMM: the FP64 tensor path (mma.sync .f64, the default) and
    the CUDA-core DFMA path (tuning knob "dgemm_dmma" = 0) both stay within
    gamma_{K+2}(f64) of the double-double oracle on ragged shapes with
    padded leading dimensions and offsets; integer data gives exact results
    on both."""
    rng = np.random.default_rng(70 + 2 * ta + tb)
    M, N, K = 301, 259, 517
    lda = (M if ta == 0 else K) + 3
    ldb = (K if tb == 0 else N) + 5
    ldc = M + 1
    A = rng.standard_normal(lda * (K if ta == 0 else M) + 7)
    B = rng.standard_normal(ldb * (N if tb == 0 else K) + 7)
    C = rng.standard_normal(ldc * N + 7)
    outs = {}
    for dmma in (1, 0):
        assert hb.set_tuning(handle, "dgemm_dmma", dmma) == 0
        try:
            dA, dB, dC = (hb.DeviceArray(handle, X) for X in (A, B, C))
            s = hb.lib_gemm(handle, O.COL, "nt"[ta], "nt"[tb], M, N, K, 1.25, dA, lda, dB, ldb,
                            -0.5, dC, ldc, 3, 5, 7)
            assert s == 0
            outs[hb.hcblasGetLastPath(handle)] = dC.download()
        finally:
            hb.set_tuning(handle, "dgemm_dmma", 1)
    assert set(outs) == {"dmma.d.128x128", "simt.d.64x64"} or \
        set(outs) == {"dmma.d.128x128", "simt.d.128x128"}, set(outs)
    _, ref = O.gemm(O.COL, ta, tb, M, N, K, 1.25, A, lda, B, ldb, -0.5, C, ldc, 3, 5, 7)
    Ad = np.abs(op_dense(A, O.COL, ta, M, K, lda, 3))
    Bd = np.abs(op_dense(B, O.COL, tb, K, N, ldb, 5))
    Cd = np.abs(O.view_c(C, O.COL, M, N, ldc, 7))
    bound = gamma("d", K) * np.linalg.norm(1.25 * (Ad @ Bd) + 0.5 * Cd)
    for path, got in outs.items():
        assert np.linalg.norm(O.view_c(got, O.COL, M, N, ldc, 7) - ref) <= bound, path
        # outside the M x N window (ld padding, the offset) nothing changed
        assert np.array_equal(got[:7], C[:7]), path
    # integer data: exact on both paths
    Ai = rng.integers(-50, 51, A.size).astype(np.float64)
    Bi = rng.integers(-50, 51, B.size).astype(np.float64)
    Ci = rng.integers(-50, 51, C.size).astype(np.float64)
    exp, _ = O.gemm(O.COL, ta, tb, M, N, K, 2.0, Ai, lda, Bi, ldb, 1.0, Ci, ldc, 3, 5, 7,
                    want_ref=False)
    for dmma in (1, 0):
        assert hb.set_tuning(handle, "dgemm_dmma", dmma) == 0
        try:
            dA, dB, dC = (hb.DeviceArray(handle, X) for X in (Ai, Bi, Ci))
            assert hb.lib_gemm(handle, O.COL, "nt"[ta], "nt"[tb], M, N, K, 2.0, dA, lda, dB,
                               ldb, 1.0, dC, ldc, 3, 5, 7) == 0
            assert np.array_equal(dC.download(), exp), dmma
        finally:
            hb.set_tuning(handle, "dgemm_dmma", 1)


@pytest.mark.parametrize("ta,tb", [(2, 0), (0, 2), (1, 2), (2, 1)])
def test_zgemm_dmma_matches_fma_path(handle, ta, tb):
    """Native ZGEMM on the FP64 tensor path (four real DMMA products per
    fragment set) against the CUDA-core path and the double-double oracle,
    conjugate transposes included; integer data exact on both."""
    rng = np.random.default_rng(80 + 3 * ta + tb)
    M, N, K = 200, 150, 333
    lda = (M if ta == 0 else K) + 2
    ldb = (K if tb == 0 else N) + 1
    ldc = M + 3
    mk = lambda n: (rng.standard_normal(n) + 1j * rng.standard_normal(n))
    A, B, C = mk(lda * (K if ta == 0 else M) + 4), mk(ldb * (N if tb == 0 else K) + 4), \
        mk(ldc * N + 4)
    alpha, beta = (0.75 - 0.5j), (0.25 + 1j)
    outs = {}
    for dmma in (1, 0):
        assert hb.set_tuning(handle, "dgemm_dmma", dmma) == 0
        try:
            dA, dB, dC = (hb.DeviceArray(handle, X) for X in (A, B, C))
            assert hb.lib_gemm(handle, O.COL, "ntc"[ta], "ntc"[tb], M, N, K, alpha, dA, lda, dB,
                               ldb, beta, dC, ldc, 1, 2, 3) == 0
            outs[hb.hcblasGetLastPath(handle)] = dC.download()
        finally:
            hb.set_tuning(handle, "dgemm_dmma", 1)
    assert "dmma.z.128x64" in outs and any(k.startswith("simt.z") for k in outs), set(outs)
    _, ref = O.gemm(O.COL, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, 1, 2, 3)
    Ad = np.abs(op_dense(A, O.COL, ta, M, K, lda, 1))
    Bd = np.abs(op_dense(B, O.COL, tb, K, N, ldb, 2))
    Cd = np.abs(O.view_c(C, O.COL, M, N, ldc, 3))
    bound = gamma("z", K) * np.linalg.norm(abs(alpha) * (Ad @ Bd) + abs(beta) * Cd)
    for path, got in outs.items():
        assert np.linalg.norm(O.view_c(got, O.COL, M, N, ldc, 3) - ref) <= bound, path
        assert np.array_equal(got[:3], C[:3]), path
    ints = lambda n: (rng.integers(-30, 31, n) + 1j * rng.integers(-30, 31, n)).astype(np.complex128)
    Ai, Bi, Ci = ints(A.size), ints(B.size), ints(C.size)
    exp, _ = O.gemm(O.COL, ta, tb, M, N, K, (2 - 1j), Ai, lda, Bi, ldb, (1 + 1j), Ci, ldc, 1, 2,
                    3, want_ref=False)
    for dmma in (1, 0):
        assert hb.set_tuning(handle, "dgemm_dmma", dmma) == 0
        try:
            dA, dB, dC = (hb.DeviceArray(handle, X) for X in (Ai, Bi, Ci))
            assert hb.lib_gemm(handle, O.COL, "ntc"[ta], "ntc"[tb], M, N, K, (2 - 1j), dA, lda,
                               dB, ldb, (1 + 1j), dC, ldc, 1, 2, 3) == 0
            assert np.array_equal(dC.download(), exp), dmma
        finally:
            hb.set_tuning(handle, "dgemm_dmma", 1)
