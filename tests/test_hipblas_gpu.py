"""The hipBLAS-style layer on a B200: handle and stream plumbing, host copies,
and every GEMM entry point against the CPU oracle (same tolerances as the
hcblas entry points, via error_bound)."""
import ctypes

import numpy as np
import pytest

import hcblas_b200 as hb
from oracle import oracle as O
from tests.test_gemm_gpu import NP, error_bound, make_case

pytestmark = pytest.mark.gpu

vp, ci, cll = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong


@pytest.fixture(scope="module")
def hip(built_lib):
    L = hb.lib()
    L.hipblasCreate.argtypes = [ctypes.POINTER(vp)]
    L.hipblasCreate.restype = ci
    L.hipblasDestroy.argtypes = [vp]
    L.hipblasDestroy.restype = ci
    L.hipblasSetStream.argtypes = [vp, vp]
    L.hipblasSetStream.restype = ci
    L.hipblasGetStream.argtypes = [vp, ctypes.POINTER(vp)]
    L.hipblasGetStream.restype = ci
    for n in ("hipblasSetMatrix", "hipblasGetMatrix"):
        getattr(L, n).argtypes = [ci, ci, ci, vp, ci, vp, ci]
        getattr(L, n).restype = ci
    for p in "SDCZH":
        f = getattr(L, f"hipblas{p}gemm")
        f.argtypes = [vp, ci, ci, ci, ci, ci, vp, vp, ci, vp, ci, vp, vp, ci]
        f.restype = ci
    for p in "SDCZ":
        f = getattr(L, f"hipblas{p}gemmBatched")
        f.argtypes = [vp, ci, ci, ci, ci, ci, vp, vp, ci, vp, ci, vp, vp, ci, ci]
        f.restype = ci
    for p in "SDH":
        f = getattr(L, f"hipblas{p}gemmStridedBatched")
        f.argtypes = [vp, ci, ci, ci, ci, ci, vp, vp, ci, cll, vp, ci, cll, vp, vp, ci, cll, ci]
        f.restype = ci
    h = vp()
    assert L.hipblasCreate(ctypes.byref(h)) == 0
    yield L, h.value
    assert L.hipblasDestroy(h.value) == 0


def test_stream_roundtrip_and_host_copies(hip, handle):
    L, h = hip
    import torch
    st = torch.cuda.Stream()
    assert L.hipblasSetStream(h, st.cuda_stream) == 0
    got = vp()
    assert L.hipblasGetStream(h, ctypes.byref(got)) == 0
    assert got.value == st.cuda_stream
    assert L.hipblasSetStream(h, None) == 0
    rows, cols, lda = 37, 21, 40
    A = np.random.default_rng(0).standard_normal(lda * cols)
    d = hb.DeviceArray(handle, nbytes=8 * rows * cols, dtype=np.float64)
    assert L.hipblasSetMatrix(rows, cols, 8, A.ctypes.data, lda, d.ptr, rows) == 0
    back = np.zeros(lda * cols)
    assert L.hipblasGetMatrix(rows, cols, 8, d.ptr, rows, back.ctypes.data, lda) == 0
    assert np.array_equal(back.reshape(cols, lda)[:, :rows], A.reshape(cols, lda)[:, :rows])


@pytest.mark.parametrize("kind", "sdczh")
@pytest.mark.parametrize("ta,tb", [(0, 0), (1, 2), (2, 1)])
def test_gemm_vs_oracle(hip, handle, kind, ta, tb):
    L, h = hip
    rng = np.random.default_rng(10 + ta * 3 + tb)
    M, N, K = 70, 45, 33
    A, lda, B, ldb, C, ldc = make_case(rng, kind, O.COL, ta, tb, M, N, K)
    dA, dB, dC = (hb.DeviceArray(handle, X) for X in (A, B, C))
    alpha = (0.5 + 1j) if kind in "cz" else 0.5
    beta = (1 - 0.5j) if kind in "cz" else 2.0
    al, be = hb.scalar_bytes(NP[kind], alpha), hb.scalar_bytes(NP[kind], beta)
    f = getattr(L, f"hipblas{kind.upper()}gemm")
    assert f(h, ta, tb, M, N, K, al.ctypes.data, dA.ptr, lda, dB.ptr, ldb, be.ctypes.data,
             dC.ptr, ldc) == 0
    _, ref = O.gemm(O.COL, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc)
    gv = O.view_c(dC.download(), O.COL, M, N, ldc)
    err = np.linalg.norm((gv.astype(ref.dtype) - ref).reshape(-1))
    assert err <= error_bound(kind, O.COL, ta, tb, M, N, K, alpha, A, lda, 0, B, ldb, 0, beta, C,
                              ldc, 0, ref)
    # the reference's quick-return rule, in hipBLAS numbering
    assert f(h, ta, tb, 0, N, K, al.ctypes.data, dA.ptr, lda, dB.ptr, ldb, be.ctypes.data,
             dC.ptr, ldc) == 6
    assert f(h, 7, tb, M, N, K, al.ctypes.data, dA.ptr, lda, dB.ptr, ldb, be.ctypes.data,
             dC.ptr, ldc) == 3


def test_batched_and_strided(hip, handle):
    L, h = hip
    rng = np.random.default_rng(3)
    M, N, K, batch = 48, 40, 24, 5
    As = [rng.standard_normal(M * K) for _ in range(batch)]
    Bs = [rng.standard_normal(K * N) for _ in range(batch)]
    Cs = [rng.standard_normal(M * N) for _ in range(batch)]
    dAs, dBs, dCs = ([hb.DeviceArray(handle, X) for X in L_] for L_ in (As, Bs, Cs))
    ptrs = [np.array([d.ptr for d in ds], dtype=np.uint64) for ds in (dAs, dBs, dCs)]
    dP = [hb.DeviceArray(handle, p) for p in ptrs]
    one, two = np.array([1.0]), np.array([2.0])
    assert L.hipblasDgemmBatched(h, 0, 0, M, N, K, one.ctypes.data, dP[0].ptr, M, dP[1].ptr, K,
                                 two.ctypes.data, dP[2].ptr, M, batch) == 0
    for i in range(batch):
        _, ref = O.gemm(O.COL, 0, 0, M, N, K, 1.0, As[i], M, Bs[i], K, 2.0, Cs[i], M)
        assert O.normwise_rel_error(O.view_c(dCs[i].download(), O.COL, M, N, M), ref) < 1e-14
    A = np.concatenate(As)
    B = np.concatenate(Bs)
    C = np.concatenate(Cs)
    dA, dB, dC = (hb.DeviceArray(handle, X) for X in (A, B, C))
    assert L.hipblasDgemmStridedBatched(h, 0, 0, M, N, K, one.ctypes.data, dA.ptr, M, M * K,
                                        dB.ptr, K, K * N, two.ctypes.data, dC.ptr, M, M * N,
                                        batch) == 0
    got = dC.download()
    for i in range(batch):
        _, ref = O.gemm(O.COL, 0, 0, M, N, K, 1.0, As[i], M, Bs[i], K, 2.0, Cs[i], M)
        gv = O.view_c(got[i * M * N:(i + 1) * M * N], O.COL, M, N, M)
        assert O.normwise_rel_error(gv, ref) < 1e-14
