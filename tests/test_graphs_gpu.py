"""CUDA-graph replay of repeated calls (tuning knob "graphs"): a replayed call
must compute exactly what the eager call computes, follow new matrix
contents, and be dropped when the workspace it captured moves."""
import numpy as np
import pytest
import torch

import hcblas_b200 as hb
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture
def stream_handle(built_lib):
    st = torch.cuda.Stream()
    s, h = hb.hcblasCreate(0, st.cuda_stream)
    assert s == 0
    assert hb.set_tuning(h, "graphs", 1) == 0
    yield h, st
    hb.hcblasDestroy(h)


def dgemm(h, dA, dB, dC, M, N, K):
    one, zero = np.array([1.0]), np.array([0.0])
    return hb.lib().hcblasDgemm(h, hb.HCBLAS_OP_N, hb.HCBLAS_OP_T, M, N, K, one.ctypes.data,
                                dA.ptr, M, dB.ptr, N, zero.ctypes.data, dC.ptr, M)


@pytest.mark.parametrize("mode,param", [(hb.HCBLAS_MATH_OZAKI_CRT, 14), (hb.HCBLAS_MATH_NATIVE, 0)])
def test_replay_matches_eager_and_follows_data(stream_handle, mode, param):
    h, st = stream_handle
    assert hb.hcblasSetMathMode(h, mode, param) == 0
    rng = np.random.default_rng(17)
    M, N, K = 384, 256, 512
    A, B = rng.standard_normal(M * K), rng.standard_normal(N * K)
    dA, dB = hb.DeviceArray(h, A), hb.DeviceArray(h, B)
    dC = hb.DeviceArray(h, nbytes=8 * M * N, dtype=np.float64)
    assert dgemm(h, dA, dB, dC, M, N, K) == 0  # eager + capture
    torch.cuda.synchronize()
    eager = dC.download()
    n0 = hb.kernel_launch_count()
    assert dgemm(h, dA, dB, dC, M, N, K) == 0  # replay
    torch.cuda.synchronize()
    replay_launches = hb.kernel_launch_count() - n0
    assert replay_launches >= 1
    assert np.array_equal(dC.download(), eager)
    A2 = rng.standard_normal(M * K)
    dA.upload(A2)
    assert dgemm(h, dA, dB, dC, M, N, K) == 0  # replay on new data
    torch.cuda.synchronize()
    _, ref = O.gemm(O.COL, 0, 1, M, N, K, 1.0, A2, M, B, N, 0.0, np.zeros(M * N), M)
    assert O.normwise_rel_error(O.view_c(dC.download(), O.COL, M, N, M), ref) < 1e-14
    assert hb.device_error(h) == 0


def test_workspace_growth_drops_graphs(stream_handle):
    h, st = stream_handle
    assert hb.hcblasSetMathMode(h, hb.HCBLAS_MATH_OZAKI_CRT, 14) == 0
    rng = np.random.default_rng(18)
    small = (128, 128, 128)
    big = (1024, 1024, 2048)  # needs a larger workspace than the small call
    arrs = {}
    for shape in (small, big):
        M, N, K = shape
        A, B = rng.standard_normal(M * K), rng.standard_normal(N * K)
        arrs[shape] = (A, B, hb.DeviceArray(h, A), hb.DeviceArray(h, B),
                       hb.DeviceArray(h, nbytes=8 * M * N, dtype=np.float64))
    for shape in (small, small, big, small):
        M, N, K = shape
        A, B, dA, dB, dC = arrs[shape]
        assert dgemm(h, dA, dB, dC, M, N, K) == 0
        torch.cuda.synchronize()
        _, ref = O.gemm(O.COL, 0, 1, M, N, K, 1.0, A, M, B, N, 0.0, np.zeros(M * N), M)
        assert O.normwise_rel_error(O.view_c(dC.download(), O.COL, M, N, M), ref) < 1e-14, shape
    assert hb.device_error(h) == 0


@pytest.mark.parametrize("graphs", [0, 1])
def test_crt_second_stream_matches_one_stream(built_lib, graphs):
    """The CRT DGEMM's op(B) passes on the handle's second stream (the
    "aux_stream" knob, forked and joined by events, also inside a captured
    graph) give the same words as every launch on the call's stream, on a
    user stream and on the legacy default stream."""
    rng = np.random.default_rng(19)
    M, N, K = 520, 300, 700
    A, B = rng.standard_normal(M * K), rng.standard_normal(N * K)
    out = {}
    for name, st in (("user", torch.cuda.Stream()), ("legacy", None)):
        s, h = hb.hcblasCreate(0, st.cuda_stream if st is not None else None)
        assert s == 0
        try:
            assert hb.set_tuning(h, "graphs", graphs if st is not None else 0) == 0
            assert hb.hcblasSetMathMode(h, hb.HCBLAS_MATH_OZAKI_CRT, 14) == 0
            dA, dB = hb.DeviceArray(h, A), hb.DeviceArray(h, B)
            for aux in (1, 0, 1):
                assert hb.set_tuning(h, "aux_stream", aux) == 0
                dC = hb.DeviceArray(h, nbytes=8 * M * N, dtype=np.float64)
                for _ in range(2):  # eager (+ capture), then replay when graphs are on
                    assert dgemm(h, dA, dB, dC, M, N, K) == 0
                torch.cuda.synchronize()
                assert hb.device_error(h) == 0
                out[(name, aux, len(out))] = dC.download()
        finally:
            hb.hcblasDestroy(h)
    ref = next(iter(out.values()))
    for k, v in out.items():
        assert np.array_equal(v, ref), k
    _, oracle = O.gemm(O.COL, 0, 1, M, N, K, 1.0, A, M, B, N, 0.0, np.zeros(M * N), M)
    assert O.normwise_rel_error(O.view_c(ref, O.COL, M, N, M), oracle) < 1e-14
