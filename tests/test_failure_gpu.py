"""Failure detection, exercised without faulting the GPU.

* A pipeline wait that runs out: the handle's wait limit is set to 1 ms
  ("wait_timeout_us") and the "inject_timeout" knob arms one HGEMM call whose
  producer withholds the single operand load of a one-tile, one-K-block
  problem with beta == 0 -- the MMA warp's bounded wait on that stage gives
  up, the kernel unwinds (no load, MMA or store is in flight: the problem
  has no other stage and the epilogue reads no C), the call returns, and
  hcblasGetDeviceError reports the code.  The next ordinary call on the same
  handle must be correct.
* A workspace that cannot be had: the "workspace_mb" limit makes the
  split-BF16 path's workspace request fail on the host; the call returns
  EXECUTION_FAILED before launching anything and leaves C untouched.
* A corrupted autotune cache: garbage lines, binary bytes and a well-formed
  key with an out-of-range choice are ignored, the bucket is tuned again and
  the result is correct.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

import hcblas_b200 as hb
from oracle import oracle as O
from tests.conftest import ROOT

pytestmark = pytest.mark.gpu

# tc_common.cuh error codes a withheld load can surface as: the MMA warp's
# wait on the stage, or the epilogue's wait on the accumulator (whichever
# limit runs out first)
TIMEOUT_CODES = {2, 4}


def hgemm_case(rng, M, N, K):
    A = rng.uniform(-1, 1, M * K).astype(np.float16)
    B = rng.uniform(-1, 1, K * N).astype(np.float16)
    return A, B


def run_hgemm(h, A, B, M, N, K, C0):
    dA, dB, dC = hb.DeviceArray(h, A), hb.DeviceArray(h, B), hb.DeviceArray(h, C0)
    rc = hb.lib_gemm(h, O.COL, "n", "n", M, N, K, 1.0, dA, M, dB, K, 0.0, dC, M)
    return rc, dC


@pytest.fixture
def fresh_handle(built_lib):
    s, h = hb.hcblasCreate(0)
    assert s == hb.HCBLAS_STATUS_SUCCESS
    yield h
    hb.hcblasDestroy(h)


def test_pipeline_wait_timeout_is_reported_and_handle_recovers(fresh_handle):
    h = fresh_handle
    rng = np.random.default_rng(41)
    M = N = 128
    K = 64
    A, B = hgemm_case(rng, M, N, K)
    C0 = np.full(M * N, 7.0, np.float16)
    assert hb.set_tuning(h, "wait_timeout_us", 1000) == 0
    try:
        assert hb.set_tuning(h, "inject_timeout", 1) == 0
        rc, dC = run_hgemm(h, A, B, M, N, K, C0)
        assert rc == 0  # the launch succeeded; the failure is reported by the device flag
        assert hb.hcblasGetLastPath(h) == "tc.h.128x128.inject_timeout"
        code = hb.device_error(h)
        assert code in TIMEOUT_CODES, code
        assert hb.device_error(h) == 0  # read and cleared
    finally:
        assert hb.set_tuning(h, "wait_timeout_us", 0) == 0
    # the injection is disarmed after one call; the handle keeps working
    for M2, N2, K2 in [(M, N, K), (320, 200, 504)]:  # leading dimensions TMA can address
        A2, B2 = hgemm_case(rng, M2, N2, K2)
        rc, dC = run_hgemm(h, A2, B2, M2, N2, K2, np.zeros(M2 * N2, np.float16))
        assert rc == 0
        assert hb.device_error(h) == 0
        assert hb.hcblasGetLastPath(h).startswith("tc.h."), hb.hcblasGetLastPath(h)
        _, ref = O.gemm(O.COL, 0, 0, M2, N2, K2, 1.0, A2, M2, B2, K2, 0.0,
                        np.zeros(M2 * N2, np.float16), M2)
        got = O.view_c(dC.download().astype(np.float64), O.COL, M2, N2, M2)
        assert O.normwise_rel_error(got, ref) < 2e-3


def test_injection_refuses_other_shapes(fresh_handle):
    """Only the one-tile, one-K-block, beta == 0 case can be injected (where
    nothing else is in flight); anything else fails on the host."""
    h = fresh_handle
    rng = np.random.default_rng(42)
    M, N, K = 256, 128, 64
    A, B = hgemm_case(rng, M, N, K)
    assert hb.set_tuning(h, "inject_timeout", 1) == 0
    rc, _ = run_hgemm(h, A, B, M, N, K, np.zeros(M * N, np.float16))
    assert rc != 0
    assert hb.device_error(h) == 0
    rc, dC = run_hgemm(h, A, B, M, N, K, np.zeros(M * N, np.float16))
    assert rc == 0 and hb.device_error(h) == 0


def test_workspace_limit_fails_cleanly(fresh_handle):
    h = fresh_handle
    rng = np.random.default_rng(43)
    M = N = K = 1024
    A = rng.standard_normal(M * K).astype(np.float32)
    B = rng.standard_normal(K * N).astype(np.float32)
    C = rng.standard_normal(M * N).astype(np.float32)
    assert hb.hcblasSetMathMode(h, hb.HCBLAS_MATH_SPLIT_BF16, 6) == 0
    try:
        assert hb.set_tuning(h, "workspace_mb", 1) == 0  # the planes need 12 MiB
        dA, dB, dC = hb.DeviceArray(h, A), hb.DeviceArray(h, B), hb.DeviceArray(h, C)
        rc = hb.lib_gemm(h, O.COL, "n", "n", M, N, K, 1.0, dA, M, dB, K, 0.5, dC, M)
        assert rc != 0
        assert np.array_equal(dC.download(), C)  # nothing ran
        assert hb.device_error(h) == 0
        assert hb.set_tuning(h, "workspace_mb", 0) == 0
        rc = hb.lib_gemm(h, O.COL, "n", "n", M, N, K, 1.0, dA, M, dB, K, 0.5, dC, M)
        assert rc == 0 and hb.device_error(h) == 0
        assert hb.hcblasGetLastPath(h).startswith("tc.split_bf16x6")
    finally:
        hb.hcblasSetMathMode(h, hb.HCBLAS_MATH_NATIVE, 0)
        hb.set_tuning(h, "workspace_mb", 0)
    _, ref = O.gemm(O.COL, 0, 0, M, N, K, 1.0, A, M, B, K, 0.5, C, M)
    assert O.normwise_rel_error(O.view_c(dC.download(), O.COL, M, N, M), ref) < 1e-6


def test_corrupted_autotune_cache_is_retuned(tmp_path):
    cache = tmp_path / "tune.txt"
    with open(cache, "wb") as f:
        f.write(b"not a cache line\n\x00\xff\xfe garbage \x01\n 7\nkey-without-choice\n")
        f.write(b"v2|x|drv0|y|0|hgemm_tc|dt4|op00|m9|n9|k9|b0 99\n")
        f.write(os.urandom(64) + b"\n")
    code = (
        "import sys, numpy as np; sys.path.insert(0, %r)\n"
        "import hcblas_b200 as hb\n"
        "from oracle import oracle as O\n"
        "s, h = hb.hcblasCreate(0); hb.set_tuning(h, 'autotune', 1)\n"
        "rng = np.random.default_rng(2); M = N = K = 512\n"
        "A = rng.uniform(-1, 1, M*K).astype(np.float16); B = rng.uniform(-1, 1, N*K).astype(np.float16)\n"
        "dA, dB = hb.DeviceArray(h, A), hb.DeviceArray(h, B)\n"
        "dC = hb.DeviceArray(h, np.zeros(M*N, np.float16))\n"
        "assert hb.lib_gemm(h, O.COL, 'n', 'n', M, N, K, 1.0, dA, M, dB, K, 0.0, dC, M) == 0\n"
        "assert hb.device_error(h) == 0\n"
        "_, ref = O.gemm(O.COL, 0, 0, M, N, K, 1.0, A, M, B, K, 0.0, np.zeros(M*N, np.float16), M)\n"
        "got = O.view_c(dC.download().astype(np.float64), O.COL, M, N, M)\n"
        "assert O.normwise_rel_error(got, ref) < 2e-3\n"
        "print('ok')\n" % ROOT)
    env = dict(os.environ, HCBLAS_AUTOTUNE_CACHE=str(cache), HCBLAS_LOG="1")
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr[-3000:]
    assert "ok" in r.stdout
    assert "autotune" in r.stderr  # nothing usable in the file: tuned again
    tail = cache.read_bytes().splitlines()[-1].decode()
    assert tail.startswith("v2|") and "hgemm_tc" in tail, tail


def test_workspace_follows_stream_switches(fresh_handle):
    """Calls on alternating streams with one handle: each stream is ordered
    after the workspace's last use on the other (no device-wide wait), and
    the workspace grows between them."""
    import torch
    h = fresh_handle
    rng = np.random.default_rng(44)
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    assert hb.hcblasSetMathMode(h, hb.HCBLAS_MATH_SPLIT_BF16, 6) == 0
    try:
        outs = []
        for i, (st, n) in enumerate([(s1, 256), (s2, 512), (s1, 768), (s2, 1024)]):
            A = rng.standard_normal(n * n).astype(np.float32)
            B = rng.standard_normal(n * n).astype(np.float32)
            dA, dB = hb.DeviceArray(h, A), hb.DeviceArray(h, B)
            dC = hb.DeviceArray(h, np.zeros(n * n, np.float32))
            assert hb.hcblasSetStream(h, st.cuda_stream) == 0
            assert hb.lib_gemm(h, O.COL, "n", "t", n, n, n, 1.0, dA, n, dB, n, 0.0, dC, n) == 0
            outs.append((A, B, dC, n))
        torch.cuda.synchronize()
        assert hb.hcblasSetStream(h, 0) == 0
        assert hb.device_error(h) == 0
        for A, B, dC, n in outs:
            _, ref = O.gemm(O.COL, 0, 1, n, n, n, 1.0, A, n, B, n, 0.0,
                            np.zeros(n * n, np.float32), n)
            assert O.normwise_rel_error(O.view_c(dC.download(), O.COL, n, n, n), ref) < 1e-6
    finally:
        hb.hcblasSetStream(h, 0)
        hb.hcblasSetMathMode(h, hb.HCBLAS_MATH_NATIVE, 0)
