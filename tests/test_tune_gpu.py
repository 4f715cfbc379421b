"""Autotuner (tuning knob "autotune"): tuned calls stay correct, decisions are
cached per size bucket and persisted to HCBLAS_AUTOTUNE_CACHE for later
processes."""
import os
import subprocess
import sys

import numpy as np
import pytest

import hcblas_b200 as hb
from oracle import oracle as O
from tests.conftest import ROOT

pytestmark = pytest.mark.gpu


@pytest.fixture
def tuned(handle):
    assert hb.set_tuning(handle, "autotune", 1) == 0
    yield handle
    hb.set_tuning(handle, "autotune", 0)


@pytest.mark.parametrize("kind,mode,param", [("h", 0, 0), ("d", 4, 14), ("s", 0, 0), ("d", 0, 0)])
def test_tuned_calls_are_correct(tuned, kind, mode, param):
    h = tuned
    rng = np.random.default_rng(90)
    M, N, K = 640, 512, 384
    dt = {"h": np.float16, "s": np.float32, "d": np.float64}[kind]
    A = rng.uniform(-1, 1, M * K).astype(dt)
    B = rng.uniform(-1, 1, N * K).astype(dt)
    C = np.zeros(M * N, dtype=dt)
    assert hb.hcblasSetMathMode(h, mode, param) == 0
    try:
        for _ in range(2):  # first call tunes, second uses the cached choice
            dA, dB, dC = (hb.DeviceArray(h, X) for X in (A, B, C))
            assert hb.lib_gemm(h, O.COL, "n", "t", M, N, K, 1.0, dA, M, dB, N, 0.0, dC, M) == 0
            assert hb.device_error(h) == 0
            _, ref = O.gemm(O.COL, 0, 1, M, N, K, 1.0, A, M, B, N, 0.0, C, M)
            err = O.normwise_rel_error(O.view_c(dC.download(), O.COL, M, N, M).astype(np.float64),
                                       ref)
            assert err < {"h": 2e-3, "s": 1e-6, "d": 1e-14}[kind], (kind, err)
    finally:
        hb.hcblasSetMathMode(h, 0, 0)


def test_cache_file_persists_decisions(tmp_path):
    cache = tmp_path / "tune.txt"
    code = (
        "import sys, numpy as np; sys.path.insert(0, %r)\n"
        "import hcblas_b200 as hb\n"
        "from oracle import oracle as O\n"
        "s, h = hb.hcblasCreate(0); hb.set_tuning(h, 'autotune', 1)\n"
        "rng = np.random.default_rng(1); M = N = K = 512\n"
        "A = rng.uniform(-1, 1, M*K).astype(np.float16); B = rng.uniform(-1, 1, N*K).astype(np.float16)\n"
        "dA, dB = hb.DeviceArray(h, A), hb.DeviceArray(h, B)\n"
        "dC = hb.DeviceArray(h, np.zeros(M*N, np.float16))\n"
        "assert hb.lib_gemm(h, O.COL, 'n', 'n', M, N, K, 1.0, dA, M, dB, K, 0.0, dC, M) == 0\n"
        "assert hb.device_error(h) == 0\n" % ROOT)
    env = dict(os.environ, HCBLAS_AUTOTUNE_CACHE=str(cache), HCBLAS_LOG="1")
    r1 = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                        timeout=300)
    assert r1.returncode == 0, r1.stderr
    assert "autotune" in r1.stderr
    lines = cache.read_text().splitlines()
    assert any("hgemm_tc" in ln for ln in lines), lines
    r2 = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                        timeout=300)
    assert r2.returncode == 0, r2.stderr
    assert "autotune" not in r2.stderr  # decided from the file, nothing re-measured
    assert cache.read_text().splitlines() == lines
