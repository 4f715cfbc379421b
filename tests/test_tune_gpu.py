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


@pytest.mark.parametrize("kind,mode,param", [("h", 0, 0), ("s", 0, 0), ("s", 1, 6), ("d", 2, 6)])
def test_tuned_calls_with_beta_update_c_once(tuned, kind, mode, param):
    """beta != 0: the candidates write a scratch matrix, so C = alpha AB + beta C
    is applied exactly once (an extra application would leave beta^2 C)."""
    h = tuned
    rng = np.random.default_rng(91)
    M, N, K = 704, 576, 448
    dt = {"h": np.float16, "s": np.float32, "d": np.float64}[kind]
    A = rng.uniform(-1, 1, M * K).astype(dt)
    B = rng.uniform(-1, 1, N * K).astype(dt)
    ldc = M + 8
    C = rng.uniform(-1, 1, ldc * N).astype(dt)
    alpha, beta = 0.75, 0.5
    assert hb.hcblasSetMathMode(h, mode, param) == 0
    try:
        for _ in range(2):  # first call tunes, second uses the cached choice
            dA, dB, dC = (hb.DeviceArray(h, X) for X in (A, B, C))
            assert hb.lib_gemm(h, O.COL, "n", "t", M, N, K, alpha, dA, M, dB, N, beta, dC,
                               ldc) == 0
            assert hb.device_error(h) == 0
            _, ref = O.gemm(O.COL, 0, 1, M, N, K, alpha, A, M, B, N, beta, C, ldc)
            got = dC.download()
            err = O.normwise_rel_error(O.view_c(got, O.COL, M, N, ldc).astype(np.float64), ref)
            tol = {"h": 2e-3, "s": 1e-6, "d": 1e-10}[kind]  # d: Ozaki-I at 6 slices
            assert err < tol, (kind, mode, err)
            # the rows between M and ldc are not C's: untouched
            assert np.array_equal(got.reshape(N, ldc)[:, M:], C.reshape(N, ldc)[:, M:])
    finally:
        hb.hcblasSetMathMode(h, 0, 0)


def test_grouped_tuned_then_reused_with_beta(tuned):
    from tests.test_grouped_gpu import check, make_problems
    h = tuned
    rng = np.random.default_rng(92)
    probs, host, dev = make_problems(h, rng, 40)
    assert hb.hgemm_grouped(h, probs, 1.0, 0.0) == 0  # tunes (beta == 0)
    assert hb.device_error(h) == 0
    check(host, dev, 1.0, 0.0)
    # C := its beta == 0 result, then the same problems with beta = 0.5
    host2 = [tuple(list(hs[:9]) + [d[2].download()] + [hs[10]]) for hs, d in zip(host, dev)]
    assert hb.hgemm_grouped(h, probs, 1.0, 0.5) == 0  # same plan, tuned configuration
    assert hb.device_error(h) == 0
    check(host2, dev, 1.0, 0.5)


def test_tuning_families_in_log(tmp_path):
    """The autotuner measures the families it covers, beta != 0 included:
    SIMT (beta 0.5), split-BF16 x6 (beta 1), the Ozaki-I slice groups and the
    grouped f16 kernel each leave a decision in the cache file."""
    cache = tmp_path / "tune.txt"
    code = (
        "import sys, numpy as np; sys.path.insert(0, %r)\n"
        "import hcblas_b200 as hb\n"
        "from oracle import oracle as O\n"
        "from tests.test_grouped_gpu import make_problems\n"
        "s, h = hb.hcblasCreate(0); hb.set_tuning(h, 'autotune', 1)\n"
        "rng = np.random.default_rng(2); M, N, K = 512, 384, 320\n"
        "A = rng.uniform(-1, 1, M*K); B = rng.uniform(-1, 1, N*K); C = rng.uniform(-1, 1, M*N)\n"
        "for dt, mode, par, beta in ((np.float32, 0, 0, 0.5), (np.float32, 1, 6, 1.0),\n"
        "                            (np.float64, 2, 6, 0.5)):\n"
        "    assert hb.hcblasSetMathMode(h, mode, par) == 0\n"
        "    dA, dB, dC = (hb.DeviceArray(h, X.astype(dt)) for X in (A, B, C))\n"
        "    assert hb.lib_gemm(h, O.COL, 'n', 'n', M, N, K, 1.0, dA, M, dB, K, beta, dC, M) == 0\n"
        "    _, ref = O.gemm(O.COL, 0, 0, M, N, K, 1.0, A.astype(dt), M, B.astype(dt), K, beta,\n"
        "                    C.astype(dt), M)\n"
        "    err = O.normwise_rel_error(O.view_c(dC.download(), O.COL, M, N, M).astype(np.float64), ref)\n"
        "    assert err < 1e-6, (mode, err)\n"
        "hb.hcblasSetMathMode(h, 0, 0)\n"
        "probs, host, dev = make_problems(h, rng, 24)\n"
        "assert hb.hgemm_grouped(h, probs, 1.0, 0.0) == 0\n"
        "assert hb.device_error(h) == 0\n" % ROOT)
    env = dict(os.environ, HCBLAS_AUTOTUNE_CACHE=str(cache))
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                       timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    text = cache.read_text()
    for fam in ("|simt|", "|split6|", "|ozaki_groups|", "|grouped_h|"):
        assert fam in text, (fam, text)
