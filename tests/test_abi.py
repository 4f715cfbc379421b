"""The C-ABI shared library: it loads, exports every entry point the public
headers declare, and applies the reference's host-side status rules without
touching a GPU (lib/src/hcblas.cpp:1304-1327, 72-80).  Also compiles a
reference-style C++ caller against include/ to prove the drop-in headers
build unchanged, and checks the hc::half conversions in hc_compat.h.
"""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import hcblas_b200 as hb
from tests.conftest import ROOT

INCLUDE = os.path.join(ROOT, "include")


def declared_functions():
    names = set()
    for h in ("hcblas.h", "hc_compat.h"):
        text = open(os.path.join(INCLUDE, h)).read()
        # C declarations only: strip the C++-only tail (inline overloads)
        text = text.split("#ifdef __cplusplus\n} /* extern \"C\" */")[0]
        for m in re.finditer(r"^(?:hcblasStatus_t|int|long long|void \*|const char \*)\s*(\w+)\(",
                             text, re.M):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol(built_lib):
    names = declared_functions()
    assert len(names) >= 40, names
    L = ctypes.CDLL(built_lib)
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert not missing, missing
    assert set(hb.EXPORTED) <= names


def test_status_rules_without_gpu(built_lib):
    L = hb.lib()
    one = np.ones(1, np.float32)
    p = one.ctypes.data
    # NULL handle -> NOT_INITIALIZED, checked before anything else
    assert L.hcblasSgemm(None, 0, 0, 4, 4, 4, p, p, 4, p, 4, p, p, 4) == hb.HCBLAS_STATUS_NOT_INITIALIZED
    assert L.hcblasSgemm(None, 0, 0, -1, 4, 4, p, p, 4, p, 4, p, p, 4) == hb.HCBLAS_STATUS_NOT_INITIALIZED
    assert L.hcblasDgemmBatched(None, 0, 0, 4, 4, 4, p, None, 4, None, 4, p, None, 4, 2) == \
        hb.HCBLAS_STATUS_NOT_INITIALIZED
    h = ctypes.c_void_p(None)
    assert L.hcblasDestroy(ctypes.byref(h)) == hb.HCBLAS_STATUS_NOT_INITIALIZED
    assert L.hcblasDestroy(None) == hb.HCBLAS_STATUS_NOT_INITIALIZED
    assert L.hcblasSetMatrix(None, 2, 2, 4, p, 2, p, 2) == hb.HCBLAS_STATUS_NOT_INITIALIZED
    assert L.hcblasSetMathMode(None, 1, 3) == hb.HCBLAS_STATUS_NOT_INITIALIZED
    assert L.hcblasLibSgemm(None, 1, b"n", b"n", 4, 4, 4, p, p, 4, p, 4, p, p, 4, 0, 0, 0) == -1
    assert hb.hcblasGetLastPath(None) == "none"
    assert b"sm_100a" in L.hcblasGetVersionString()


def test_create_without_device_fails_cleanly(built_lib):
    if hb.lib().hcblas_device_count() > 0:
        pytest.skip("a GPU is present")
    s, h = hb.hcblasCreate(0)
    assert s == hb.HCBLAS_STATUS_NOT_INITIALIZED and not h


CPP_CALLER = r"""
#include "hcblas.h"
#include "hcblaslib.h"
#include <cstdio>
#include <cstdlib>
#include <cstring>
// A reference-style caller: the statements below have the shape of
// test/unit/hcblas_sgemm.cpp:34-80 and test/unit-api/test-blas.cpp:1851-1930.
int main(int argc, char** argv) {
  if (argc > 1 && std::strcmp(argv[1], "half") == 0) {
    for (unsigned b = 0; b < 65536; ++b) {
      float f = hc::half::to_float((uint16_t)b);
      unsigned u; std::memcpy(&u, &f, 4);
      std::printf("%08x\n", u);
    }
    return 0;
  }
  if (argc > 1 && std::strcmp(argv[1], "round") == 0) {
    unsigned u;
    while (std::scanf("%x", &u) == 1) {
      float f; std::memcpy(&f, &u, 4);
      std::printf("%04x\n", (unsigned)hc::half::from_float(f));
    }
    return 0;
  }
  hc::accelerator accl;
  hc::accelerator_view av = accl.get_default_view();
  hcblasHandle_t handle = NULL;
  hcblasStatus_t status = hcblasCreate(&handle, &av);
  if (status != HCBLAS_STATUS_SUCCESS) { std::printf("create=%d\n", (int)status); return 0; }
  Hcblaslibrary hc(&av);
  std::printf("order=%d initialized=%d\n", (int)handle->Order, (int)hc.initialized);
  int M = 189, N = 9, K = 19;
  float alpha = 1, beta = 1;
  float* devA = hc::am_alloc(sizeof(float) * M * K, hc.currentAccl, 0);
  float* devB = hc::am_alloc(sizeof(float) * K * N, hc.currentAccl, 0);
  float* devC = hc::am_alloc(sizeof(float) * M * N, hc.currentAccl, 0);
  hcblasStatus st = hc.hcblas_sgemm(hc.currentAcclView, ColMajor, NoTrans, Trans, M, N, K, alpha,
                                    devA, M, devB, N, beta, devC, M, 0, 0, 0);
  std::printf("status=%d\n", (int)st);
  hc::am_free(devA); hc::am_free(devB); hc::am_free(devC);
  hcblasDestroy(&handle);
  return 0;
}
"""


@pytest.fixture(scope="module")
def cpp_caller(built_lib, tmp_path_factory):
    d = tmp_path_factory.mktemp("cpp")
    src = d / "caller.cpp"
    src.write_text(CPP_CALLER)
    exe = d / "caller"
    libdir = os.path.dirname(built_lib)
    cmd = ["/usr/bin/g++", "-std=c++17", "-O1", f"-I{INCLUDE}", str(src), "-o", str(exe),
           f"-L{libdir}", "-lhcblas", f"-Wl,-rpath,{libdir}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return str(exe)


def test_reference_style_cpp_caller_compiles_and_links(cpp_caller):
    r = subprocess.run([cpp_caller], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    if hb.lib().hcblas_device_count() == 0:
        assert "create=1" in r.stdout


def test_hc_half_to_float_all_encodings(cpp_caller):
    r = subprocess.run([cpp_caller, "half"], capture_output=True, text=True, timeout=120)
    got = np.array([int(x, 16) for x in r.stdout.split()], dtype=np.uint32).view(np.float32)
    ref = np.arange(65536, dtype=np.uint16).view(np.float16).astype(np.float32)
    nan = np.isnan(ref)
    assert np.array_equal(np.isnan(got), nan)
    assert np.array_equal(got[~nan], ref[~nan])


def test_hc_half_from_float_rounding(cpp_caller):
    rng = np.random.default_rng(11)
    xs = np.concatenate([
        (rng.standard_normal(20000) * 10.0 ** rng.integers(-9, 6, 20000)).astype(np.float32),
        np.arange(65536, dtype=np.uint16).view(np.float16).astype(np.float32)[::13],
        np.array([65504, 65519.99, 65520, 1e9, 2 ** -25, 2 ** -24, 1.5 * 2 ** -25,
                  2 ** -14, 0.0, -0.0, np.inf, -np.inf], dtype=np.float32)])
    xs = xs[np.isfinite(xs) | np.isinf(xs)]
    inp = "\n".join(f"{v:08x}" for v in xs.view(np.uint32))
    r = subprocess.run([cpp_caller, "round"], input=inp, capture_output=True, text=True,
                       timeout=120)
    got = np.array([int(x, 16) for x in r.stdout.split()], dtype=np.uint16)
    with np.errstate(over="ignore"):
        ref = xs.astype(np.float16).view(np.uint16)
    assert np.array_equal(got, ref)


def hip_declared():
    text = open(os.path.join(INCLUDE, "hipblas.h")).read()
    return set(m.group(1) for m in re.finditer(r"^hipblasStatus_t\s+(\w+)\(", text, re.M))


def test_hipblas_layer_exports_and_status_rules(built_lib):
    """The hipBLAS-style layer (reference lib/src/hcc_detail/hipblas.cpp):
    every declared entry point is exported; status rules hold without a GPU;
    hipblasStatus_t keeps the reference's numbering (ARCH_MISMATCH at 4)."""
    names = hip_declared()
    assert len(names) >= 20, names
    L = ctypes.CDLL(built_lib)
    assert not [n for n in sorted(names) if not hasattr(L, n)]
    L.hipblasCreate.argtypes = [ctypes.c_void_p]
    L.hipblasCreate.restype = ctypes.c_int
    L.hipblasDestroy.argtypes = [ctypes.c_void_p]
    L.hipblasDestroy.restype = ctypes.c_int
    assert L.hipblasCreate(None) == 3            # INVALID_VALUE
    assert L.hipblasDestroy(None) == 1           # NOT_INITIALIZED
    f = L.hipblasSgemm
    vp, ci = ctypes.c_void_p, ctypes.c_int
    f.argtypes = [vp, ci, ci, ci, ci, ci, vp, vp, ci, vp, ci, vp, vp, ci]
    f.restype = ci
    one = np.ones(1, np.float32)
    p = one.ctypes.data
    assert f(None, 0, 0, 4, 4, 4, p, p, 4, p, 4, p, p, 4) == 1   # NULL handle
    text = open(os.path.join(INCLUDE, "hipblas.h")).read()
    assert "HIPBLAS_STATUS_ARCH_MISMATCH = 4" in text
    assert "HIPBLAS_STATUS_EXECUTION_FAILED = 6" in text
