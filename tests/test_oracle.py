"""Pin the CPU oracle (oracle/gemm_oracle.c) before trusting it.

The oracle restates CBLAS xGEMM; here it is checked against
  * exact integer answers of the reference tests' own input recipes
    (test/unit/hcblas_dgemm.cpp:201-353, hcblas_cgemm.cpp:216-545),
  * OpenBLAS 0.3.30's CBLAS on seeded float inputs with offsets, padded
    leading dimensions, every order / transpose / conjugate transpose,
  * the reference's SGEMM U[0,2) recipe and its 1e-5 L2 bound
    (test/unit/hcblas_sgemm.cpp:222-261),
  * the C-API all-ones case (test/unit-api/test-blas.cpp:1851-1937),
  * IEEE binary16 conversions (all 65536 encodings),
  * a cancellation case that only double-double accumulation gets right.
No GPU is used.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.conftest import GOLDEN

NP = {"s": np.float32, "d": np.float64, "c": np.complex64, "z": np.complex128}
UNIT = {"s": 2.0 ** -24, "d": 2.0 ** -53, "c": 2.0 ** -24, "z": 2.0 ** -53}


@pytest.mark.parametrize("kind", "sdcz")
def test_int_chain_exact(kind):
    f = np.load(os.path.join(GOLDEN, f"int_chain_{kind}.npz"))
    M, N, K = int(f["M"]), int(f["N"]), int(f["K"])
    A, B, C = f["A"], f["B"], f["C"].copy()
    for step, expect in zip(f["steps"], f["states"]):
        order, ta, tb, lda, ldb, ldc, ar, ai, br, bi = [int(v) for v in step]
        alpha = complex(ar, ai) if kind in "cz" else float(ar)
        beta = complex(br, bi) if kind in "cz" else float(br)
        C, _ = O.gemm(order, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc,
                      want_ref=False)
        assert np.array_equal(C, expect), f"step {step.tolist()}"


def _bound(kind, K):
    u = UNIT[kind]
    return (K + 4) * u / (1 - (K + 4) * u) * (4 if kind in "cz" else 1)


def test_float_cases_vs_openblas():
    f = np.load(os.path.join(GOLDEN, "float_cases.npz"))
    worst = {}
    for row in f["meta"]:
        idx, kind_i, order, ta, tb, M, N, K, lda, ldb, ldc, ao, bo, co = [int(v) for v in row]
        kind = "sdcz"[kind_i]
        key = f"c{idx:03d}"
        A, B, C, out = f[key + "_A"], f[key + "_B"], f[key + "_C"], f[key + "_out"]
        alpha, beta = complex(f[key + "_alpha"][0]), complex(f[key + "_beta"][0])
        if kind in "sd":
            alpha, beta = alpha.real, beta.real
        got, ref = O.gemm(order, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc,
                          ao, bo, co)
        # untouched entries (padding, offsets) must be bit-identical
        mask = np.ones(C.size, bool)
        for n in range(N):
            for m in range(M):
                mask[co + (m + n * ldc if order == O.COL else m * ldc + n)] = False
        assert np.array_equal(got[mask], C[mask], equal_nan=True)
        cv = O.view_c(out, order, M, N, ldc, co)
        assert np.all(np.isfinite(cv)), "beta = 0 must not read the NaN-filled C"
        err = O.normwise_rel_error(cv, ref)
        assert err <= _bound(kind, K), (key, kind, order, ta, tb, err)
        worst[kind] = max(worst.get(kind, 0.0), err)
    assert set(worst) == set("sdcz")


def test_sgemm_recipe_l2():
    f = np.load(os.path.join(GOLDEN, "sgemm_recipe.npz"))
    tol = float(f["tolerance"])
    for i, s in enumerate(f["shapes"]):
        M = N = K = int(s)
        A, B, C, out = f[f"s{i}_A"], f[f"s{i}_B"], f[f"s{i}_C"], f[f"s{i}_out"]
        al, be = (float(v) for v in f[f"s{i}_ab"])
        got, _ = O.gemm(O.COL, 0, 0, M, N, K, al, A, M, B, K, be, C, M)
        assert O.compare_l2fe(out, got) < tol
        assert O.compare_l2fe(out, got) < 1e-6


def test_capi_ones():
    f = np.load(os.path.join(GOLDEN, "capi_ones.npz"))
    M, N, K = int(f["M"]), int(f["N"]), int(f["K"])
    got, _ = O.gemm(O.COL, 0, 0, M, N, K, 2.0, f["A"], M, f["B"], K, 2.0, f["C"], M)
    assert np.array_equal(got, f["out"])


def test_recipe_generators_match_reference_shape_classes():
    # test/unit/test_constants.h evaluates to these under glibc
    assert O.srand_rand(1) % 10 + 1 == 4
    assert O.srand_rand(1) % 89 + 11 == 48
    assert O.srand_rand(1) % 923 + 101 == 777
    assert O.srand_rand(1) % 3071 + 1025 == 1133


def test_half_conversions_all_encodings():
    bits = np.arange(65536, dtype=np.uint16)
    ref = bits.view(np.float16).astype(np.float64)
    got = np.array([O.half_to_double(int(b)) for b in bits])
    nan = np.isnan(ref)
    assert np.array_equal(np.isnan(got), nan)
    assert np.array_equal(got[~nan], ref[~nan])
    rng = np.random.default_rng(7)
    xs = np.concatenate([rng.standard_normal(3000) * 10.0 ** rng.integers(-9, 6, 3000),
                         ref[~nan][::37] + 1e-12, [65519.0, 65520.0, 2 ** -25, 3 * 2 ** -26]])
    for x in xs:
        h = O.double_to_half(float(x))
        assert h == np.float16(x).view(np.uint16), x


def test_double_double_accumulation():
    # row [1e16, 1, -1e16] . col [1, 1, 1] = 1 exactly; plain FP64 gives 0
    A = np.array([1e16, 1.0, -1e16])
    B = np.ones(3)
    C = np.zeros(1)
    got, ref = O.gemm(O.ROW, 0, 0, 1, 1, 3, 1.0, A, 3, B, 1, 0.0, C, 1)
    assert got[0] == 1.0 and ref[0, 0] == 1.0
    assert (A[0] + A[1]) + A[2] == 0.0


def test_beta_zero_does_not_read_c():
    A = np.ones(4, np.float32)
    B = np.ones(4, np.float32)
    C = np.full(1, np.nan, np.float32)
    got, _ = O.gemm(O.COL, 0, 0, 1, 1, 4, 1.0, A, 1, B, 4, 0.0, C, 1)
    assert got[0] == 4.0
